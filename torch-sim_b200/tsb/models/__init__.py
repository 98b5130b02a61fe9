"""Classical pair-potential models on the tsb CUDA kernels."""

from .interface import ModelInterface
from .lennard_jones import (LennardJonesModel, LennardJonesMultiModel,
                            UnbatchedLennardJonesModel, kob_andersen_model)
from .morse import MorseModel
from .pair_potential import PairTableModel
from .particle_life import PairForcesModel, ParticleLifeModel, ParticleLifeMultiModel
from .soft_sphere import SoftSphereModel, SoftSphereMultiModel
from .verlet import VerletListModel

__all__ = ["LennardJonesModel", "LennardJonesMultiModel", "ModelInterface", "MorseModel",
           "PairForcesModel", "ParticleLifeModel", "ParticleLifeMultiModel",
           "PairTableModel", "SoftSphereModel", "SoftSphereMultiModel",
           "UnbatchedLennardJonesModel", "VerletListModel", "kob_andersen_model"]
