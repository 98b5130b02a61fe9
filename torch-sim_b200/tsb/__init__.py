"""tsb -- B200-native (sm_100a) TorchSim classical-potential hot path.

Drop-ins for the reference's plugin API, all running on hand-written CUDA
kernels reached through the C ABI in ``include/tsb.h``:

* ``tsb.neighbors.torchsim_nl``           periodic cell-list neighbour list
* ``tsb.models.LennardJonesModel`` / ``MorseModel`` / ``SoftSphereModel`` /
  ``SoftSphereMultiModel`` / ``LennardJonesMultiModel``  energy, forces, stress
* ``tsb.integrators.nve_step`` / ``nvt_langevin_step`` (+ ``*_init``)
* ``tsb.optimizers.fire_init`` / ``fire_step`` (ASE / VV FIRE, Frechet filter)
* ``tsb.integrators.run_md``              persistent fused batched MD
* ``tsb.ops``                             the same kernels as ``torch.ops.tsb.*``
  operators (CUDA and fake implementations), which the drop-ins call

Submodules are imported lazily; importing ``tsb`` does not load the CUDA library.
"""

import importlib

__version__ = "0.1.0"
_SUBMODULES = ("neighbors", "models", "integrators", "optimizers", "state", "workloads",
               "build", "adjoint", "ops")


def __getattr__(name):
    if name in _SUBMODULES:
        return importlib.import_module(f".{name}", __name__)
    raise AttributeError(name)
