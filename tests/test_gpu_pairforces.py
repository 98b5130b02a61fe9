"""Force-defined pair models on the GPU (particle life, generic PairForcesModel).

* ParticleLifeModel (CUDA kernel, FP64 pair math) and PairForcesModel with an
  asymmetric species-dependent force vs the reference (golden/pairforces.npz):
  forces, stress and per-atom stresses to rtol 1e-10; energies zero.
* Mixed precision (FP32 pair math): max|dF|/max|F| <= 1e-5.
* ParticleLifeMultiModel with an asymmetric species matrix == PairForcesModel
  with the equivalent Python force (both directions of each pair, full-list
  stress weights).
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _state(s, dtype=torch.float64):
    from tsb.state import SimState

    dev = torch.device("cuda")
    T = lambda x, dt=dtype: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    return SimState(positions=T(s["positions"]), masses=T(s["masses"]), cell=T(s["cell"]),
                    pbc=True, atomic_numbers=T(s["atomic_numbers"], torch.int64),
                    system_idx=T(s["system_idx"], torch.int64))


def _cmp(out, ref, rtol):
    for k in ("energy", "forces", "stress", "stresses"):
        np.testing.assert_allclose(out[k].detach().cpu().numpy(), ref[k], rtol=rtol,
                                   atol=1e-12 * max(1.0, np.abs(ref[k]).max()))


def test_particle_life_matches_reference(golden):
    from tsb import models

    s, g = golden["pairforces"]["sys"], golden["pairforces"]["plife"]
    m = models.ParticleLifeModel(sigma=1.0, epsilon=1.0, beta=0.3, cutoff=1.2,
                                 compute_stress=True, per_atom_stresses=True, precision="fp64")
    _cmp(m(_state(s)), g, 1e-10)
    mixed = models.ParticleLifeModel(sigma=1.0, epsilon=1.0, beta=0.3, cutoff=1.2)
    f = mixed(_state(s))["forces"].cpu().numpy()
    assert np.abs(f - g["forces"]).max() / np.abs(g["forces"]).max() < 1e-5


def test_pair_forces_model_matches_reference(golden):
    from tsb import models

    s, g = golden["pairforces"]["sys"], golden["pairforces"]["asym"]

    def asym_force(r, zi, zj):
        return (1.0 + zi.to(r.dtype) - 0.5 * zj.to(r.dtype)) * (1.1 - r)

    m = models.PairForcesModel(asym_force, cutoff=1.1, compute_stress=True,
                               per_atom_stresses=True)
    _cmp(m(_state(s)), g, 1e-10)


def test_particle_life_multi_matches_generic_force_model(golden):
    from tsb import models

    s = golden["pairforces"]["sys"]
    A = np.array([[1.0, -0.5], [0.8, 0.3]])
    beta = np.array([[0.3, 0.25], [0.35, 0.3]])
    sigma = np.array([[1.0, 0.9], [1.0, 0.95]])
    km = models.ParticleLifeMultiModel([1, 2], A, beta, sigma, cutoff=1.2,
                                       compute_stress=True, per_atom_stresses=True,
                                       precision="fp64")
    At, bt, st = (torch.as_tensor(x, device="cuda") for x in (A, beta, sigma))

    def plife(r, zi, zj):
        a, b, sg = At[zi - 1, zj - 1], bt[zi - 1, zj - 1], st[zi - 1, zj - 1]
        inner = torch.where(r < b, r / b - 1.0, torch.zeros_like(r))
        outer = torch.where((r >= b) & (r < sg),
                            a * (1.0 - torch.abs(2.0 * r - 1.0 - b) / (1.0 - b)),
                            torch.zeros_like(r))
        return inner + outer

    gm = models.PairForcesModel(plife, cutoff=1.2, compute_stress=True, per_atom_stresses=True)
    st_ = _state(s)
    a, b = km(st_), gm(st_)
    for k in ("forces", "stress", "stresses"):
        np.testing.assert_allclose(a[k].cpu().numpy(), b[k].cpu().numpy(), rtol=1e-10,
                                   atol=1e-12)
    assert float(a["energy"].abs().max()) == 0.0
