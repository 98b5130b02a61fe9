"""Pairs whose distance lies within FP32 rounding of the cutoff.

A truncated potential has a force step at the cutoff (Morse at 6 A: 0.013
eV/A; Kob-Andersen LJ at 2.5 sigma_ab: ~0.04 eps/sigma), so a pair counted on
one side of the cutoff by FP32 arithmetic and on the other by the FP64
reference changes forces by that step.  Every force path (fused MD kernel,
fused-search model, Verlet-list model) decides inside/outside as the FP64
reference does; the pair arithmetic stays FP32.

Layout: isolated pairs, each at distance rc (1 + delta) with |delta| down to
1e-8 (below FP32 resolution of r^2), half of them across the periodic boundary
(decided through a ghost image in the fused kernel), along an oblique
direction so that every coordinate is rounded.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

DELTAS = (-3e-7, -1e-7, -3e-8, -1e-8, 1e-8, 3e-8, 1e-7, 3e-7)


def _pairs_state(rcs, z_pairs, L=60.0, mass=63.546):
    """One cubic system: pair k at distance rcs[k] * (1 + DELTAS[k % 8])."""
    from tsb.state import state_from_arrays

    u = np.array([1.0, 0.37, 0.21])
    u /= np.linalg.norm(u)
    pos, zs = [], []
    for k, (rc, (za, zb)) in enumerate(zip(rcs, z_pairs)):
        d = rc * (1.0 + DELTAS[k % len(DELTAS)])
        row, col = divmod(k % 16, 4)
        a = np.array([20.123456789 if k < 8 else 1.987654321, 5.0 + 14.0 * col,
                      5.0 + 14.0 * row])
        b = a + (d * u if k < 8 else -d * u)  # k >= 8: partner across x = 0
        pos += [a, b]
        zs += [za, zb]
    pos = np.array(pos)
    d = {"positions": pos, "masses": np.full(len(pos), mass), "cell": np.eye(3)[None] * L,
         "pbc": np.array([True] * 3), "atomic_numbers": np.array(zs, dtype=np.int64),
         "system_idx": np.zeros(len(pos), dtype=np.int64)}
    return state_from_arrays(d, device="cuda")


def _fused_forces(st, model):
    from tsb import integrators
    from tsb.state import MDState

    md = MDState.from_state(st, momenta=torch.zeros_like(st.positions),
                            energy=torch.zeros(st.n_systems, dtype=torch.float64, device="cuda"),
                            forces=torch.zeros_like(st.positions))
    out = integrators.run_md(md, model, 0, integrator="nve", dt=1.0, skin=0.7)
    return out.energy, out.forces


def _check(st, model, ref, step):
    r = ref(st)
    n_in = sum(1 for dl in DELTAS if dl < 0)
    fr = r["forces"]
    # each misclassified pair would move two atoms' forces by `step`
    tol_f = 1e-3 * step
    e, f = _fused_forces(st, model)
    assert (f - fr).abs().max().item() < tol_f, "fused MD kernel"
    # energy: a misclassified Morse pair moves it by |V(6 A)| = 0.0096 eV (the
    # shifted LJ pair energy vanishes at its cutoff: forces carry that check)
    torch.testing.assert_close(e, r["energy"], rtol=0.0, atol=1e-6)
    out = model(st)
    assert (out["forces"] - fr).abs().max().item() < tol_f, "fused-search model"
    torch.testing.assert_close(out["energy"], r["energy"], rtol=0.0, atol=1e-6)
    # inside pairs carry the force step, outside pairs none
    nz = (fr.abs().sum(1) > 0.5 * step).sum().item()
    assert nz == 2 * n_in * (len(fr) // (2 * len(DELTAS)))
    return out


def test_morse_pairs_at_cutoff():
    from tsb import models

    kw = dict(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0, compute_stress=True)
    m = models.MorseModel(**kw)
    ref = models.MorseModel(precision="fp64", **kw)
    st = _pairs_state([6.0] * 16, [(29, 29)] * 16)
    _check(st, m, ref, step=0.013)
    vm = models.VerletListModel(models.MorseModel(**kw), skin=1.0)
    r = ref(st)
    assert (vm(st)["forces"] - r["forces"]).abs().max().item() < 1.3e-5, "Verlet-list model"


def test_kob_andersen_pairs_at_species_cutoffs():
    """Species-dependent cutoffs 2.5 sigma_ab (AA 8.5, AB 6.8, BB 7.48 A)."""
    from tsb import models

    m = models.kob_andersen_model()
    ref = models.kob_andersen_model(precision="fp64")
    kinds = [(1, 1), (1, 2), (2, 2)]
    rc = {(1, 1): 8.5, (1, 2): 6.8, (2, 2): 7.48}
    zp = [kinds[k % 3] for k in range(16)]
    st = _pairs_state([rc[z] for z in zp], zp, L=64.0)
    # LJ force at 2.5 sigma_ab, smallest over the three pair types (eps_BB = 0.5 eps)
    step = 0.5 * 0.0104 * 24 * (1 / 2.5 ** 7 - 2 / 2.5 ** 13) / (0.88 * 3.4)
    _check(st, m, ref, step=step)
