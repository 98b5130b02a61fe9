"""Dynamic pruning of the fused kernel's Verlet list (``prune_skin``).

Between list builds the kernel evaluates only the shell pairs that lay within
cutoff + prune_skin at the last pruning, and prunes again when an atom moved
more than prune_skin / 2 since then.  A pair left out must stay outside the
cutoff until the next pruning, so the forces, energies and stresses of a pruned
run are those of the full list:

* forces, energy and stress at the kernel's positions against the FP64 oracle
  after launches of an odd number of steps (so the checks fall at every phase
  of the pruning and list-build cycles), with a narrow pruning skin that prunes
  every few steps: max|dF| / max|F| <= 1e-5, energy rtol 2e-6, stress 1e-5 of
  max|stress|.  A pair within the cutoff that pruning dropped would show as an
  error of F(rc) = 0.013 eV/A (~4e-3 of max|F|);
* trajectories with and without pruning agree to FP32 rounding (only the
  order of the FP32 force sums differs).

Reference: torch_sim/integrators/nvt.py:144-240 (BAOAB), nve.py:74-130,
torch_sim/models/pair_potential.py:200-274, morse.py:23-47.
"""

import numpy as np
import pytest
import torch

from oracle import pair as opair

pytestmark = pytest.mark.gpu

MORSE = (2.866, 0.3429, 1.3588)


def _setup(n_sys, seed, integrator, skin, prune):
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(n_sys, 8, 512, seed=seed)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed + 7
    m = models.MorseModel(sigma=MORSE[0], epsilon=MORSE[1], alpha=MORSE[2], cutoff=6.0)
    kT = 1000.0 * workloads.KB_EV
    dt = 0.002 * workloads.METAL_TIME
    md = integrators.nvt_langevin_init(st, m, kT=kT)
    r = integrators.FusedMD(md, m, integrator=integrator, dt=dt,
                            kT=None if integrator == "nve" else kT,
                            gamma=10.0 / workloads.METAL_TIME
                            if integrator == "nvt_langevin" else None,
                            skin=skin, seed=99 + seed, prune=prune)
    return d, r


def test_pruned_forces_match_oracle_at_every_phase():
    d, r = _setup(20, 11, "nvt_langevin", skin=1.2, prune=0.15)
    assert r.prune == 0.15
    counts = np.bincount(d["system_idx"])
    assert counts.max() >= 400
    tab = opair.single_table(opair.MORSE, *MORSE)
    cell_row = np.transpose(d["cell"], (0, 2, 1))
    pbc = np.ones((cell_row.shape[0], 3), bool)
    worst = 0.0
    for k in range(8):
        r.launch(7)
        torch.cuda.synchronize()
        r.check()
        x = r.x.cpu().numpy()
        ref = opair.pair_forward(opair.MORSE, tab, np.zeros(len(x), int), x, cell_row, pbc,
                                 d["system_idx"], 6.0)
        err = np.abs(r.f.cpu().numpy() - ref["forces"]).max() / np.abs(ref["forces"]).max()
        worst = max(worst, err)
        assert err <= 1e-5, (k, err)
        np.testing.assert_allclose(r.energy.cpu().numpy(), ref["energy"], rtol=2e-6)
        s = r.stress.cpu().numpy()
        assert np.abs(s - ref["stress"]).max() <= 1e-5 * np.abs(ref["stress"]).max()
    print(f"worst force error with pruning: {worst:.2e}")


@pytest.mark.parametrize("prune", [0.2, 0.5])
def test_pruning_does_not_change_the_trajectory(prune):
    out = []
    for pr in (0.0, prune):
        d, r = _setup(12, 12, "nve", skin=1.0, prune=pr)
        r.launch(40)
        torch.cuda.synchronize()
        r.check()
        out.append((r.x.cpu().numpy(), r.energy.cpu().numpy(), r.f.cpu().numpy()))
    np.testing.assert_allclose(out[0][0], out[1][0], atol=1e-5)
    np.testing.assert_allclose(out[0][1], out[1][1], rtol=1e-5)
    assert np.abs(out[0][2] - out[1][2]).max() <= 1e-4 * np.abs(out[0][2]).max()


def test_prune_at_or_above_skin_is_off():
    """prune >= skin leaves the whole list to every step (same results bit for
    bit as prune = 0: the same pairs in the same order)."""
    out = []
    for pr in (0.0, 0.7, 2.0):
        d, r = _setup(6, 13, "nvt_langevin", skin=0.7, prune=pr)
        r.launch(25)
        torch.cuda.synchronize()
        r.check()
        out.append(r.x.cpu().numpy())
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


@pytest.mark.parametrize("shear", [12.0, 25.0])
def test_list_build_window_on_skewed_cells(shear):
    """The list build searches, per row of bins, only the z range that the
    lattice's metric allows within the list radius; on strongly sheared cells
    (up to 25 degrees) no pair within the cutoff may be missed: forces and
    energies after several launches match the FP64 oracle."""
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(10, 60, 512, seed=21, shear_deg=shear)
    st = state_from_arrays(d, device="cuda")
    st.rng = 5
    m = models.MorseModel(sigma=MORSE[0], epsilon=MORSE[1], alpha=MORSE[2], cutoff=6.0)
    kT = 1000.0 * workloads.KB_EV
    md = integrators.nvt_langevin_init(st, m, kT=kT)
    r = integrators.FusedMD(md, m, integrator="nvt_langevin", dt=0.002 * workloads.METAL_TIME,
                            kT=kT, gamma=10.0 / workloads.METAL_TIME, skin=1.0, prune=0.3,
                            seed=17)
    tab = opair.single_table(opair.MORSE, *MORSE)
    cell_row = np.transpose(d["cell"], (0, 2, 1))
    pbc = np.ones((cell_row.shape[0], 3), bool)
    for k in range(4):
        r.launch(13)
        torch.cuda.synchronize()
        r.check()
        x = r.x.cpu().numpy()
        ref = opair.pair_forward(opair.MORSE, tab, np.zeros(len(x), int), x, cell_row, pbc,
                                 d["system_idx"], 6.0)
        err = np.abs(r.f.cpu().numpy() - ref["forces"]).max() / np.abs(ref["forces"]).max()
        assert err <= 1e-5, (k, err)
        np.testing.assert_allclose(r.energy.cpu().numpy(), ref["energy"], rtol=2e-6)
