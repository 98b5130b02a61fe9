"""Trajectory frames written by the persistent fused kernel (tsb_fused_md_ex) and
drained by tsb.trajectory.FusedTrajectory.

Frames every 5 steps, 3 frames per chunk, 40 steps (8 frames, chunks overlap the
copies of the previous chunk).  Each frame equals the state of a run advanced
5 steps per launch (positions to 1e-5 A: the two runs differ only in where the
Verlet list is rebuilt; potential energies to 1e-6), the last frame equals the
final positions, and each system's file holds its frames.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_fused_trajectory_frames(tmp_path):
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays
    from tsb.trajectory import FusedTrajectory

    d = workloads.copper_batch(6, 16, 200, seed=12)
    st = state_from_arrays(d, device="cuda")
    st.rng = 3
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    md = integrators.nvt_langevin_init(st, m, kT=800 * workloads.KB_EV)
    kw = dict(integrator="nvt_langevin", dt=0.002 * workloads.METAL_TIME,
              kT=800 * workloads.KB_EV, gamma=10.0 / workloads.METAL_TIME, skin=0.5, seed=5)
    names = [str(tmp_path / f"sys{s}.npz") for s in range(md.n_systems)]
    a = integrators.FusedMD(md.clone(), m, **kw)
    traj = FusedTrajectory(a, names, state_frequency=5, frames_per_chunk=3)
    traj.run(40)
    torch.cuda.synchronize()
    a.check()
    traj.close()
    b = integrators.FusedMD(md.clone(), m, **kw)
    ref_x, ref_e = [], []
    for _ in range(8):
        b.launch(5)
        torch.cuda.synchronize()
        b.check()
        ref_x.append(b.x.float().cpu().numpy())
        ref_e.append(b.energy.cpu().numpy())
    lo = np.concatenate([[0], np.cumsum(np.bincount(d["system_idx"]))[:-1]])
    hi = np.cumsum(np.bincount(d["system_idx"]))
    for s, fn in enumerate(names):
        f = np.load(fn)
        assert f["positions"].shape == (8, hi[s] - lo[s], 3)
        assert f["positions"].dtype == np.float32
        np.testing.assert_array_equal(f["step"], np.arange(5, 45, 5))
        np.testing.assert_array_equal(f["atomic_numbers"], d["atomic_numbers"][lo[s]:hi[s]])
        for k in range(8):
            np.testing.assert_allclose(f["positions"][k], ref_x[k][lo[s]:hi[s]], atol=1e-5)
            np.testing.assert_allclose(f["potential_energy"][k], ref_e[k][s], rtol=1e-6)
        np.testing.assert_array_equal(f["positions"][-1],
                                      a.x[lo[s]:hi[s]].float().cpu().numpy())


def test_frames_follow_the_reference_reporter(tmp_path):
    """Frame steps and contents against the oracle replay of the same run: the
    reference runner reports after step k = 1, 2, ... and its reporter writes
    when k % state_frequency == 0 (torch_sim/runners.py:384-396,
    trajectory.py:267-340), so the frames are the states after steps 4, 8, ...,
    20, as float32 positions; the frame energies are the potential energies of
    those states."""
    from oracle import fused_md, pair as opair
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays
    from tsb.trajectory import FusedTrajectory

    d = workloads.copper_batch(4, 16, 200, seed=19)
    st = state_from_arrays(d, device="cuda")
    st.rng = 6
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    kT = 800 * workloads.KB_EV
    md = integrators.nvt_langevin_init(st, m, kT=kT)
    kw = dict(integrator="nvt_langevin", dt=0.002 * workloads.METAL_TIME, kT=kT,
              gamma=10.0 / workloads.METAL_TIME, skin=0.5, seed=21)
    names = [str(tmp_path / f"r{s}.npz") for s in range(md.n_systems)]
    run = integrators.FusedMD(md.clone(), m, **kw)
    x, p, f = (t.cpu().numpy().copy() for t in (run.x, run.p, run.f))
    traj = FusedTrajectory(run, names, state_frequency=4, frames_per_chunk=2)
    traj.run(20)
    torch.cuda.synchronize()
    run.check()
    traj.close()
    tab = opair.single_table(opair.MORSE, 2.866, 0.3429, 1.3588)
    cell_row = np.transpose(d["cell"], (0, 2, 1))
    sp = np.zeros(len(x), int)
    lo = np.concatenate([[0], np.cumsum(np.bincount(d["system_idx"]))[:-1]])
    hi = np.cumsum(np.bincount(d["system_idx"]))
    files = [np.load(fn) for fn in names]
    for k in range(5):
        o = fused_md.run(opair.MORSE, tab, sp, x, p, f, d["masses"], cell_row,
                         d["system_idx"], 6.0, 4, kw["dt"], integrator="nvt_langevin", kT=kT,
                         gamma=kw["gamma"], seed=run.seed, counter=4 * k, skin=1.0)
        x, p, f = o["positions"], o["momenta"], o["forces"]
        for s in range(md.n_systems):
            assert int(files[s]["step"][k]) == 4 * (k + 1)
            np.testing.assert_allclose(files[s]["positions"][k], x[lo[s]:hi[s]], rtol=0,
                                       atol=1e-4)
            np.testing.assert_allclose(files[s]["potential_energy"][k], o["energy"][s],
                                       rtol=2e-6)
