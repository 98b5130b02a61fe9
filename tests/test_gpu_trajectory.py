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
