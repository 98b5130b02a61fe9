"""GPU integrator steps and the persistent fused MD kernel.

* nve_step / nvt_langevin_step (with the reference's recorded noise) vs the
  reference trajectories in golden/md.npz, FP64 model: rtol 1e-9.
* run_md (fused, FP32 pair math) vs the step-by-step path with the same model
  settings, energy conservation, Langevin temperature, determinism and
  batch independence.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _mdstate(g, k=0):
    from tsb.state import MDState

    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    return MDState(positions=T(g["positions"][k]), masses=T(g["masses"]), cell=T(g["cell"]),
                   pbc=True, atomic_numbers=T(np.full(len(g["masses"]), 18), torch.int64),
                   system_idx=T(g["system_idx"], torch.int64), momenta=T(g["momenta"][k]),
                   energy=T(g["energy"][k]), forces=T(g["forces"][k]))


def test_nve_matches_reference(golden):
    from tsb import integrators, models

    g = golden["md"]["nve"]
    st = _mdstate(g)
    m = models.LennardJonesModel(sigma=3.405, epsilon=0.0104, precision="fp64")
    for k in range(1, g["positions"].shape[0]):
        st = integrators.nve_step(st, m, dt=float(g["dt"]))
        np.testing.assert_allclose(st.positions.cpu(), g["positions"][k], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(st.momenta.cpu(), g["momenta"][k], rtol=1e-9, atol=1e-13)
        np.testing.assert_allclose(st.energy.cpu(), g["energy"][k], rtol=1e-10)


def test_langevin_matches_reference_with_injected_noise(golden):
    from tsb import integrators, models

    g = golden["md"]["nvt"]
    st = _mdstate(g)
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          precision="fp64")
    for k in range(1, g["positions"].shape[0]):
        noise = torch.as_tensor(g["noise"][k - 1], device="cuda")
        st = integrators.nvt_langevin_step(st, m, dt=float(g["dt"]), kT=float(g["kT"]),
                                           gamma=float(g["gamma"]), noise=noise)
        np.testing.assert_allclose(st.positions.cpu(), g["positions"][k], rtol=1e-12, atol=1e-12)
        np.testing.assert_allclose(st.momenta.cpu(), g["momenta"][k], rtol=1e-9, atol=1e-12)


def _cu_state(n_sys=16, seed=0, n_max=512, kT=1000.0):
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(n_sys, 8, n_max, seed=seed)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed + 1
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    md = integrators.nvt_langevin_init(st, m, kT=kT * workloads.KB_EV)
    return md, m


def test_fused_nve_matches_stepwise():
    """Fused kernel == nve_step loop (same FP32 pair math) to accumulated rounding."""
    from tsb import integrators, workloads

    md, m = _cu_state(8, seed=3, n_max=300)
    dt = 0.002 * workloads.METAL_TIME
    a = md.clone()
    a._philox_seed, a._philox_counter = 0, 0
    for _ in range(10):
        a = integrators.nve_step(a, m, dt=dt)
    b = md.clone()
    b = integrators.run_md(b, m, 10, integrator="nve", dt=dt, skin=1.0)
    # FP32 pair math on both paths, different rounding (SMEM FP32 coordinates vs
    # FP64 displacements): differences stay at the 1e-6 relative force level
    np.testing.assert_allclose(b.positions.cpu(), a.positions.cpu(), atol=1e-6)
    np.testing.assert_allclose(b.momenta.cpu(), a.momenta.cpu(), atol=5e-5, rtol=1e-4)
    fa, fb = a.forces.cpu().numpy(), b.forces.cpu().numpy()
    assert np.abs(fa - fb).max() / np.abs(fa).max() < 2e-5
    np.testing.assert_allclose(b.energy.cpu(), a.energy.cpu(), rtol=1e-6)


def _etot(s):
    from tsb import quantities

    ke = quantities.calc_kinetic_energy(masses=s.masses, momenta=s.momenta,
                                        system_idx=s.system_idx, n_systems=s.n_systems)
    return (ke + s.energy).cpu().numpy()


def test_fused_nve_energy_conservation_shifted_lj():
    """Energy-shifted LJ (continuous energy): total energy per atom conserved to
    1e-4 eV over 500 fused NVE steps of 2 fs (cf. test_integrators.py:1078-1100)."""
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.argon_fcc((3, 3, 3), jitter=0.05, seed=11, n_systems=24)
    st = state_from_arrays(d, device="cuda")
    st.rng = 5
    m = models.LennardJonesModel(sigma=3.405, epsilon=0.0104, shift_energy=True)
    md = integrators.nve_init(st, m, kT=40.0 * workloads.KB_EV)
    dt = 0.002 * workloads.METAL_TIME
    md = integrators.run_md(md, m, 1, integrator="nve", dt=dt)
    e0 = _etot(md)
    md, reb = integrators.run_md(md, m, 500, integrator="nve", dt=dt, return_rebuilds=True)
    drift = np.abs(_etot(md) - e0) / 108
    assert drift.max() < 1e-4, drift.max()
    assert int(reb.min()) >= 1


def test_fused_nve_drift_matches_stepwise_morse():
    """Truncated (unshifted) Morse at 6 A: pairs crossing the cutoff change the
    energy by ~0.01 eV; the fused kernel must show the same physics as the
    step-by-step path (per-system drift of the same size)."""
    from tsb import integrators, workloads

    md, m = _cu_state(16, seed=5, kT=300.0)
    dt = 0.002 * workloads.METAL_TIME
    a = integrators.run_md(md.clone(), m, 1, integrator="nve", dt=dt)
    b = a.clone()
    b._philox_seed, b._philox_counter = 0, 0
    e0 = _etot(a)
    a = integrators.run_md(a, m, 200, integrator="nve", dt=dt)
    for _ in range(200):
        b = integrators.nve_step(b, m, dt=dt)
    n_at = np.bincount(md.system_idx.cpu().numpy())
    da = np.abs(_etot(a) - e0) / n_at
    db = np.abs(_etot(b) - e0) / n_at
    assert da.max() < 1e-2 and db.max() < 1e-2
    assert np.median(da) < 3 * np.median(db) + 1e-5


def test_fused_langevin_temperature():
    from tsb import integrators, quantities, workloads

    md, m = _cu_state(48, seed=7, kT=1000.0)
    dt = 0.002 * workloads.METAL_TIME
    kT = 1000.0 * workloads.KB_EV
    gamma = 10.0 / workloads.METAL_TIME
    md = integrators.run_md(md, m, 1500, integrator="nvt_langevin", dt=dt, kT=kT, gamma=gamma)
    temps = []
    for _ in range(10):
        md = integrators.run_md(md, m, 50, integrator="nvt_langevin", dt=dt, kT=kT,
                                gamma=gamma)
        t = quantities.calc_kT(masses=md.masses, momenta=md.momenta,
                               system_idx=md.system_idx, n_systems=md.n_systems)
        n_at = torch.bincount(md.system_idx).double()
        temps.append(float((t * n_at).sum() / n_at.sum()) / workloads.KB_EV)
    assert abs(np.mean(temps) - 1000.0) < 60.0, temps


def test_fused_deterministic_and_batch_independent():
    from tsb import integrators, workloads
    from tsb.state import MDState

    md, m = _cu_state(10, seed=9)
    dt = 0.002 * workloads.METAL_TIME
    kw = dict(integrator="nvt_langevin", dt=dt, kT=1000 * workloads.KB_EV,
              gamma=10.0 / workloads.METAL_TIME, seed=1234)
    a = integrators.run_md(md.clone(), m, 60, **kw)
    b = integrators.run_md(md.clone(), m, 60, **kw)
    assert torch.equal(a.positions, b.positions) and torch.equal(a.momenta, b.momenta)
    # system 4 alone must follow the same trajectory as inside the batch,
    # given the same Philox stream (atom index enters the counter, so keep offsets)
    sel = md.system_idx == 4
    idx = torch.nonzero(sel).flatten()
    sub = MDState(positions=md.positions[sel], masses=md.masses[sel], cell=md.cell[4:5],
                  pbc=md.pbc, atomic_numbers=md.atomic_numbers[sel],
                  system_idx=torch.zeros(int(sel.sum()), dtype=torch.int64, device="cuda"),
                  momenta=md.momenta[sel], energy=md.energy[4:5], forces=md.forces[sel])
    kw_nve = dict(integrator="nve", dt=dt)
    c = integrators.run_md(md.clone(), m, 40, **kw_nve)
    d = integrators.run_md(sub, m, 40, **kw_nve)
    assert torch.equal(c.positions[idx], d.positions)
    assert torch.equal(c.energy[4], d.energy[0])


def test_fused_rejects_unsupported():
    from tsb import integrators, models, workloads
    from tsb.state import MDState, state_from_arrays

    d = workloads.argon_fcc((6, 6, 6), seed=0)  # 864 atoms > 512
    st = state_from_arrays(d, device="cuda")
    m = models.LennardJonesModel(sigma=3.405, epsilon=0.0104)
    md = MDState.from_state(st, momenta=torch.zeros_like(st.positions),
                            energy=torch.zeros(1, dtype=torch.float64, device="cuda"),
                            forces=torch.zeros_like(st.positions))
    with pytest.raises(integrators.FusedMDError):
        integrators.FusedMD(md, m, integrator="nve", dt=0.1)


def test_run_md_routes_oversized_systems_and_bins():
    """A batch with systems above the fused kernel's 512 atoms: those advance
    through the per-call steps (as they would alone), the rest through the fused
    kernel (in memory-bounded bins when max_memory_scaler is given), each system
    exactly as when it runs by itself (torch_sim/autobatching.py:475-765 is the
    admission policy this replaces)."""
    from tsb import integrators, models, workloads
    from tsb.state import select_systems, state_from_arrays

    big = workloads.argon_fcc((6, 6, 6), jitter=0.05, seed=4)
    small = workloads.argon_fcc((3, 3, 3), jitter=0.05, seed=5, n_systems=3)
    from tsb.workloads import _pack  # noqa: PLC2701

    def split(d):
        out = []
        off = np.concatenate([[0], np.cumsum(np.bincount(d["system_idx"]))])
        for s in range(len(off) - 1):
            a, b = off[s], off[s + 1]
            out.append({"positions": d["positions"][a:b], "cell_row": d["cell"][s].T,
                        "masses": d["masses"][a:b], "atomic_numbers": d["atomic_numbers"][a:b]})
        return out

    systems = split(small)[:1] + split(big) + split(small)[1:]
    d = _pack(systems)
    st = state_from_arrays(d, device="cuda")
    st.rng = 3
    m = models.LennardJonesModel(sigma=3.405, epsilon=0.0104)
    md = integrators.nve_init(st, m, kT=40 * workloads.KB_EV)
    dt = 0.002 * workloads.METAL_TIME
    ref = [integrators.run_md(select_systems(md, [s]), m, 20, integrator="nve", dt=dt, skin=0.5)
           if s != 1 else None for s in range(4)]
    alone = select_systems(md, [1])
    for _ in range(20):
        alone = integrators.nve_step(alone, m, dt=dt)
    ref[1] = alone
    for scaler in (None, 3000.0):
        out, reb = integrators.run_md(md.clone(), m, 20, integrator="nve", dt=dt, skin=0.5,
                                      return_rebuilds=True, max_memory_scaler=scaler)
        assert int(reb[1]) == -1 and bool((reb[[0, 2, 3]] >= 1).all())
        for s in range(4):
            got = select_systems(out, [s])
            assert torch.equal(got.positions, ref[s].positions), (scaler, s)
            assert torch.equal(got.momenta, ref[s].momenta), (scaler, s)
            assert torch.equal(got.energy, ref[s].energy), (scaler, s)


def test_fused_adaptive_skin_same_physics():
    """A skin too large for the shared-memory tables is shrunk per system on the
    device; the trajectory matches a run at a small skin to FP32 rounding."""
    from tsb import integrators, workloads

    md, m = _cu_state(12, seed=13, kT=600.0)
    dt = 0.002 * workloads.METAL_TIME
    a = integrators.run_md(md.clone(), m, 30, integrator="nve", dt=dt, skin=2.5)
    b = integrators.run_md(md.clone(), m, 30, integrator="nve", dt=dt, skin=0.3)
    np.testing.assert_allclose(a.positions.cpu(), b.positions.cpu(), atol=1e-5)
    np.testing.assert_allclose(a.energy.cpu(), b.energy.cpu(), rtol=1e-5)


def test_fused_graph_replay_matches_direct_launches():
    """The persistent kernel under a captured CUDA graph: two replays equal two
    direct launches bitwise (the device Philox counter advances per replay)."""
    from tsb import integrators, workloads

    md, m = _cu_state(6, seed=17)
    kw = dict(integrator="nvt_langevin", dt=0.002 * workloads.METAL_TIME,
              kT=1000 * workloads.KB_EV, gamma=10.0 / workloads.METAL_TIME, seed=99)
    a = integrators.FusedMD(md.clone(), m, **kw)
    a.launch(25)
    a.launch(25)
    b = integrators.FusedMD(md.clone(), m, **kw)
    g = b.graph(25)
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    a.check()
    b.check()
    assert a.counter == b.counter == 50
    assert torch.equal(a.x, b.x) and torch.equal(a.p, b.p) and torch.equal(a.energy, b.energy)


def test_block_shapes_agree():
    """The same batch run with every system in 512-thread blocks and with small
    systems in 256-thread blocks (two per SM): the trajectories agree to FP32
    rounding (the lane split of each neighbour list, and so the summation order,
    differs) and both shapes are used."""
    from tsb import integrators, workloads

    md, m = _cu_state(24, seed=4)
    kw = dict(integrator="nve", dt=0.002 * workloads.METAL_TIME, skin=0.5)
    a = integrators.FusedMD(md.clone(), m, shapes="wide", **kw)
    b = integrators.FusedMD(md.clone(), m, shapes="auto", **kw)
    assert a.n_wide == -1 and 0 < b.n_wide < md.n_systems
    for r in (a, b):
        r.launch(40)
        torch.cuda.synchronize()
        r.check()
    np.testing.assert_allclose(b.x.cpu().numpy(), a.x.cpu().numpy(), atol=1e-5)
    np.testing.assert_allclose(b.energy.cpu().numpy(), a.energy.cpu().numpy(), rtol=1e-5)
    np.testing.assert_allclose(b.stress.cpu().numpy(), a.stress.cpu().numpy(), rtol=1e-4,
                               atol=1e-7)
