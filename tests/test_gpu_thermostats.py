"""NVT Nose-Hoover-chain and V-rescale (CSVR) steps on the GPU.

* Trajectories vs the reference (tests/golden/thermostats.npz, written by
  make_thermostats.py): FP64 model, rtol 1e-9 on momenta, chain variables and
  the Nose-Hoover invariant; V-rescale with the reference's random numbers
  injected.
* The device CSVR sampler: with the kinetic energy at its target, lambda^2 has
  mean 1 and variance 2 c2^2 dof + 4 c1 c2 (r1 ~ N(0,1), 2 g ~ chi^2(dof - 1)).
* Temperature control of both thermostats on a Morse Cu batch.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _state(g, s, k=0):
    from tsb.state import MDState

    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    n = len(s["masses"])
    return MDState(positions=T(g["positions"][k]), masses=T(s["masses"]), cell=T(s["cell"]),
                   pbc=True, atomic_numbers=T(np.full(n, 29), torch.int64),
                   system_idx=T(s["system_idx"], torch.int64), momenta=T(g["momenta"][k]),
                   energy=T(np.zeros(3)), forces=T(np.zeros((n, 3))))


def _morse64():
    from tsb import models

    return models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                             precision="fp64")


def test_nose_hoover_matches_reference(golden):
    from tsb import integrators as I

    s, g = golden["thermostats"]["sys"], golden["thermostats"]["nhc"]
    dt, kT = float(s["dt"]), float(s["kT"])
    m = _morse64()
    st = I.nvt_nose_hoover_init(_state(g, s), m, kT=kT, dt=dt, chain_length=3, chain_steps=3,
                                sy_steps=3)
    np.testing.assert_allclose(st.chain.masses.cpu(), g["Q"][0], rtol=1e-14)
    np.testing.assert_allclose(st.chain.kinetic_energy.cpu(), g["KE"][0], rtol=1e-12)
    np.testing.assert_array_equal(st.chain.degrees_of_freedom.cpu(), g["dof"])
    for k in range(1, g["positions"].shape[0]):
        st = I.nvt_nose_hoover_step(st, m, dt=dt, kT=kT)
        np.testing.assert_allclose(st.positions.cpu(), g["positions"][k], rtol=1e-12,
                                   atol=1e-12)
        np.testing.assert_allclose(st.momenta.cpu(), g["momenta"][k], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(st.chain.positions.cpu(), g["xi"][k], rtol=1e-9,
                                   atol=1e-14)
        np.testing.assert_allclose(st.chain.momenta.cpu(), g["p_xi"][k], rtol=1e-9,
                                   atol=1e-14)
        np.testing.assert_allclose(st.chain.kinetic_energy.cpu(), g["KE"][k], rtol=1e-10)
        np.testing.assert_allclose(I.nvt_nose_hoover_invariant(st, kT).cpu(),
                                   g["invariant"][k], rtol=1e-11)


def test_vrescale_matches_reference_with_injected_noise(golden):
    from tsb import integrators as I

    s, g = golden["thermostats"]["sys"], golden["thermostats"]["vr"]
    dt, kT = float(s["dt"]), float(s["kT"])
    m = _morse64()
    st = I.nvt_vrescale_init(_state(g, s), m, kT=kT)
    for k in range(1, g["positions"].shape[0]):
        noise = np.stack([g["r1"][k - 1], g["gamma"][k - 1]], axis=1)
        st = I.nvt_vrescale_step(m, st, dt=dt, kT=kT, noise=noise)
        np.testing.assert_allclose(st.positions.cpu(), g["positions"][k], rtol=1e-12,
                                   atol=1e-12)
        np.testing.assert_allclose(st.momenta.cpu(), g["momenta"][k], rtol=1e-9, atol=1e-12)
        np.testing.assert_allclose(st.energy.cpu(), g["energy"][k], rtol=1e-10)


def test_vrescale_device_sampler_moments():
    """4096 systems of 4 atoms (dof 9) at their own current temperature."""
    from tsb import _lib as L
    from tsb import integrators as I
    from tsb.state import MDState

    dev = torch.device("cuda")
    S, n_per = 4096, 4
    n = S * n_per
    g = torch.Generator(device=dev).manual_seed(3)
    masses = torch.full((n,), 63.546, dtype=torch.float64, device=dev)
    p = torch.randn((n, 3), dtype=torch.float64, device=dev, generator=g)
    sysi = torch.arange(S, device=dev).repeat_interleave(n_per)
    p0 = p.clone()
    st = MDState(positions=torch.zeros_like(p), masses=masses,
                 cell=torch.eye(3, dtype=torch.float64, device=dev).expand(S, 3, 3) * 20,
                 pbc=True, atomic_numbers=torch.full((n,), 29, device=dev), system_idx=sysi,
                 momenta=p, energy=torch.zeros(S, dtype=torch.float64, device=dev),
                 forces=torch.zeros_like(p))
    dof = I._dof(st)
    kT = (2.0 * I.kinetic_energy(st) / dof).contiguous()  # KE at its target
    dt, tau = 0.2, 2.0
    dt_s = torch.full((S,), dt, dtype=torch.float64, device=dev)
    tau_s = torch.full((S,), tau, dtype=torch.float64, device=dev)
    lam = torch.empty(S, dtype=torch.float64, device=dev)
    ws = L.Workspace.get(dev, L.load().tsb_thermostat_workspace_size(S))
    L.call("tsb_vrescale", L.ptr(st.momenta), L.ptr(masses), L.ptr(sysi), n, S, L.F64,
           L.ptr(dof), L.ptr(kT), L.ptr(tau_s), L.ptr(dt_s), None, 99, 0, L.ptr(lam), L.ptr(ws),
           ws.numel(), L.stream_ptr(dev))
    lam2 = (lam ** 2).cpu().numpy()
    c1 = np.exp(-dt / tau)
    c2 = (1 - c1) / 9.0
    var = 2 * c2 ** 2 * 9 + 4 * c1 * c2
    assert abs(lam2.mean() - 1.0) < 5 * np.sqrt(var / S)
    assert abs(lam2.var() - var) < 0.15 * var
    # the momenta were scaled by lambda
    np.testing.assert_allclose(st.momenta.cpu().numpy(), (p0 * lam[sysi, None]).cpu().numpy(),
                               rtol=1e-15)


@pytest.mark.parametrize("thermostat", ["nose_hoover", "vrescale"])
def test_thermostat_holds_temperature(thermostat):
    from tsb import integrators as I
    from tsb import models, quantities, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(16, 64, 256, seed=5)
    st = state_from_arrays(d, device="cuda")
    st.rng = 4
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    kT = 600.0 * workloads.KB_EV
    dt = 0.002 * workloads.METAL_TIME
    if thermostat == "nose_hoover":
        md = I.nvt_nose_hoover_init(st, m, kT=kT, dt=dt)
        step = lambda s: I.nvt_nose_hoover_step(s, m, dt=dt, kT=kT)  # noqa: E731
    else:
        md = I.nvt_vrescale_init(st, m, kT=kT)
        step = lambda s: I.nvt_vrescale_step(m, s, dt=dt, kT=kT)  # noqa: E731
    temps = []
    for k in range(600):
        md = step(md)
        if k >= 300 and k % 10 == 0:
            t = quantities.calc_kT(masses=md.masses, momenta=md.momenta,
                                   system_idx=md.system_idx, n_systems=md.n_systems)
            n_at = torch.bincount(md.system_idx).double()
            temps.append(float((t * n_at).sum() / n_at.sum()) / workloads.KB_EV)
    # calc_kT divides by 3N; the thermostats target kT on 3N - 3 degrees of freedom
    assert abs(np.mean(temps) - 600.0) < 45.0, temps


def _cu_batch(n_sys=10, seed=8):
    from tsb import models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(n_sys, 16, 300, seed=seed)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    return st, m


def test_fused_nose_hoover_matches_step_function():
    """Persistent kernel with the chain inside == nvt_nose_hoover_step loop (FP32
    pair math on both paths; chain arithmetic shared)."""
    from tsb import integrators as I
    from tsb import workloads

    st, m = _cu_batch()
    kT, dt = 800.0 * workloads.KB_EV, 0.002 * workloads.METAL_TIME
    md = I.nvt_nose_hoover_init(st, m, kT=kT, dt=dt)
    a = md.clone()
    for _ in range(20):
        a = I.nvt_nose_hoover_step(a, m, dt=dt, kT=kT)
    b = I.run_md(md.clone(), m, 20, integrator="nvt_nose_hoover", dt=dt, kT=kT, skin=0.5)
    np.testing.assert_allclose(b.positions.cpu(), a.positions.cpu(), atol=2e-6)
    np.testing.assert_allclose(b.momenta.cpu(), a.momenta.cpu(), atol=1e-4, rtol=1e-4)
    np.testing.assert_allclose(b.chain.momenta.cpu(), a.chain.momenta.cpu(), rtol=1e-4,
                               atol=1e-7)
    np.testing.assert_allclose(b.chain.positions.cpu(), a.chain.positions.cpu(), rtol=1e-4,
                               atol=1e-8)
    np.testing.assert_allclose(b.chain.kinetic_energy.cpu(), a.chain.kinetic_energy.cpu(),
                               rtol=1e-5)
    np.testing.assert_allclose(I.nvt_nose_hoover_invariant(b, kT).cpu(),
                               I.nvt_nose_hoover_invariant(a, kT).cpu(), rtol=1e-6)


def test_fused_vrescale_matches_step_function():
    """Same Philox draws (seed, system, step) in the kernel and the step function."""
    from tsb import integrators as I
    from tsb import workloads

    st, m = _cu_batch(seed=9)
    kT, dt = 800.0 * workloads.KB_EV, 0.002 * workloads.METAL_TIME
    md = I.nvt_vrescale_init(st, m, kT=kT)
    a = md.clone()
    a._philox_seed, a._philox_counter = 77, 0
    for _ in range(20):
        a = I.nvt_vrescale_step(m, a, dt=dt, kT=kT)
    b = md.clone()
    b._philox_seed, b._philox_counter = 77, 0
    b = I.run_md(b, m, 20, integrator="nvt_vrescale", dt=dt, kT=kT, skin=0.5)
    np.testing.assert_allclose(b.positions.cpu(), a.positions.cpu(), atol=2e-6)
    np.testing.assert_allclose(b.momenta.cpu(), a.momenta.cpu(), atol=1e-4, rtol=1e-4)
