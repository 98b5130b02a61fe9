"""NPT Langevin (isotropic, anisotropic) and C-rescale (all variants) on the GPU.

* 8 steps vs the reference (golden/npt.npz) with the reference's cell and
  particle noise injected; FP64 model: positions, cell and strain to 1e-12,
  momenta and strain velocity to 1e-9, stress to 1e-9.
* Device noise: a run is reproducible from its seed, and the barostat responds:
  the same systems end with a smaller volume at 20 GPa than at 0 GPa.
"""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GPA = 0.006241509074460764  # eV / A^3


def test_npt_langevin_isotropic_matches_reference(golden):
    from tsb import integrators as I
    from tsb import models
    from tsb.state import MDState

    s, g = golden["npt"]["sys"], golden["npt"]["npt"]
    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    n = len(s["masses"])
    st = MDState(positions=T(g["positions"][0]), masses=T(s["masses"]), cell=T(s["cell"]),
                 pbc=True, atomic_numbers=T(s["atomic_numbers"], torch.int64),
                 system_idx=T(s["system_idx"], torch.int64), momenta=T(g["momenta"][0]),
                 energy=T(np.zeros(3)), forces=T(np.zeros((n, 3))))
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          compute_stress=True, precision="fp64")
    dt, kT, p = float(g["dt"]), float(g["kT"]), float(g["p_ext"])
    st = I.npt_langevin_isotropic_init(st, m, kT=kT, dt=dt)
    np.testing.assert_allclose(st.cell_masses.cpu(), g["cell_masses"][0], rtol=1e-14)
    np.testing.assert_allclose(st.stress.cpu(), g["stress"][0], rtol=1e-9, atol=1e-14)
    for k in range(1, g["positions"].shape[0]):
        st = I.npt_langevin_isotropic_step(st, m, dt=dt, kT=kT, external_pressure=p,
                                           noise=(g["cell_noise"][k - 1],
                                                  g["particle_noise"][k - 1]))
        for key, rt in (("positions", 1e-12), ("cell", 1e-12), ("cell_positions", 1e-9),
                        ("momenta", 1e-9), ("cell_velocities", 1e-9), ("stress", 1e-9)):
            np.testing.assert_allclose(getattr(st, key).cpu(), g[key][k], rtol=rt,
                                       atol=1e-14, err_msg=key)


def _run(p_gpa, seed=3, steps=300):
    from tsb import integrators as I
    from tsb import models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(6, 100, 250, seed=4)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          compute_stress=True)
    kT, dt = 300 * workloads.KB_EV, 0.002 * workloads.METAL_TIME
    md = I.npt_langevin_isotropic_init(st, m, kT=kT, dt=dt, b_tau=50 * dt)
    for _ in range(steps):
        md = I.npt_langevin_isotropic_step(md, m, dt=dt, kT=kT,
                                           external_pressure=p_gpa * GPA)
    return md


def test_npt_device_noise_reproducible_and_barostat_responds():
    a = _run(0.0)
    b = _run(0.0)
    assert torch.equal(a.positions, b.positions) and torch.equal(a.cell, b.cell)
    c = _run(20.0)
    va = torch.linalg.det(a.cell).abs()
    vc = torch.linalg.det(c.cell).abs()
    assert bool((vc < va).all()), (va, vc)
    assert torch.isfinite(a.positions).all() and torch.isfinite(c.momenta).all()


@pytest.mark.parametrize("grp", ["crescale", "crescale_aniso", "crescale_tri",
                                 "crescale_tri_dev", "crescale_tri_avg"])
def test_npt_crescale_matches_reference(golden, grp):
    """8 steps of each C-rescale variant (isotropic, anisotropic, triclinic with a
    scalar and a tensor pressure, triclinic average) vs the reference
    (golden/crescale.npz) with its V-rescale and barostat draws injected; FP64
    model, max|d| / max|ref| <= 1e-9."""
    from tsb import integrators as I
    from tsb import models
    from tsb.state import MDState

    s, g = golden["crescale"]["sys"], golden["crescale"][grp]
    step = {"crescale": I.npt_crescale_isotropic_step,
            "crescale_aniso": I.npt_crescale_anisotropic_step,
            "crescale_tri": I.npt_crescale_triclinic_step,
            "crescale_tri_dev": I.npt_crescale_triclinic_step,
            "crescale_tri_avg": I.npt_crescale_triclinic_average_step}[grp]
    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    n = len(s["masses"])
    st = MDState(positions=T(g["positions"][0]), masses=T(s["masses"]), cell=T(s["cell"]),
                 pbc=True, atomic_numbers=T(s["atomic_numbers"], torch.int64),
                 system_idx=T(s["system_idx"], torch.int64), momenta=T(g["momenta"][0]),
                 energy=T(np.zeros(3)), forces=T(np.zeros((n, 3))))
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          compute_stress=True, precision="fp64")
    dt, kT, tau = (float(g[k]) for k in ("dt", "kT", "tau"))
    p = g["p_ext"]
    st = I.npt_crescale_init(st, m, kT=kT, dt=dt, tau_p=g["tau_p"],
                             isothermal_compressibility=g["isothermal_compressibility"])
    np.testing.assert_allclose(st.stress.cpu(), g["stress"][0], rtol=1e-9, atol=1e-14)
    for k in range(1, g["positions"].shape[0]):
        noise = (np.stack([g["r1_a"][k - 1], g["gamma_a"][k - 1]], axis=1),
                 g["cell_noise"][k - 1],
                 np.stack([g["r1_b"][k - 1], g["gamma_b"][k - 1]], axis=1))
        st = step(st, m, dt=dt, kT=kT, external_pressure=p, tau=tau, noise=noise)
        for key in ("positions", "momenta", "cell", "stress", "energy"):
            np.testing.assert_allclose(getattr(st, key).cpu(), g[key][k], rtol=0,
                                       atol=1e-9 * np.abs(g[key][k]).max(),
                                       err_msg=f"step {k} {key}")


def _run_crescale(p_gpa, seed=3, steps=300):
    from tsb import integrators as I
    from tsb import models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(6, 100, 250, seed=4)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          compute_stress=True)
    kT, dt = 300 * workloads.KB_EV, 0.002 * workloads.METAL_TIME
    # the default compressibility, 1e-6 / bar (copper: about 7e-7 / bar)
    md = I.npt_crescale_init(st, m, kT=kT, dt=dt, tau_p=100 * dt)
    for _ in range(steps):
        md = I.npt_crescale_isotropic_step(md, m, dt=dt, kT=kT, external_pressure=p_gpa * GPA,
                                           tau=10 * dt)
    return md


def test_npt_crescale_device_noise_reproducible_and_barostat_responds():
    a = _run_crescale(0.0)
    b = _run_crescale(0.0)
    assert torch.equal(a.positions, b.positions) and torch.equal(a.cell, b.cell)
    c = _run_crescale(20.0)
    va = torch.linalg.det(a.cell).abs()
    vc = torch.linalg.det(c.cell).abs()
    assert bool((vc < va).all()), (va, vc)
    assert torch.isfinite(a.positions).all() and torch.isfinite(c.momenta).all()


def test_npt_langevin_anisotropic_matches_reference(golden):
    """8 per-axis NPT Langevin steps at (1.0, 1.3, 0.7) GPa vs the reference
    (golden/npt.npz, npt_aniso) with its cell and particle noise injected; FP64
    model, max|d| / max|ref| <= 1e-9."""
    from tsb import integrators as I
    from tsb import models
    from tsb.state import MDState

    s, g = golden["npt"]["sys"], golden["npt"]["npt_aniso"]
    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    n = len(s["masses"])
    st = MDState(positions=T(g["positions"][0]), masses=T(s["masses"]), cell=T(s["cell"]),
                 pbc=True, atomic_numbers=T(s["atomic_numbers"], torch.int64),
                 system_idx=T(s["system_idx"], torch.int64), momenta=T(g["momenta"][0]),
                 energy=T(np.zeros(3)), forces=T(np.zeros((n, 3))))
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          compute_stress=True, precision="fp64")
    dt, kT = float(g["dt"]), float(g["kT"])
    st = I.npt_langevin_anisotropic_init(st, m, kT=kT, dt=dt)
    for k in range(1, g["positions"].shape[0]):
        st = I.npt_langevin_anisotropic_step(st, m, dt=dt, kT=kT, external_pressure=g["p_ext"],
                                             noise=(g["cell_noise"][k - 1],
                                                    g["particle_noise"][k - 1]))
        for key in ("positions", "momenta", "cell", "cell_positions", "cell_velocities",
                    "stress"):
            np.testing.assert_allclose(getattr(st, key).cpu(), g[key][k], rtol=0,
                                       atol=1e-9 * np.abs(g[key][k]).max(),
                                       err_msg=f"step {k} {key}")


def test_npt_nose_hoover_isotropic_matches_reference(golden):
    """8 MTK isotropic NPT steps with Nose-Hoover chains vs the reference
    (golden/npt.npz, npt_nh; deterministic): positions, momenta, cell, log volume,
    cell momentum, both chains and the conserved quantity; FP64 model,
    max|d| / max|ref| <= 1e-9."""
    from tsb import integrators as I
    from tsb import models
    from tsb.state import MDState

    s, g = golden["npt"]["sys"], golden["npt"]["npt_nh"]
    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    n = len(s["masses"])
    st = MDState(positions=T(g["positions"][0]), masses=T(s["masses"]), cell=T(g["cell"][0]),
                 pbc=True, atomic_numbers=T(s["atomic_numbers"], torch.int64),
                 system_idx=T(s["system_idx"], torch.int64), momenta=T(g["momenta"][0]),
                 energy=T(np.zeros(3)), forces=T(np.zeros((n, 3))))
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0,
                          compute_stress=True, precision="fp64")
    dt, kT, p = float(g["dt"]), float(g["kT"]), float(g["p_ext"])
    st = I.npt_nose_hoover_isotropic_init(st, m, kT=kT, dt=dt)

    def close(got, ref, what):
        np.testing.assert_allclose(got.detach().cpu().numpy().reshape(ref.shape), ref, rtol=0,
                                   atol=1e-9 * max(np.abs(ref).max(), 1e-30), err_msg=what)

    close(I.npt_nose_hoover_isotropic_invariant(st, kT, p), g["invariant"][0], "invariant 0")
    for k in range(1, g["positions"].shape[0]):
        st = I.npt_nose_hoover_isotropic_step(st, m, dt=dt, kT=kT, external_pressure=p)
        for key in ("positions", "momenta", "cell", "cell_position", "cell_momentum",
                    "stress"):
            close(getattr(st, key), g[key][k], f"step {k} {key}")
        for ch, name in ((st.thermostat, "thermostat"), (st.barostat, "barostat")):
            close(ch.positions, g[f"{name}_positions"][k], f"step {k} {name} xi")
            close(ch.momenta, g[f"{name}_momenta"][k], f"step {k} {name} p_xi")
        close(I.npt_nose_hoover_isotropic_invariant(st, kT, p), g["invariant"][k],
              f"step {k} invariant")
