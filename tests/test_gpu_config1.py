"""The 256-atom Lennard-Jones argon NVE case on the GPU against the reference's
own run (tests/golden/config1.npz, made by make_config1.py): argon fcc 4x4x4,
N(0, 0.05 A) jitter, LJ sigma 3.405 A, epsilon 0.0104 eV, cutoff 2.5 sigma,
Maxwell-Boltzmann momenta at 50 K from state.rng = 2024, 100 velocity-Verlet
steps of 2 fs, float64; truncated (the reference LennardJonesModel) and
energy-shifted LJ.

* pair set of the neighbour-list drop-in: integer-exact;
* initial momenta: ``initialize_momenta`` with a CPU generator seeded as the
  reference seeds ``state.rng`` replays the reference's draw (md.py:113-166);
* per-call ``nve_step`` with the FP64 model: positions every 10 steps within
  1e-9 A, energies within 1e-10 relative, stresses within 1e-8 relative;
* the persistent fused kernel (FP32 pair arithmetic) over the same 100 steps:
  positions within 2e-4 A of the reference, forces at the end within 1e-5 of
  max|F| of the FP64 forces at the same positions, and the energy-shifted total
  energy drift within 2e-4 eV over the 100 steps (reference: 9.5e-5 eV).
"""

import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
SIGMA, EPS, RC = 3.405, 0.0104, 2.5 * 3.405


@pytest.fixture(scope="module")
def c1():
    return np.load(os.path.join(GOLDEN, "config1.npz"))


def _state(c1, name):
    from tsb.state import MDState

    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    return MDState(positions=T(c1[f"{name}/positions"][0]), masses=T(c1["init/masses"]),
                   cell=T(c1["init/cell"]), pbc=True,
                   atomic_numbers=T(c1["init/atomic_numbers"], torch.int64),
                   system_idx=T(c1["init/system_idx"], torch.int64),
                   momenta=T(c1[f"{name}/momenta"][0]),
                   energy=T(c1[f"{name}/epot"][:1]), forces=T(c1[f"{name}/forces0"]))


def _model(name, precision):
    from tsb import models

    return models.LennardJonesModel(sigma=SIGMA, epsilon=EPS, cutoff=RC,
                                    shift_energy=(name == "lj_shift"), precision=precision,
                                    compute_stress=True)


def test_pair_set_matches_reference(c1):
    from oracle import neighbors as onl
    from tsb import neighbors

    dev = torch.device("cuda")
    pos = torch.as_tensor(c1["init/positions"], device=dev)
    cell_row = torch.as_tensor(c1["init/cell"], device=dev).mT
    m, sm, sh = neighbors.torchsim_nl(pos, cell_row, torch.ones(3, dtype=torch.bool,
                                                                 device=dev),
                                      RC, torch.as_tensor(c1["init/system_idx"], device=dev))
    got = onl.sort_pairs(m.cpu().numpy(), sm.cpu().numpy(), sh.cpu().numpy())
    ref = onl.sort_pairs(c1["pairs/ij"].astype(np.int64),
                         np.zeros(c1["pairs/ij"].shape[1], int),
                         c1["pairs/shifts"].astype(np.float64))
    assert np.array_equal(got[0], ref[0])
    assert np.array_equal(np.rint(got[2]).astype(int), ref[2].astype(int))


def test_initial_momenta_replay_the_reference_draw(c1):
    from tsb import integrators

    dev = torch.device("cuda")
    pos = torch.as_tensor(c1["init/positions"], device=dev)
    g = torch.Generator(device="cpu").manual_seed(2024)
    p = integrators.initialize_momenta(pos, torch.as_tensor(c1["init/masses"], device=dev),
                                       torch.as_tensor(c1["init/system_idx"], device=dev),
                                       torch.tensor(float(c1["kT"]), dtype=torch.float64,
                                                    device=dev), g)
    np.testing.assert_allclose(p.cpu().numpy(), c1["lj/momenta"][0], rtol=1e-12, atol=1e-15)


@pytest.mark.parametrize("name", ["lj", "lj_shift"])
def test_per_call_nve_matches_reference(c1, name):
    from tsb import integrators

    md = _state(c1, name)
    m = _model(name, "fp64")
    every = int(c1["every"])
    for step in range(1, 101):
        md = integrators.nve_step(md, m, dt=float(c1["dt"]))
        np.testing.assert_allclose(md.energy.cpu().numpy()[0], c1[f"{name}/epot"][step],
                                   rtol=1e-10)
        if step % every == 0:
            k = step // every
            np.testing.assert_allclose(md.positions.cpu().numpy(), c1[f"{name}/positions"][k],
                                       rtol=0, atol=1e-9)
            np.testing.assert_allclose(md.momenta.cpu().numpy(), c1[f"{name}/momenta"][k],
                                       rtol=1e-7, atol=1e-9)
            s = m(md)["stress"].cpu().numpy()[0]
            np.testing.assert_allclose(s, c1[f"{name}/stress"][step], rtol=1e-8, atol=1e-13)


@pytest.mark.parametrize("name", ["lj", "lj_shift"])
def test_fused_kernel_on_config1(c1, name):
    from oracle import pair as opair
    from tsb import integrators, quantities

    md = _state(c1, name)
    m = _model(name, "mixed")
    r = integrators.FusedMD(md, m, integrator="nve", dt=float(c1["dt"]), skin=1.0, seed=0)
    every = int(c1["every"])
    etot = []
    for k in range(1, 11):
        r.launch(every)
        torch.cuda.synchronize()
        r.check()
        dx = np.abs(r.x.cpu().numpy() - c1[f"{name}/positions"][k]).max()
        assert dx <= 2e-4, (k, dx)
        ke = quantities.calc_kinetic_energy(masses=md.masses, momenta=r.p,
                                            system_idx=md.system_idx, n_systems=1)
        etot.append(float(r.energy[0] + ke[0]))
    x = r.x.cpu().numpy()
    shift = float(c1["shift"]) if name == "lj_shift" else 0.0
    ref = opair.pair_forward(opair.LJ, opair.single_table(opair.LJ, SIGMA, EPS, eshift=shift),
                             np.zeros(256, int), x, np.transpose(c1["init/cell"], (0, 2, 1)),
                             c1["init/pbc"], c1["init/system_idx"], RC)
    ferr = np.abs(r.f.cpu().numpy() - ref["forces"]).max() / np.abs(ref["forces"]).max()
    assert ferr <= 1e-5, ferr
    np.testing.assert_allclose(r.energy.cpu().numpy(), ref["energy"], rtol=2e-6)
    if name == "lj_shift":
        e0 = c1["lj_shift/epot"][0] + c1["lj_shift/ekin"][0]
        drift = np.abs(np.array(etot) - e0).max()
        assert drift <= 2e-4, drift
