"""The persistent fused MD kernel against the oracle, on the batched Cu workload.

The fused kernel (FP32 pair arithmetic, FP64 positions, momenta, energy and
virial) advances a batch of Cu fcc systems with Morse forces (strained and
sheared triclinic cells, 8-512 atoms) by several launches of 20 steps; the
oracle (``oracle.fused_md``: FP64 reference pair model, reference integrator
steps, the kernel's own Philox draws) replays the same trajectories.  Compared
after every launch:

* forces at the kernel's positions vs the FP64 oracle forces there:
  max|dF| / max|F| <= 1e-5 (the precision bar of the FP32 pair arithmetic);
* potential energy and stress at the kernel's positions vs FP64:
  relative 2e-6 (energy) and 1e-5 of max|stress| (virial), both summed in FP64;
* the trajectories themselves: positions within 1e-3 A and momenta within
  5e-3 sqrt(m kT) of the oracle's.  Each step the FP32 forces differ from FP64
  by ~6e-6 of max|F|; with smooth forces those differences grow to ~1e-6 A and
  ~1e-5 sqrt(m kT) over 60 steps (measured on B200).  The reference's Morse is
  truncated without a shift, so its force jumps by F(rc) = 0.013 eV/A when a
  pair crosses the cutoff; two trajectories 1e-7 A apart can see a crossing one
  step apart, which moves one momentum by F(rc) dt = 1.1e-3 sqrt(m kT) and the
  positions by ~1e-4 A over the following 20 steps (measured: 7.8e-4
  sqrt(m kT) and 7.7e-5 A in the NVE run).  The bounds allow a few such events.

Reference: torch_sim/integrators/nvt.py:27-86, 144-240 (BAOAB), nve.py:74-130,
nvt.py:381-488 (Nose-Hoover chain), nvt.py:715-741 (V-rescale),
torch_sim/models/pair_potential.py:200-274 (stress), morse.py:23-47.
"""

import numpy as np
import pytest
import torch

from oracle import fused_md, pair as opair

pytestmark = pytest.mark.gpu

MORSE = (2.866, 0.3429, 1.3588)


def _batch(n_sys, seed):
    """Seeded Cu batch with at least two systems of 400-512 atoms."""
    from tsb import workloads

    d = workloads.copper_batch(n_sys, 8, 512, seed=seed)
    counts = np.bincount(d["system_idx"])
    assert (counts >= 400).sum() >= 2, counts
    return d


def _setup(n_sys, seed, integrator, skin=0.7):
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = _batch(n_sys, seed)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed + 100
    m = models.MorseModel(sigma=MORSE[0], epsilon=MORSE[1], alpha=MORSE[2], cutoff=6.0)
    kT = 1000.0 * workloads.KB_EV
    dt = 0.002 * workloads.METAL_TIME
    gamma = 10.0 / workloads.METAL_TIME
    if integrator == "nvt_nose_hoover":
        md = integrators.nvt_nose_hoover_init(st, m, kT=kT, dt=dt)
    else:
        md = integrators.nvt_langevin_init(st, m, kT=kT)
    r = integrators.FusedMD(md, m, integrator=integrator, dt=dt,
                            kT=None if integrator == "nve" else kT,
                            gamma=gamma if integrator == "nvt_langevin" else None,
                            skin=skin, seed=4242 + seed)
    return d, md, r, dict(dt=dt, kT=kT, gamma=gamma)


def _oracle_forces(d, x):
    tab = opair.single_table(opair.MORSE, *MORSE)
    cell_row = np.transpose(d["cell"], (0, 2, 1))
    pbc = np.ones((cell_row.shape[0], 3), bool)
    return opair.pair_forward(opair.MORSE, tab, np.zeros(len(x), int), x, cell_row, pbc,
                              d["system_idx"], 6.0)


def _compare_at_kernel_positions(d, r):
    x = r.x.cpu().numpy()
    ref = _oracle_forces(d, x)
    f = r.f.cpu().numpy()
    err = np.abs(f - ref["forces"]).max() / np.abs(ref["forces"]).max()
    assert err <= 1e-5, err
    e = r.energy.cpu().numpy()
    print(f"  energy rel err {np.abs(e / ref['energy'] - 1).max():.2e}", end="")
    np.testing.assert_allclose(e, ref["energy"], rtol=2e-6)
    s = r.stress.cpu().numpy()
    serr = np.abs(s - ref["stress"]).max() / np.abs(ref["stress"]).max()
    print(f", stress err {serr:.2e}")
    assert serr <= 1e-5, serr
    return err


def _run_compare(n_sys, seed, integrator, launches=3, per=20):
    from tsb import workloads

    # a narrow skin (0.4 A) makes the lists expire every few steps
    d, md, r, kw = _setup(n_sys, seed, integrator, skin=0.4)
    counts = np.bincount(d["system_idx"])
    x0, p0, f0 = (t.cpu().numpy().copy() for t in (r.x, r.p, r.f))
    chain = None
    if integrator == "nvt_nose_hoover":
        c = md.chain
        chain = {"xi": c.positions.cpu().numpy(), "p_xi": c.momenta.cpu().numpy(),
                 "ke": c.kinetic_energy.cpu().numpy(), "dof": c.degrees_of_freedom.cpu().numpy(),
                 "tau": c.tau.cpu().numpy()}
    tab = opair.single_table(opair.MORSE, *MORSE)
    cell_row = np.transpose(d["cell"], (0, 2, 1))
    sp = np.zeros(len(x0), int)
    pscale = np.sqrt(d["masses"] * kw["kT"])[:, None]
    xs, ps, fs = x0, p0, f0
    rebuilds = np.zeros(n_sys)
    for k in range(launches):
        r.launch(per)
        torch.cuda.synchronize()
        r.check()
        rebuilds += r.rebuilds.cpu().numpy()
        o = fused_md.run(opair.MORSE, tab, sp, xs, ps, fs, d["masses"], cell_row,
                         d["system_idx"], 6.0, per, kw["dt"], integrator=integrator,
                         kT=kw["kT"], gamma=kw["gamma"], seed=r.seed, counter=k * per,
                         skin=1.0, chain=chain, chain_steps=getattr(md, "chain_steps", 1),
                         sy_steps=getattr(md, "sy_steps", 1))
        xs, ps, fs, chain = o["positions"], o["momenta"], o["forces"], o.get("chain")
        ferr = _compare_at_kernel_positions(d, r)
        dx = np.abs(r.x.cpu().numpy() - xs).max()
        dp = (np.abs(r.p.cpu().numpy() - ps) / pscale).max()
        print(f"{integrator} launch {k}: force err {ferr:.2e}, max|dx| {dx:.2e} A, "
              f"max|dp|/sqrt(m kT) {dp:.2e}")
        assert dx <= 1e-3, (k, dx)
        assert dp <= 5e-3, (k, dp)
        # the trajectory moved (several list lifetimes) and stayed physical
        assert np.abs(xs - x0).max() > 0.1
        assert np.isfinite(r.energy.cpu().numpy()).all()
    # every launch starts with a list build; the larger systems also rebuilt
    # their lists inside the launches (list reuse and device-side rebuilds)
    assert (rebuilds >= launches).all(), rebuilds
    assert (rebuilds[counts >= 200] >= launches + 1).all(), (rebuilds, counts)
    assert counts.max() >= 400
    if integrator == "nvt_nose_hoover":
        for got, ref in ((r.cxi, chain["xi"]), (r.cpxi, chain["p_xi"])):
            got = got.cpu().numpy()
            assert np.abs(got - ref).max() <= 1e-4 * np.abs(ref).max(), (got, ref)
    return workloads


@pytest.mark.parametrize("integrator", ["nvt_langevin", "nve"])
def test_fused_trajectory_matches_oracle(integrator):
    _run_compare(16, 1, integrator)


@pytest.mark.parametrize("integrator", ["nvt_nose_hoover", "nvt_vrescale"])
def test_fused_thermostat_trajectory_matches_oracle(integrator):
    _run_compare(8, 3, integrator, launches=2)


def test_fused_stress_matches_model_stress():
    """The kernel's FP64-summed stress equals the per-call FP64 model's stress
    at the same positions (pair_potential.py:200-274)."""
    from tsb import models

    d, md, r, kw = _setup(12, 5, "nvt_langevin")
    r.launch(30)
    torch.cuda.synchronize()
    r.check()
    md.positions = r.x.clone()
    ref = models.MorseModel(sigma=MORSE[0], epsilon=MORSE[1], alpha=MORSE[2], cutoff=6.0,
                            precision="fp64", compute_stress=True)(md)
    s, rs = r.stress.cpu().numpy(), ref["stress"].cpu().numpy()
    assert np.abs(s - rs).max() / np.abs(rs).max() <= 1e-5
    np.testing.assert_allclose(s, np.transpose(s, (0, 2, 1)), rtol=0, atol=0)
    np.testing.assert_allclose(r.energy.cpu().numpy(), ref["energy"].cpu().numpy(), rtol=2e-6)
