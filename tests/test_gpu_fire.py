"""GPU FIRE (+ Frechet cell filter) vs the reference trajectories and the oracle.

Tolerances: ASE-FIRE + Frechet rtol 1e-7 (FP64; the reference picks the Pade
scaling from the whole batch and takes the matrix log by eigen-cases, tsb per
system and by inverse scaling-and-squaring -- both agree to rounding); VV-FIRE
rtol 1e-9.
"""

import numpy as np
import pytest
import torch

from oracle import fire as ofire
from oracle import pair as opair

pytestmark = pytest.mark.gpu


def _ka_state(g, k=0, cell=None):
    from tsb.state import SimState

    dev = torch.device("cuda")
    T = lambda x, dt=torch.float64: torch.as_tensor(np.asarray(x), dtype=dt, device=dev)  # noqa
    c = g["cell"][k] if cell is None else cell
    return SimState(positions=T(g["positions"][k]), masses=T(g["masses"]),
                    cell=T(c), pbc=True,
                    atomic_numbers=T(g["atomic_numbers"], torch.int64),
                    system_idx=T(g["system_idx"], torch.int64))


def _ka_model(stress=True):
    from tsb import models

    return models.kob_andersen_model(compute_stress=stress, precision="fp64")


def test_ase_fire_frechet_matches_reference(golden):
    from tsb import optimizers

    g = golden["fire"]["ase_frechet"]
    m = _ka_model()
    st = optimizers.fire_init(_ka_state(g), m, cell_filter="frechet")
    np.testing.assert_allclose(st.cell_forces.cpu(), g["cell_forces"][0], rtol=1e-9,
                               atol=1e-12)
    for k in range(1, g["positions"].shape[0]):
        st = optimizers.fire_step(st, m)
        for key in ("positions", "cell", "energy", "forces", "cell_forces", "cell_positions",
                    "velocities", "dt", "alpha"):
            got = getattr(st, key).cpu().numpy()
            np.testing.assert_allclose(got, g[key][k], rtol=1e-7, atol=1e-10,
                                       err_msg=f"step {k} {key}")
        np.testing.assert_array_equal(st.n_pos.cpu().numpy(), g["n_pos"][k])


def test_vv_fire_matches_reference(golden):
    from tsb import optimizers

    g = golden["fire"]["vv"]
    m = _ka_model(stress=False)
    st = optimizers.fire_init(_ka_state(g, cell=g["cell"]), m, fire_flavor="vv_fire")
    for k in range(1, g["positions"].shape[0]):
        st = optimizers.fire_step(st, m, fire_flavor="vv_fire")
        for key in ("positions", "energy", "forces", "velocities", "dt", "alpha"):
            np.testing.assert_allclose(getattr(st, key).cpu().numpy(), g[key][k], rtol=1e-9,
                                       atol=1e-11, err_msg=f"step {k} {key}")
        np.testing.assert_array_equal(st.n_pos.cpu().numpy(), g["n_pos"][k])


def test_frechet_cell_forces_deformed_cell_vs_oracle():
    """Cell forces for a strained + sheared cell (logm, Frechet adjoint)."""
    from tsb import optimizers, workloads
    from tsb.state import state_from_arrays

    d = workloads.kob_andersen_batch(3, 64, 120, seed=21)
    st0 = state_from_arrays(d, device="cuda")
    m = _ka_model()
    st = optimizers.fire_init(st0, m, cell_filter="frechet")
    rng = np.random.default_rng(3)
    Fd = np.eye(3)[None] + rng.normal(0, 0.04, (3, 3, 3))
    new_cell = Fd @ d["cell"]
    st.cell = torch.as_tensor(new_cell, device="cuda").contiguous()
    st.stress = torch.as_tensor(rng.normal(0, 1e-3, (3, 3, 3)), device="cuda").contiguous()
    optimizers._cell_forces(st, init=False)
    ref = {"cell": new_cell, "reference_cell": d["cell"], "stress": st.stress.cpu().numpy(),
           "pressure": np.zeros((3, 3, 3)),
           "cell_factor": np.bincount(d["system_idx"]).astype(float)}
    ofire.compute_cell_forces(ref)
    np.testing.assert_allclose(st.cell_forces.cpu().numpy(), ref["cell_forces"], rtol=1e-10,
                               atol=1e-14)


def test_optimize_batched_converges_with_frozen_systems():
    from tsb import optimizers, workloads
    from tsb.state import state_from_arrays

    d = workloads.kob_andersen_batch(6, 64, 160, seed=8)
    st = state_from_arrays(d, device="cuda")
    m = _ka_model()
    e0 = m(st)["energy"].cpu().numpy()
    st, steps, conv = optimizers.optimize(st, m, fmax=1e-3, max_steps=6000,
                                          cell_filter="frechet")
    assert bool(conv.all()), (steps, conv)
    out = m(st)
    fmax = torch.zeros(6, dtype=torch.float64, device="cuda").scatter_reduce(
        0, st.system_idx, out["forces"].norm(dim=1), reduce="amax")
    # frozen at the step they converged: their stored forces are below fmax
    assert float(fmax.max()) < 1e-3
    assert float(st.cell_forces.norm(dim=2).max()) < 1e-3
    assert np.all(out["energy"].cpu().numpy() < e0)


def test_fire_nan_isolation():
    """A fresh (NaN-velocity) system does not perturb its batch neighbours
    (test_optimizers.py:722-786)."""
    from tsb import optimizers, workloads
    from tsb.state import state_from_arrays

    d = workloads.kob_andersen_batch(3, 64, 100, seed=2)
    m = _ka_model(stress=False)
    a = optimizers.fire_init(state_from_arrays(d, device="cuda"), m)
    for _ in range(5):
        a = optimizers.fire_step(a, m)
    b = a.clone()
    sel = b.system_idx == 1
    b.velocities[sel] = float("nan")
    a = optimizers.fire_step(a, m)
    b = optimizers.fire_step(b, m)
    other = ~sel
    assert torch.equal(a.positions[other], b.positions[other])
    assert torch.isfinite(b.positions).all()


def test_graph_replayed_relax_equals_eager_steps():
    """The relax loop as CUDA-graph replays (FIRE + Frechet step, device-decided
    Verlet-list rebuilds, convergence mask) equals the same steps run eagerly,
    bitwise, and leaves converged systems frozen."""
    from tsb import models, optimizers, workloads
    from tsb.state import state_from_arrays

    d = workloads.kob_andersen_batch(5, 64, 200, seed=12)
    outs = []
    for graph in (False, True):
        st = state_from_arrays(d, device="cuda")
        m = models.VerletListModel(_ka_model(), skin=1.0)
        st = optimizers.fire_init(st, m, cell_filter="frechet")
        n_steps, k = 60, 20
        if graph:
            st, steps, conv = optimizers.optimize(st, m, fmax=1e-9, max_steps=n_steps,
                                                  cell_filter="frechet", graph_steps=k)
            assert steps == n_steps
        else:
            active = torch.ones(st.n_systems, dtype=torch.uint8, device="cuda")
            n_active = torch.zeros(1, dtype=torch.int32, device="cuda")
            optimizers.converged_mask(st, 1e-9, True, active, n_active)
            for _ in range(n_steps):
                optimizers.fire_step(st, m, active=active)
                optimizers.converged_mask(st, 1e-9, True, active, n_active)
        torch.cuda.synchronize()
        outs.append((st.positions.clone(), st.cell.clone(), st.energy.clone(),
                     st.forces.clone(), m.n_builds))
    for a, b in zip(outs[0][:4], outs[1][:4]):
        assert torch.equal(a, b)
