"""The ``torch.ops.tsb`` operators on the GPU, and the drop-ins fed a state with
exactly the reference SimState's fields.

* A loop of per-call ``nvt_langevin_step`` (neighbour search + pair forces +
  BAOAB kernels, all through the operators) captured in one CUDA graph and
  replayed equals the same steps run eagerly, bitwise; the device-resident noise
  counter advances on every replay.
* ``torch.compile(fullgraph=True)`` traces through the pair operator.
* The interface checks of the reference's ``validate_model_outputs``
  (torch_sim/models/interface.py:387-611): no mutation of the input, output
  keys and shapes, batched == single-system outputs (atol 1e-4), invariance
  under a lattice translation of one atom, a non-periodic molecule -- on a
  state object that carries only ``torch_sim.SimState``'s fields with its
  column-vector cell (torch_sim/state.py:120-325).
"""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _cu_md(n_sys=6, seed=3):
    from tsb import integrators, models, workloads
    from tsb.state import state_from_arrays

    d = workloads.copper_batch(n_sys, 8, 300, seed=seed)
    st = state_from_arrays(d, device="cuda")
    st.rng = seed
    m = models.MorseModel(sigma=2.866, epsilon=0.3429, alpha=1.3588, cutoff=6.0)
    return integrators.nvt_langevin_init(st, m, kT=1000 * workloads.KB_EV), m


def test_per_call_langevin_loop_captured_in_a_cuda_graph():
    from tsb import integrators, workloads

    md, m = _cu_md()
    kw = dict(dt=0.002 * workloads.METAL_TIME, kT=1000 * workloads.KB_EV,
              gamma=10.0 / workloads.METAL_TIME)
    a, b = md.clone(), md.clone()
    for s in (a, b):
        s._philox_seed, s._philox_counter = 11, 0
        integrators.use_device_counter(s)
    k = 5
    # eager: 2 k steps
    for _ in range(2 * k):
        a = integrators.nvt_langevin_step(a, m, **kw)
    # warm-up on the state to be captured (workspaces, cached sizes), on a side
    # stream, then put its state back
    snap = {f: getattr(b, f).clone() for f in ("positions", "momenta", "forces", "energy")}
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        integrators.nvt_langevin_step(b, m, **kw)
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    for f, v in snap.items():
        setattr(b, f, v.clone())
    b._philox_counter = 0
    b._philox_counter_dev.zero_()
    torch.cuda.synchronize()
    with torch.cuda.graph(g):
        for _ in range(k):
            b = integrators.nvt_langevin_step(b, m, **kw)
    # capture runs nothing: b is still the initial state with counter 0
    assert int(b._philox_counter_dev.item()) == 0
    g.replay()
    g.replay()
    torch.cuda.synchronize()
    assert int(b._philox_counter_dev.item()) == 2 * k
    assert int(a._philox_counter_dev.item()) == 2 * k
    assert torch.equal(a.positions, b.positions)
    assert torch.equal(a.momenta, b.momenta)
    assert torch.equal(a.forces, b.forces)
    assert torch.equal(a.energy, b.energy)


def test_torch_compile_traces_the_pair_operator():
    from tsb import _lib as L

    md, m = _cu_md(4, seed=5)
    ins = m._inputs(md)
    n_sys = md.n_systems
    msa = L.max_system_atoms(md.system_idx, n_sys)
    flags = L.OUT_FORCES | L.OUT_STRESS

    def f(pos):
        e, frc, st, _, _ = torch.ops.tsb.pair_forward(pos, *ins[1:], m.kind, m.n_species,
                                                      m.cutoff, flags, n_sys, msa)
        return e.sum(), frc * 2.0, st

    cf = torch.compile(f, fullgraph=True, backend="aot_eager")
    got = cf(ins[0])
    ref = f(ins[0])
    for u, v in zip(got, ref):
        torch.testing.assert_close(u, v, rtol=0, atol=0)


# ------------------------------------------------ reference-shaped state object
@dataclasses.dataclass
class RefShapedState:
    """Carries exactly the fields of torch_sim.SimState (state.py:120-180):
    positions [N,3], masses [N], cell [S,3,3] (column vectors), pbc [3] bool,
    atomic_numbers [N], system_idx [N]; plus the derived properties the
    reference defines on it (n_atoms, n_systems, device, dtype, clone)."""

    positions: torch.Tensor
    masses: torch.Tensor
    cell: torch.Tensor
    pbc: torch.Tensor
    atomic_numbers: torch.Tensor
    system_idx: torch.Tensor

    @property
    def n_atoms(self) -> int:
        return self.positions.shape[0]

    @property
    def n_systems(self) -> int:
        return int(torch.unique(self.system_idx).shape[0])

    @property
    def device(self) -> torch.device:
        return self.positions.device

    @property
    def dtype(self) -> torch.dtype:
        return self.positions.dtype

    @property
    def rng(self):
        """The reference's lazily seeded generator; unseeded here (None)."""
        return None

    def clone(self) -> "RefShapedState":
        return RefShapedState(*(getattr(self, f.name).clone()
                                for f in dataclasses.fields(self)))


def _structures():
    """Si diamond (8 atoms, a = 5.43, cubic), Mg hcp (a = 3.21, c = 5.21) repeated
    3x2x1 (12 atoms), Fe bcc primitive (1 atom, a = 2.87): the three systems of
    the reference's validator, built from their lattice definitions."""
    fcc = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0]])
    si_f = np.concatenate([fcc, fcc + 0.25])
    si_cell = np.eye(3) * 5.43
    a, c = 3.21, 5.21
    mg_prim = np.array([[a, 0, 0], [-a / 2, a * np.sqrt(3) / 2, 0], [0, 0, c]])
    mg_basis = np.array([[1 / 3, 2 / 3, 0.25], [2 / 3, 1 / 3, 0.75]])
    mg_f = np.array([(b + [i, j, 0]) / [3, 2, 1] for i in range(3) for j in range(2)
                     for b in mg_basis])
    mg_cell = mg_prim * np.array([[3], [2], [1]])
    fe_cell = 2.87 / 2 * np.array([[-1, 1, 1], [1, -1, 1], [1, 1, -1]])
    fe_f = np.zeros((1, 3))
    return [(si_f @ si_cell, si_cell, 14, 28.0855), (mg_f @ mg_cell, mg_cell, 12, 24.305),
            (fe_f @ fe_cell, fe_cell, 26, 55.845)]


def _state(systems, periodic=True):
    dev = torch.device("cuda")
    pos = np.concatenate([s[0] for s in systems])
    z = np.concatenate([np.full(len(s[0]), s[2]) for s in systems])
    mass = np.concatenate([np.full(len(s[0]), s[3]) for s in systems])
    sysi = np.concatenate([np.full(len(s[0]), k) for k, s in enumerate(systems)])
    cell = np.stack([s[1].T for s in systems])  # column-vector convention
    T = lambda x, dt=torch.float64: torch.as_tensor(x, dtype=dt, device=dev)  # noqa: E731
    return RefShapedState(T(pos), T(mass), T(cell), T([periodic] * 3, torch.bool),
                          T(z, torch.int64), T(sysi, torch.int64))


def _benzene():
    ang = np.arange(6) * np.pi / 3
    ring = lambda r: np.stack([r * np.cos(ang), r * np.sin(ang), np.zeros(6)], 1)  # noqa
    pos = np.concatenate([ring(1.397), ring(2.481)])
    return [(pos, np.zeros((3, 3)), 6, 12.011)], np.array([6] * 6 + [1] * 6)


@pytest.mark.parametrize("model_name", ["lj", "morse", "soft_sphere"])
def test_models_satisfy_the_reference_interface_checks(model_name):
    from tsb import models

    ctor = {"lj": lambda: models.LennardJonesModel(sigma=2.0, epsilon=0.01, cutoff=5.0,
                                                   compute_stress=True),
            "morse": lambda: models.MorseModel(sigma=2.5, epsilon=0.3, alpha=1.4,
                                               cutoff=5.0, compute_stress=True),
            "soft_sphere": lambda: models.SoftSphereModel(sigma=2.6, epsilon=0.05,
                                                          alpha=2.0, cutoff=2.6,
                                                          compute_stress=True)}
    m = ctor[model_name]()
    atol = 1e-4  # VALIDATE_ATOL, interface.py:47
    systems = _structures()
    st = _state(systems)
    og = st.clone()
    out = m(st)
    for f in dataclasses.fields(st):  # the model did not mutate its input
        assert torch.equal(getattr(st, f.name), getattr(og, f.name)), f.name
    assert {"energy", "forces", "stress"} <= set(out)
    assert out["energy"].shape == (3,) and out["forces"].shape == (21, 3)
    assert out["stress"].shape == (3, 3, 3)
    assert all(not v.requires_grad for v in out.values())
    off = 0
    singles = []
    for k, sysdef in enumerate(systems):
        s1 = _state([sysdef])
        o1 = m(s1)
        n = s1.n_atoms
        assert o1["energy"].shape == (1,) and o1["forces"].shape == (n, 3)
        assert o1["stress"].shape == (1, 3, 3)
        torch.testing.assert_close(o1["energy"], out["energy"][k:k + 1], atol=atol, rtol=0)
        torch.testing.assert_close(o1["forces"], out["forces"][off:off + n], atol=atol, rtol=0)
        off += n
        singles.append((s1, o1))
    # translate one Si atom by three lattice vectors (column convention): unchanged
    s1, o1 = singles[0]
    sh = s1.clone()
    sh.positions[0] = sh.positions[0] + 3 * sh.cell[0, :, 0]
    o2 = m(sh)
    for key in ("energy", "forces", "stress"):
        torch.testing.assert_close(o2[key], o1[key], atol=atol, rtol=0)
    # a non-periodic molecule
    mol, z = _benzene()
    bs = _state(mol, periodic=False)
    bs.atomic_numbers = torch.as_tensor(z, device="cuda")
    ob = m(bs)
    assert ob["energy"].shape == (1,) and ob["forces"].shape == (12, 3)
    assert torch.isfinite(ob["forces"]).all()


def test_reference_shaped_state_through_a_step_function():
    """nve_init / nve_step take the reference-shaped state (as ts.integrate hands
    the registered (init, step) pair its SimState, runners.py:308-320)."""
    from tsb import integrators, models, workloads

    st = _state(_structures()[:2])
    m = models.LennardJonesModel(sigma=2.0, epsilon=0.01, cutoff=5.0)
    md = integrators.nve_init(st, m, kT=100 * workloads.KB_EV)
    e0 = md.energy.clone()
    for _ in range(5):
        md = integrators.nve_step(md, m, dt=0.001 * workloads.METAL_TIME)
    assert md.positions.shape == st.positions.shape
    assert torch.isfinite(md.energy).all() and not torch.equal(md.energy, e0)


@pytest.mark.parametrize("name", ["nve", "nvt_langevin"])
def test_steps_driven_like_the_reference_runner(name):
    """ts.integrate with an (init, step) tuple (torch_sim/runners.py:308-396)
    converts the timestep (ps) and temperature (K) to internal units as 0-d
    tensors on the state's device, then calls init_func(state=, model=, kT=, dt=)
    and step_func(state=, model=, dt=, kT=) by keyword.  The tsb pairs take
    exactly that and give the same trajectory as calls with plain floats."""
    from tsb import integrators, workloads

    init, step = {"nve": (integrators.nve_init, integrators.nve_step),
                  "nvt_langevin": (integrators.nvt_langevin_init,
                                   integrators.nvt_langevin_step)}[name]
    md0, m = _cu_md(3, seed=8)
    st = md0.clone()
    dev, dt_ = st.device, st.dtype
    timestep, temperature = 0.002, 800.0                 # ps, K (the runner's inputs)
    kTs = torch.as_tensor(temperature, dtype=dt_, device=dev).expand(4) * workloads.KB_EV
    dt = torch.as_tensor(timestep * workloads.METAL_TIME, dtype=dt_, device=dev)
    a = init(state=st, model=m, kT=kTs[0], dt=dt)
    a._philox_seed, a._philox_counter = 5, 0
    for k in range(4):
        a = step(state=a, model=m, dt=dt, kT=kTs[k])
    b = init(md0.clone(), m, kT=temperature * workloads.KB_EV)
    b._philox_seed, b._philox_counter = 5, 0
    for _ in range(4):
        b = step(b, m, dt=float(dt), kT=temperature * workloads.KB_EV)
    torch.testing.assert_close(a.positions, b.positions, rtol=0, atol=0)
    torch.testing.assert_close(a.momenta, b.momenta, rtol=0, atol=0)
