"""FIRE optimisation with the Frechet cell filter on the tsb kernels.

Drop-ins for the reference optimizer registry (torch_sim/optimizers/__init__.py:47-52):

* ``fire_init(state, model, *, dt_start, alpha_start, fire_flavor, cell_filter,
  **filter_kwargs)``  <- torch_sim/optimizers/fire.py:21-114 and
  frechet_cell_filter_init (cell_filters.py:230-284)
* ``fire_step(state, model, *, dt_max, n_min, f_inc, f_dec, alpha_start, f_alpha,
  max_step, fire_flavor)`` <- fire.py:117-176 with _ase_fire_step (:288-499) and
  _vv_fire_step (:179-285), compute_cell_forces (cell_filters.py:353-399)
* ``generate_force_convergence_fn`` <- runners.py:501-538
* ``optimize(...)`` -- batched relaxation in which converged systems are frozen
  on the device (a per-system mask read by every kernel, the force kernel
  included) instead of being swapped out of the batch by the host autobatcher
  (autobatching.py:1040-1152, kept only as an admission policy).

Only ``cell_filter`` None or "frechet" is supported (the unit-cell filter is
not on this hot path).
"""

from __future__ import annotations

import torch

from . import _lib as L
from . import ops as _ops  # noqa: F401  (registers torch.ops.tsb.*)
from .state import CellFireState, FireState

ASE, VV = "ase_fire", "vv_fire"


def _cell_filter_name(cell_filter):
    if cell_filter is None:
        return None
    name = getattr(cell_filter, "value", cell_filter)
    if name != "frechet":
        raise NotImplementedError(f"cell filter {cell_filter!r}: only 'frechet' is supported")
    return name


def _counts(state):
    return torch.bincount(state.system_idx, minlength=state.n_systems)


def _eval_model(state, model, active=None):
    """Model forward writing into the state's buffers; systems with active == 0
    keep their previous forces/energy/stress."""
    if active is None or not hasattr(model, "forward_into"):
        out = model(state)
        state.forces = out["forces"].contiguous()
        state.energy = out["energy"]
        if "stress" in out:
            state.stress = out["stress"]
        return
    model.forward_into(state, energy=state.energy, forces=state.forces,
                       stress=getattr(state, "stress", None), sys_active=active)


def _cell_forces(state, init, active=None):
    torch.ops.tsb.frechet_cell_forces_(state.cell_forces, state.stress, state.cell,
                                       state.reference_cell, state.pressure, state.cell_factor,
                                       int(init), active)


def fire_init(state, model, *, dt_start=0.1, alpha_start=0.1, fire_flavor=ASE,
              cell_filter=None, cell_factor=None, scalar_pressure=0.0, **_filter_kwargs):
    if fire_flavor not in (ASE, VV):
        raise ValueError(f"Unknown fire_flavor={fire_flavor!r}")
    L.require_cuda(state.positions, "state.positions")
    cf_name = _cell_filter_name(cell_filter)
    dev, dt_ = state.device, state.dtype
    n_sys = state.n_systems
    out = model(state)
    stress = out.get("stress")
    common = dict(forces=out["forces"].contiguous(), energy=out["energy"], stress=stress,
                  velocities=torch.full_like(state.positions, float("nan")),
                  dt=torch.full((n_sys,), float(dt_start), dtype=dt_, device=dev),
                  alpha=torch.full((n_sys,), float(alpha_start), dtype=dt_, device=dev),
                  n_pos=torch.zeros(n_sys, dtype=torch.int32, device=dev))
    if cf_name is None:
        st = FireState.from_state(state, **common)
        st.positions = st.positions.contiguous().clone()
        return st
    if stress is None:
        raise ValueError("the Frechet cell filter needs a model with compute_stress=True")
    counts = _counts(state).to(dt_)
    if cell_factor is None:
        cfac = counts
    else:
        cfac = torch.as_tensor(cell_factor, dtype=dt_, device=dev).expand(n_sys).contiguous()
    # cell masses (cell_filters.py:97-101): summed on the host, in atom order, so
    # that repeated runs get bitwise equal values (a GPU index_add_ sums in a
    # run-dependent order)
    masses = torch.zeros(n_sys, dtype=dt_).index_add_(
        0, state.system_idx.cpu(), state.masses.to(dt_).cpu()).to(dev)
    st = CellFireState.from_state(
        state, **common, reference_cell=state.cell.clone().contiguous(), cell_filter="frechet",
        cell_factor=cfac.contiguous(),
        pressure=(float(scalar_pressure) * torch.eye(3, dtype=dt_, device=dev)).expand(
            n_sys, 3, 3).contiguous(),
        cell_positions=torch.zeros((n_sys, 3, 3), dtype=dt_, device=dev),
        cell_forces=torch.zeros((n_sys, 3, 3), dtype=dt_, device=dev),
        cell_velocities=torch.full((n_sys, 3, 3), float("nan"), dtype=dt_, device=dev),
        cell_masses=masses)
    st.positions = st.positions.contiguous().clone()
    st.cell = st.cell.contiguous().clone()
    st.stress = st.stress.contiguous()
    _cell_forces(st, init=True)
    return st


def _fire_kernel(name, state, hyper, active):
    is_cell = isinstance(state, CellFireState)
    c = (lambda k: getattr(state, k)) if is_cell else (lambda k: None)  # noqa: E731
    op = {"tsb_fire_ase_pre": torch.ops.tsb.fire_ase_pre_,
          "tsb_fire_vv_pre": torch.ops.tsb.fire_vv_pre_,
          "tsb_fire_vv_post": torch.ops.tsb.fire_vv_post_}[name]
    op(1 if is_cell else 0, state.positions, state.velocities, state.forces, state.masses,
       state.system_idx, state.dt, state.alpha, state.n_pos, c("cell"), c("reference_cell"),
       c("cell_factor"), c("cell_positions"), c("cell_velocities"), c("cell_forces"),
       c("cell_masses"), active, float(hyper["dt_max"]), int(hyper["n_min"]),
       float(hyper["f_inc"]), float(hyper["f_dec"]), float(hyper["alpha_start"]),
       float(hyper["f_alpha"]), float(hyper["max_step"]), float(hyper["eps"]))


def _contiguous(state):
    for k in ("positions", "velocities", "forces", "masses", "dt", "alpha", "n_pos",
              "system_idx"):
        t = getattr(state, k)
        if not t.is_contiguous():
            setattr(state, k, t.contiguous())


def fire_step(state, model, *, dt_max=1.0, n_min=5, f_inc=1.1, f_dec=0.5, alpha_start=0.1,
              f_alpha=0.99, max_step=0.2, fire_flavor=ASE, active=None):
    """One FIRE step (mutates and returns ``state``).  ``active`` (uint8 [S],
    optional) freezes systems with 0."""
    if fire_flavor not in (ASE, VV):
        raise ValueError(f"Unknown fire_flavor={fire_flavor!r}")
    _contiguous(state)
    eps = 1e-8 if state.dtype == torch.float32 else 1e-16
    hyper = dict(dt_max=dt_max, n_min=n_min, f_inc=f_inc, f_dec=f_dec,
                 alpha_start=alpha_start, f_alpha=f_alpha, max_step=max_step, eps=eps)
    is_cell = isinstance(state, CellFireState)
    if fire_flavor == ASE:
        _fire_kernel("tsb_fire_ase_pre", state, hyper, active)
        _eval_model(state, model, active)
        if is_cell:
            _cell_forces(state, init=False, active=active)
    else:
        _fire_kernel("tsb_fire_vv_pre", state, hyper, active)
        _eval_model(state, model, active)
        if is_cell:
            _cell_forces(state, init=False, active=active)
        _fire_kernel("tsb_fire_vv_post", state, hyper, active)
    return state


def generate_force_convergence_fn(force_tol=1e-1, *, include_cell_forces=False):
    """Per-system convergence test (runners.py:501-538), evaluated on the device."""

    def convergence_fn(state, last_energy=None):  # noqa: ARG001
        active = torch.ones(state.n_systems, dtype=torch.uint8, device=state.device)
        n_active = torch.zeros(1, dtype=torch.int32, device=state.device)
        converged_mask(state, force_tol, include_cell_forces, active, n_active)
        return active == 0

    return convergence_fn


def converged_mask(state, fmax, include_cell_forces, active, n_active):
    cf = state.cell_forces if (include_cell_forces and isinstance(state, CellFireState)) else None
    if include_cell_forces and cf is None:
        raise ValueError("cell_forces not found in state")
    torch.ops.tsb.fire_converged_(state.forces, state.system_idx, state.n_systems, cf,
                                  float(fmax), active, n_active)


_GRAPH_FIELDS = ("positions", "velocities", "forces", "energy", "stress", "dt", "alpha", "n_pos",
                 "cell", "cell_positions", "cell_velocities", "cell_forces")


def _snapshot(state):
    return {k: getattr(state, k).clone() for k in _GRAPH_FIELDS
            if isinstance(getattr(state, k, None), torch.Tensor)}


def _restore(state, snap):
    for k, v in snap.items():
        getattr(state, k).copy_(v)


def _optimize_graph(state, model, fmax, max_steps, fire_flavor, include_cell_forces, active,
                    n_active, graph_steps, step_kwargs):
    """The relax loop as CUDA-graph replays of ``graph_steps`` (FIRE step +
    device convergence mask) each; the host reads the number of active systems
    once per replay.  Needs a model whose calls read nothing back to the host
    (a VerletListModel in graph-safe mode, or a per-call PairTableModel)."""
    from .models.verlet import VerletListModel

    vl = model if isinstance(model, VerletListModel) else None
    if vl is not None:
        vl.set_graph_safe(True)
    dev = state.device

    def body():
        for _ in range(graph_steps):
            fire_step(state, model, fire_flavor=fire_flavor, active=active, **step_kwargs)
            converged_mask(state, fmax, include_cell_forces, active, n_active)

    steps = 0
    try:
        while steps < max_steps:
            # warm-up pass outside capture (workspaces, cached sizes), undone after
            snap = _snapshot(state)
            act0 = active.clone()
            s = torch.cuda.Stream(dev)
            s.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(s):
                fire_step(state, model, fire_flavor=fire_flavor, active=active, **step_kwargs)
                converged_mask(state, fmax, include_cell_forces, active, n_active)
            torch.cuda.current_stream(dev).wait_stream(s)
            torch.cuda.synchronize(dev)
            _restore(state, snap)
            active.copy_(act0)
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g):
                body()
            regrow = False
            while steps < max_steps:
                snap = _snapshot(state)
                act0 = active.clone()
                g.replay()
                over = vl.check_overflow() if vl is not None else 0
                if over:
                    # a list overflowed inside the replay: undo it, grow, recapture
                    _restore(state, snap)
                    active.copy_(act0)
                    vl.grow(over, state)
                    regrow = True
                    break
                steps += graph_steps
                if int(n_active.item()) == 0:
                    return steps
            del g
            if not regrow:
                break
    finally:
        if vl is not None:
            vl.set_graph_safe(False)
    return steps


def optimize(state, model, *, fmax=1e-3, max_steps=10000, cell_filter="frechet",
             fire_flavor=ASE, include_cell_forces=None, check_every=20, init_kwargs=None,
             graph_steps=0, **step_kwargs):
    """Relax every system of the batch to max|F| < fmax with FIRE.

    Converged systems are frozen on the device after every step; the host reads
    the number of still-active systems every ``check_every`` steps to stop.
    With ``graph_steps`` > 0 the loop runs as replays of one CUDA graph of
    ``graph_steps`` steps (FIRE step, device-decided Verlet-list rebuilds,
    convergence mask), read back once per replay; the step count is then a
    multiple of graph_steps, and converged systems stay frozen inside a replay.
    Returns ``(state, steps, converged)``; ``converged`` is a bool [S] tensor.
    """
    if include_cell_forces is None:
        include_cell_forces = cell_filter is not None
    if not isinstance(state, FireState):
        state = fire_init(state, model, fire_flavor=fire_flavor, cell_filter=cell_filter,
                          **(init_kwargs or {}))
    n_sys = state.n_systems
    active = torch.ones(n_sys, dtype=torch.uint8, device=state.device)
    n_active = torch.zeros(1, dtype=torch.int32, device=state.device)
    steps = 0
    converged_mask(state, fmax, include_cell_forces, active, n_active)
    if graph_steps > 0:
        _contiguous(state)
        steps = _optimize_graph(state, model, fmax, max_steps, fire_flavor, include_cell_forces,
                                active, n_active, int(graph_steps), step_kwargs)
        return state, steps, active == 0
    while steps < max_steps:
        fire_step(state, model, fire_flavor=fire_flavor, active=active, **step_kwargs)
        converged_mask(state, fmax, include_cell_forces, active, n_active)
        steps += 1
        if steps % check_every == 0 and int(n_active.item()) == 0:
            break
    return state, steps, active == 0
