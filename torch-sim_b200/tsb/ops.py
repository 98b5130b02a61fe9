"""The C ABI as PyTorch operators (``torch.ops.tsb.*``).

Every kernel entry that the drop-ins call per step is registered as an operator
of the ``tsb`` library with a CUDA implementation (the C-ABI call on the
current stream) and a fake implementation (shapes and dtypes only), so that

* the dispatcher sees each call, with its mutated arguments declared in the
  schema (``Tensor(a!)``), and orders it on the current CUDA stream;
* ``torch.compile`` can trace through the drop-ins (fake kernels give the
  output metadata; the neighbour list's pair count is a data-dependent size);
* a per-call step loop (``nvt_langevin_step`` and friends) can be captured in
  a CUDA graph: no operator below reads the device from the host, and the
  Langevin noise counter can live on the device (``counter_dev``).

There is no CPU kernel: calling an operator with CPU tensors raises
``NotImplementedError`` from the dispatcher.

The operators replace the tensor-level calls behind the reference's plugin
interface: torch_sim/neighbors/__init__.py:46-98 (neighbour list),
torch_sim/models/interface.py:71-201 and pair_potential.py:351-464 (model
forward), torch_sim/integrators/md.py:169-208, nvt.py:27-86, 144-240,
nve.py:74-130 (MD step pieces), torch_sim/optimizers/fire.py:288-499 and
cell_filters.py:353-399 (FIRE and the Frechet cell filter), called from
torch_sim/runners.py:308-320, 387-393, 630-643, 714.
"""

from __future__ import annotations

import torch

from . import _lib as L

_LIB = torch.library.Library("tsb", "DEF")
_P = L.ptr


def _u64(v: int) -> int:
    """Signed int64 (operator schema) -> the uint64 the C ABI takes."""
    return int(v) & (2**64 - 1)


def _i64(v: int) -> int:
    """uint64 -> signed int64 for an operator argument."""
    v = int(v) & (2**64 - 1)
    return v - 2**64 if v >= 2**63 else v


def _define(schema: str, cuda_impl, fake_impl) -> None:
    name = schema.split("(", 1)[0]
    _LIB.define(schema)
    _LIB.impl(name, cuda_impl, "CUDA")
    torch.library.register_fake(f"tsb::{name}", fake_impl, lib=_LIB)


def _stream(t: torch.Tensor) -> int:
    return L.stream_ptr(t.device)


# ---------------------------------------------------------------- neighbour list
def _nl_build(positions, cell_row, pbc, system_idx, cutoff, flags, n_systems, capacity):
    n = positions.shape[0]
    dev, dt = positions.device, positions.dtype
    ws = L.Workspace.get(dev, L.load().tsb_nl_workspace_size(n, n_systems))
    n_pairs = torch.zeros(1, dtype=torch.int64, device=dev)
    cap = int(capacity)
    for _ in range(2):
        mapping = torch.empty((2, max(cap, 1)), dtype=torch.int64, device=dev)
        sysmap = torch.empty(max(cap, 1), dtype=torch.int64, device=dev)
        shifts = torch.empty((max(cap, 1), 3), dtype=dt, device=dev)
        L.call("tsb_nl_build", _P(positions), _P(cell_row), _P(pbc), _P(system_idx), n,
               n_systems, L.dtype_code(dt), float(cutoff), int(flags), _P(mapping),
               mapping.shape[1], _P(sysmap), _P(shifts), cap, _P(n_pairs), _P(ws), ws.numel(),
               _stream(positions))
        p = int(n_pairs.item())
        if p <= cap:
            break
        cap = int(p * 1.15) + 16
    return mapping[:, :p].contiguous(), sysmap[:p].contiguous(), shifts[:p].contiguous()


def _nl_build_fake(positions, cell_row, pbc, system_idx, cutoff, flags, n_systems, capacity):
    p = torch.library.get_ctx().new_dynamic_size()
    dev, dt = positions.device, positions.dtype
    return (positions.new_empty((2, p), dtype=torch.int64),
            positions.new_empty((p,), dtype=torch.int64),
            torch.empty((p, 3), dtype=dt, device=dev))


_define("nl_build(Tensor positions, Tensor cell_row, Tensor pbc, Tensor system_idx, "
        "float cutoff, int flags, int n_systems, int capacity) -> (Tensor, Tensor, Tensor)",
        _nl_build, _nl_build_fake)


# ---------------------------------------------------------------- pair model
def _pair_flags(flags):
    return (bool(flags & L.OUT_FORCES), bool(flags & L.OUT_STRESS),
            bool(flags & L.OUT_ENERGIES), bool(flags & L.OUT_STRESSES))


def _pair_outputs(positions, n_systems, flags):
    dev, dt = positions.device, positions.dtype
    n = positions.shape[0]
    f, s, e, ss = _pair_flags(flags)
    return (torch.empty(n_systems, dtype=dt, device=dev),
            torch.empty((n, 3) if f else (0, 3), dtype=dt, device=dev),
            torch.empty((n_systems, 3, 3) if s else (0, 3, 3), dtype=dt, device=dev),
            torch.empty(n if e else 0, dtype=dt, device=dev),
            torch.empty((n, 3, 3) if ss else (0, 3, 3), dtype=dt, device=dev))


def _pair_call(positions, cell_row, pbc, system_idx, species, table, kind, n_species, cutoff,
               flags, n_systems, max_system_atoms, energy, forces, stress, energies, stresses,
               sys_active):
    n = positions.shape[0]
    ws = L.Workspace.get(positions.device, L.load().tsb_pair_workspace_size(n, n_systems))
    nz = lambda t: _P(t) if (t is not None and t.numel()) else None  # noqa: E731
    L.call("tsb_pair_forward", int(kind), _P(table), int(n_species), _P(species),
           _P(positions), _P(cell_row), _P(pbc), _P(system_idx), n, n_systems,
           L.dtype_code(positions.dtype), float(cutoff), int(flags), _P(energy), nz(forces),
           nz(stress), nz(energies), nz(stresses), _P(sys_active), int(max_system_atoms),
           _P(ws), ws.numel(), _stream(positions))


def _pair_forward(positions, cell_row, pbc, system_idx, species, table, kind, n_species,
                  cutoff, flags, n_systems, max_system_atoms):
    out = _pair_outputs(positions, n_systems, flags)
    _pair_call(positions, cell_row, pbc, system_idx, species, table, kind, n_species, cutoff,
               flags, n_systems, max_system_atoms, *out, None)
    return out


def _pair_forward_fake(positions, cell_row, pbc, system_idx, species, table, kind, n_species,
                       cutoff, flags, n_systems, max_system_atoms):
    return _pair_outputs(positions, n_systems, flags)


_define("pair_forward(Tensor positions, Tensor cell_row, Tensor pbc, Tensor system_idx, "
        "Tensor? species, Tensor table, int kind, int n_species, float cutoff, int flags, "
        "int n_systems, int max_system_atoms) -> (Tensor, Tensor, Tensor, Tensor, Tensor)",
        _pair_forward, _pair_forward_fake)


def _pair_forward_into(positions, cell_row, pbc, system_idx, species, table, kind, n_species,
                       cutoff, flags, n_systems, max_system_atoms, energy, forces, stress,
                       sys_active):
    _pair_call(positions, cell_row, pbc, system_idx, species, table, kind, n_species, cutoff,
               flags, n_systems, max_system_atoms, energy, forces, stress, None, None,
               sys_active)


def _noop(*_a):
    return None


_define("pair_forward_into_(Tensor positions, Tensor cell_row, Tensor pbc, Tensor system_idx, "
        "Tensor? species, Tensor table, int kind, int n_species, float cutoff, int flags, "
        "int n_systems, int max_system_atoms, Tensor(a!) energy, Tensor(b!)? forces, "
        "Tensor(c!)? stress, Tensor? sys_active) -> ()", _pair_forward_into, _noop)


# ---------------------------------------------------------------- MD step pieces
def _md_kick(momenta, forces, system_idx, dt, scale):
    L.call("tsb_md_kick", _P(momenta), _P(forces), _P(system_idx), _P(dt), float(scale),
           momenta.shape[0], L.dtype_code(momenta.dtype), _stream(momenta))


_define("md_kick_(Tensor(a!) momenta, Tensor forces, Tensor system_idx, Tensor dt, "
        "float scale) -> ()", _md_kick, _noop)


def _md_drift(positions, momenta, masses, system_idx, dt, scale):
    L.call("tsb_md_drift", _P(positions), _P(momenta), _P(masses), _P(system_idx), _P(dt),
           float(scale), positions.shape[0], L.dtype_code(positions.dtype), _stream(positions))


_define("md_drift_(Tensor(a!) positions, Tensor momenta, Tensor masses, Tensor system_idx, "
        "Tensor dt, float scale) -> ()", _md_drift, _noop)


def _md_baoab_boa(positions, momenta, forces, masses, system_idx, dt, kT, gamma, noise, seed,
                  counter, counter_dev):
    L.call("tsb_md_baoab_boa", _P(positions), _P(momenta), _P(forces), _P(masses),
           _P(system_idx), _P(dt), _P(kT), _P(gamma), _P(noise), _u64(seed), _u64(counter),
           _P(counter_dev), positions.shape[0], L.dtype_code(positions.dtype),
           _stream(positions))


_define("md_baoab_boa_(Tensor(a!) positions, Tensor(b!) momenta, Tensor forces, Tensor masses, "
        "Tensor system_idx, Tensor dt, Tensor kT, Tensor gamma, Tensor? noise, int seed, "
        "int counter, Tensor(c!)? counter_dev) -> ()", _md_baoab_boa, _noop)


# ---------------------------------------------------------------- fused MD
def _fused_md(integrator, kind, table, n_species, species, positions, momenta, forces, masses,
              cell_row, system_idx, order, cutoff, skin, n_steps, dt, kT, gamma, tau, chain_xi,
              chain_pxi, chain_q, chain_ke, chain_dt, chain_length, chain_steps, sy_steps, seed,
              counter, counter_dev, frame_x, frame_e, report_every, lanes_max, n_wide,
              prune_skin, energy, stress, n_rebuilds, status, workspace):
    n_frames = frame_x.shape[0] if frame_x is not None else 0
    L.call("tsb_fused_md_ex", int(integrator), int(kind), _P(table), int(n_species),
           _P(species), _P(positions), _P(momenta), _P(forces), _P(masses), _P(cell_row),
           _P(system_idx), positions.shape[0], energy.shape[0], _P(order), float(cutoff),
           float(skin), int(n_steps), _P(dt), _P(kT), _P(gamma), _P(tau), _P(chain_xi),
           _P(chain_pxi), _P(chain_q), _P(chain_ke), _P(chain_dt), int(chain_length),
           int(chain_steps), int(sy_steps), _u64(seed), _u64(counter), _P(counter_dev),
           _P(frame_x), _P(frame_e), int(report_every), int(n_frames), int(lanes_max),
           int(n_wide), float(prune_skin), _P(energy), _P(stress),
           _P(n_rebuilds), _P(status), _P(workspace), workspace.numel(), _stream(positions))


_define("fused_md_(int integrator, int kind, Tensor table, int n_species, Tensor? species, "
        "Tensor(a!) positions, Tensor(b!) momenta, Tensor(c!) forces, Tensor masses, "
        "Tensor cell_row, Tensor system_idx, Tensor? order, float cutoff, float skin, "
        "int n_steps, Tensor dt, Tensor? kT, Tensor? gamma, Tensor? tau, "
        "Tensor(d!)? chain_xi, Tensor(e!)? chain_pxi, Tensor(f!)? chain_q, "
        "Tensor(g!)? chain_ke, Tensor? chain_dt, int chain_length, int chain_steps, "
        "int sy_steps, int seed, int counter, Tensor(h!)? counter_dev, Tensor(i!)? frame_x, "
        "Tensor(j!)? frame_e, int report_every, int lanes_max, int n_wide, "
        "float prune_skin, Tensor(k!) energy, "
        "Tensor(l!)? stress, "
        "Tensor(m!)? n_rebuilds, Tensor(n!) status, Tensor(o!) workspace) -> ()",
        _fused_md, _noop)


# ---------------------------------------------------------------- FIRE
def _fire(name):
    def impl(is_cell, positions, velocities, forces, masses, system_idx, dt, alpha, n_pos, cell,
             reference_cell, cell_factor, cell_positions, cell_velocities, cell_forces,
             cell_masses, sys_active, dt_max, n_min, f_inc, f_dec, alpha_start, f_alpha,
             max_step, eps):
        n_sys = dt.shape[0]
        ws = L.Workspace.get(positions.device, L.load().tsb_fire_workspace_size(n_sys))
        L.call(name, int(is_cell), _P(positions), _P(velocities), _P(forces), _P(masses),
               _P(system_idx), positions.shape[0], n_sys, _P(dt), _P(alpha), _P(n_pos),
               _P(cell), _P(reference_cell), _P(cell_factor), _P(cell_positions),
               _P(cell_velocities), _P(cell_forces), _P(cell_masses), _P(sys_active),
               float(dt_max), int(n_min), float(f_inc), float(f_dec), float(alpha_start),
               float(f_alpha), float(max_step), float(eps), L.dtype_code(positions.dtype),
               _P(ws), ws.numel(), _stream(positions))
    return impl


_FIRE_SCHEMA = ("(int is_cell, Tensor(a!) positions, Tensor(b!) velocities, Tensor forces, "
                "Tensor masses, Tensor system_idx, Tensor(c!) dt, Tensor(d!) alpha, "
                "Tensor(e!) n_pos, Tensor(f!)? cell, Tensor? reference_cell, "
                "Tensor? cell_factor, Tensor(g!)? cell_positions, Tensor(h!)? cell_velocities, "
                "Tensor? cell_forces, Tensor? cell_masses, Tensor? sys_active, float dt_max, "
                "int n_min, float f_inc, float f_dec, float alpha_start, float f_alpha, "
                "float max_step, float eps) -> ()")
for _name in ("fire_ase_pre_", "fire_vv_pre_", "fire_vv_post_"):
    _define(_name + _FIRE_SCHEMA, _fire("tsb_" + _name.rstrip("_")), _noop)


def _frechet_cell_forces(cell_forces, stress, cell, reference_cell, pressure, cell_factor,
                         init, sys_active):
    L.call("tsb_frechet_cell_forces", _P(cell_forces), _P(stress), _P(cell),
           _P(reference_cell), _P(pressure), _P(cell_factor), cell.shape[0], int(init),
           _P(sys_active), L.dtype_code(cell.dtype), _stream(cell))


_define("frechet_cell_forces_(Tensor(a!) cell_forces, Tensor stress, Tensor cell, "
        "Tensor reference_cell, Tensor pressure, Tensor cell_factor, int init, "
        "Tensor? sys_active) -> ()", _frechet_cell_forces, _noop)


def _fire_converged(forces, system_idx, n_systems, cell_forces, fmax, active, n_active):
    ws = L.Workspace.get(forces.device, L.load().tsb_fire_workspace_size(n_systems))
    L.call("tsb_fire_converged", _P(forces), _P(system_idx), forces.shape[0], int(n_systems),
           _P(cell_forces), float(fmax), _P(active), _P(n_active), L.dtype_code(forces.dtype),
           _P(ws), ws.numel(), _stream(forces))


_define("fire_converged_(Tensor forces, Tensor system_idx, int n_systems, Tensor? cell_forces, "
        "float fmax, Tensor(a!) active, Tensor(b!) n_active) -> ()", _fire_converged, _noop)


# ---------------------------------------------------------------- Verlet lists
def _vlist_check(positions, cell_row, system_idx, sys_active, n_systems, cutoff, skin, prune,
                 flags, workspace):
    L.call("tsb_vlist_check", _P(positions), _P(cell_row), _P(system_idx), _P(sys_active),
           positions.shape[0], int(n_systems), L.dtype_code(positions.dtype), float(cutoff),
           float(skin), float(prune), _P(flags), _P(workspace), workspace.numel(),
           _stream(positions))


_define("vlist_check_(Tensor positions, Tensor cell_row, Tensor system_idx, Tensor? sys_active, "
        "int n_systems, float cutoff, float skin, float prune, Tensor(a!) flags, "
        "Tensor(b!) workspace) -> ()", _vlist_check, _noop)


def _vlist_build(positions, cell_row, pbc, system_idx, species, n_systems, cutoff, skin, lst,
                 counts, max_neighbors, max_system_atoms, flags, workspace):
    L.call("tsb_vlist_build", _P(positions), _P(cell_row), _P(pbc), _P(system_idx),
           _P(species), positions.shape[0], int(n_systems), L.dtype_code(positions.dtype),
           float(cutoff), float(skin), _P(lst), _P(counts), int(max_neighbors),
           int(max_system_atoms), _P(flags), _P(workspace), workspace.numel(),
           _stream(positions))


_define("vlist_build_(Tensor positions, Tensor cell_row, Tensor pbc, Tensor system_idx, "
        "Tensor? species, int n_systems, float cutoff, float skin, Tensor(a!) nlist, "
        "Tensor(b!) counts, int max_neighbors, int max_system_atoms, Tensor(c!) flags, "
        "Tensor(d!) workspace) -> ()", _vlist_build, _noop)


def _vlist_forces(kind, table, n_species, species, lst, counts, positions, cell_row,
                  system_idx, sys_active, n_systems, cutoff, prune, flags, energy, forces,
                  stress, energies, stresses, workspace):
    nz = lambda t: _P(t) if (t is not None and t.numel()) else None  # noqa: E731
    L.call("tsb_vlist_forces", int(kind), _P(table), int(n_species), _P(species), _P(lst),
           _P(counts), _P(positions), _P(cell_row), _P(system_idx), _P(sys_active),
           positions.shape[0], int(n_systems), L.dtype_code(positions.dtype), float(cutoff),
           float(prune), int(flags), _P(energy), nz(forces), nz(stress), nz(energies),
           nz(stresses), _P(workspace), workspace.numel(), _stream(positions))


# with prune > 0 the lists are reordered in place (front parts), so nlist is written
_define("vlist_forces_(int kind, Tensor table, int n_species, Tensor? species, "
        "Tensor(g!) nlist, Tensor counts, Tensor positions, Tensor cell_row, "
        "Tensor system_idx, Tensor? sys_active, int n_systems, float cutoff, float prune, "
        "int flags, Tensor(a!) energy, Tensor(b!)? forces, Tensor(c!)? stress, "
        "Tensor(d!)? energies, Tensor(e!)? stresses, Tensor(f!) workspace) -> ()",
        _vlist_forces, _noop)


OPS = ("nl_build", "pair_forward", "pair_forward_into_", "md_kick_", "md_drift_",
       "md_baoab_boa_", "fused_md_", "fire_ase_pre_", "fire_vv_pre_", "fire_vv_post_",
       "frechet_cell_forces_", "fire_converged_", "vlist_check_", "vlist_build_",
       "vlist_forces_")
