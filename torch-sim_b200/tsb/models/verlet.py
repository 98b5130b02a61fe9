"""Verlet-list model wrapper: neighbour lists kept between calls.

``VerletListModel(model, skin=1.0)`` wraps a tsb ``PairTableModel`` (LJ, Morse,
soft sphere).  Each system's list holds every pair within cutoff + skin and is
rebuilt, per system, only when its atoms' drift and its cell's deformation since
the build could have brought a pair from beyond cutoff + skin to inside the
cutoff (C ABI: tsb_vlist_check / tsb_vlist_build / tsb_vlist_forces).  The
reference rebuilds its list in every call (torch_sim/models/pair_potential.py:
168-174); the pairs inside the cutoff, and therefore energy, forces and stress,
are the same.  Works for one large system (500,000 atoms) and for batches of
small ones whose atoms and cells move (FIRE with a cell filter, NPT, MD).

Every periodic cell must be at least cutoff + skin wide (image shifts in
{-1,0,1}^3); narrower cells raise ValueError.  The wrapper keeps its own device
workspace (the list frame) and reads two flags from the device per call.

One fully periodic system with FP32 pair arithmetic and no per-atom outputs (the
500,000-atom workload) takes the single-system kernels (tsb_verlet_build /
tsb_verlet_check / tsb_verlet_forces: atom order, per-block sums fused into the
force kernel), about 10 % faster there; its list expires when an atom moved more
than skin/2 or the cell changed.
"""

from __future__ import annotations

import torch

from .. import _lib as L
from .. import ops as _ops  # noqa: F401  (registers torch.ops.tsb.*)
from .interface import ModelInterface
from .pair_potential import PairTableModel


class VerletListModel(ModelInterface):
    def __init__(self, model: PairTableModel, *, skin: float = 1.0, max_neighbors: int = 0,
                 prune: float | None = None):
        """``prune`` (Angstrom, batched lists only): between rebuilds each atom
        evaluates only the list entries that were within its pair cutoff +
        ``prune`` at the system's last pruning; a system is pruned again when its
        atoms' drift or its cell's deformation could bring a left-out pair inside
        the cutoff.  Results equal those of the whole list to FP64 rounding.
        Default 0 (off): on the FIRE + Frechet relax workload the non-affine
        steps use up the drift allowance within a few steps and the re-prunings
        cost more than the shorter lists save (0.54 against 0.47 ms per step
        with 0.2 to 0.45 A)."""
        super().__init__()
        if not isinstance(model, PairTableModel):
            raise TypeError("VerletListModel wraps a tsb PairTableModel")
        if model.kind not in (L.POT_LJ, L.POT_MORSE, L.POT_SOFT):
            raise TypeError("VerletListModel supports LJ, Morse and soft-sphere tables")
        self.model = model
        self._device, self._dtype = model.device, model.dtype
        self._compute_forces, self._compute_stress = True, model.compute_stress
        self.per_atom_energies = getattr(model, "per_atom_energies", False)
        self.per_atom_stresses = getattr(model, "per_atom_stresses", False)
        self.skin = float(skin)
        self.prune = 0.0 if prune is None else float(prune)
        if not (0.0 <= self.prune):
            raise ValueError("prune must be >= 0")
        if self.prune >= self.skin:
            self.prune = 0.0  # the whole list is within cutoff + skin anyway
        self.max_neighbors = int(max_neighbors)
        self.n_builds = 0
        self._key = None
        self._last_single = False
        # graph-safe mode: the rebuild is decided on the device (no host reads),
        # list overflow is recorded in a sticky device flag (see set_graph_safe)
        self.graph_safe = False
        self.sticky = None

    # -------------------------------------------------------------- buffers
    def _ensure(self, state, pos, cell_row):
        n, ns = state.n_atoms, state.n_systems
        sysi, z = state.system_idx, state.atomic_numbers
        key = (n, ns, pos.dtype, pos.device, sysi.data_ptr(), sysi._version, z.data_ptr(),
               z._version)
        if self._key == key:
            return
        dev = pos.device
        rcs = self.model.cutoff + self.skin
        counts = torch.bincount(sysi, minlength=ns).double()
        self.max_system_atoms = int(counts.max()) if ns else 0
        vol = torch.linalg.det(cell_row.double()).abs().clamp_min(1e-30)
        dens = float((counts / vol).max())
        est = int(4.19 * rcs ** 3 * dens * 1.35) + 16
        if not (est < 4096):
            est = 4096
        self.cap = max(self.max_neighbors, est)
        self.list = torch.empty(self.cap * n, dtype=torch.int32, device=dev)
        self.counts = torch.empty(n, dtype=torch.int32, device=dev)
        self.flags = torch.zeros(2, dtype=torch.int32, device=dev)
        self.ws = torch.empty(L.load().tsb_vlist_workspace_size(n, ns), dtype=torch.uint8,
                              device=dev)
        self._reset(n, ns, dev)
        self._key = key

    def _reset(self, n, ns, dev):
        L.call("tsb_vlist_reset", n, ns, L.ptr(self.ws), self.ws.numel(), L.stream_ptr(dev))

    def set_graph_safe(self, on: bool = True) -> None:
        """Graph-safe mode for CUDA-graph capture of step loops: every call checks
        the lists and launches the rebuild unconditionally (the rebuild kernels
        only touch the systems the check marked as expired), and nothing is read
        back to the host.  A list that overflows or a cell narrower than cutoff +
        skin is recorded in ``self.sticky`` (device int32 [1], maximum over
        calls); ``check_overflow()`` reads it after a replay."""
        self.graph_safe = bool(on)

    def check_overflow(self) -> int:
        """0, or the neighbour count that overflowed the lists since the last
        reset (1 << 30 for a cell narrower than cutoff + skin)."""
        return 0 if self.sticky is None else int(self.sticky.item())

    def grow(self, needed: int, state) -> None:
        """Regrow the lists to hold ``needed`` neighbours per atom and mark every
        system for a rebuild (after an overflow seen by check_overflow)."""
        if needed >= (1 << 30):
            raise ValueError("VerletListModel needs every periodic cell width >= cutoff + skin")
        dev = state.positions.device
        self.cap = int(needed * 1.2) + 8
        self.list = torch.empty(self.cap * state.n_atoms, dtype=torch.int32, device=dev)
        self._reset(state.n_atoms, state.n_systems, dev)
        if self.sticky is not None:
            self.sticky.zero_()

    # ---------------------------------------------------------------- lists
    def _update_lists(self, state, pos, cell_row, pbc, sysi, species, active):
        n, ns, dev = state.n_atoms, state.n_systems, pos.device
        cutoff = self.model.cutoff
        if self.graph_safe:
            if self.sticky is None or self.sticky.device != dev:
                self.sticky = torch.zeros(1, dtype=torch.int32, device=dev)
            torch.ops.tsb.vlist_check_(pos, cell_row, sysi, active, ns, cutoff, self.skin,
                                       self.prune, self.flags, self.ws)
            torch.ops.tsb.vlist_build_(pos, cell_row, pbc, sysi, species, ns, cutoff, self.skin,
                                       self.list, self.counts, self.cap, self.max_system_atoms,
                                       self.flags, self.ws)
            torch.maximum(self.sticky, self.flags[1:], out=self.sticky)
            return
        while True:
            torch.ops.tsb.vlist_check_(pos, cell_row, sysi, active, ns, cutoff, self.skin,
                                       self.prune, self.flags, self.ws)
            if not int(self.flags[0].item()):
                return
            torch.ops.tsb.vlist_build_(pos, cell_row, pbc, sysi, species, ns, cutoff, self.skin,
                                       self.list, self.counts, self.cap, self.max_system_atoms,
                                       self.flags, self.ws)
            self.n_builds += 1
            st = int(self.flags[1].item())
            if st == 0:
                return
            if st >= (1 << 30):
                raise ValueError("VerletListModel needs every periodic cell width >= "
                                 "cutoff + skin")
            # a list overflowed: regrow and rebuild every system
            self.cap = int(st * 1.2) + 8
            self.list = torch.empty(self.cap * n, dtype=torch.int32, device=dev)
            self._reset(n, ns, dev)

    def _run(self, state, energy, forces, stress, energies, stresses, active):
        if state.dtype != self._dtype:
            raise TypeError(f"SimState dtype {state.dtype} does not match model dtype "
                            f"{self._dtype}.")
        pos = state.positions.contiguous()
        L.require_cuda(pos, "state.positions")
        n_sys = state.n_systems
        cell_row = state.cell.mT.contiguous()
        pbc = L.pbc_rows(state.pbc, n_sys, pos.device)
        sysi = state.system_idx.contiguous()
        species = self.model._species(state.atomic_numbers)
        self._ensure(state, pos, cell_row)
        self._update_lists(state, pos, cell_row, pbc, sysi, species, active)
        m = self.model
        table = m.table if m.table.device == pos.device else m.table.to(pos.device)
        flags = 0
        if forces is not None:
            flags |= L.OUT_FORCES
        if stress is not None:
            flags |= L.OUT_STRESS
        if energies is not None:
            flags |= L.OUT_ENERGIES
        if stresses is not None:
            flags |= L.OUT_STRESSES
        if m.precision == "fp64":
            flags |= L.MATH_FP64
        torch.ops.tsb.vlist_forces_(m.kind, table, m.n_species, species, self.list, self.counts,
                                    pos, cell_row, sysi, active, n_sys, m.cutoff, self.prune,
                                    flags, energy, forces, stress, energies, stresses, self.ws)

    # ------------------------------------------------- one large system
    def _single_ok(self, state):
        if (state.n_systems != 1 or self.model.precision == "fp64" or self.per_atom_energies
                or self.per_atom_stresses):
            return False
        pbc = state.pbc
        key = (pbc.data_ptr(), pbc._version) if isinstance(pbc, torch.Tensor) else bool(pbc)
        if getattr(self, "_pbc_key", None) != key:  # one device read per pbc tensor
            self._pbc_key = key
            self._pbc_all = bool(L.pbc_rows(pbc, 1, state.positions.device).all())
        return self._pbc_all

    def _s_ensure(self, state):
        n = state.n_atoms
        key = (n, state.positions.dtype, state.positions.device)
        if getattr(self, "_s_key", None) == key:
            return
        dev = state.device
        rcs = self.model.cutoff + self.skin
        vol = float(torch.det(state.cell[0].double()).abs())
        est = int(4.2 * rcs ** 3 * n / vol * 1.35) + 16
        self.s_cap = max(self.max_neighbors, est)
        self.s_list = torch.empty(self.s_cap * n, dtype=torch.int32, device=dev)
        self.s_counts = torch.empty(n, dtype=torch.int32, device=dev)
        self.s_ref = torch.empty((n, 3), dtype=torch.float64, device=dev)
        self.s_wraps = torch.empty((n, 3), dtype=torch.int32, device=dev)
        self.s_status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.s_expired = torch.zeros(1, dtype=torch.int32, device=dev)
        self.s_e_atom = torch.empty(n, dtype=torch.float64, device=dev)
        self.s_vir_atom = torch.empty((n, 6), dtype=torch.float64, device=dev)
        self.s_ws = torch.empty(L.load().tsb_verlet_workspace_size(n), dtype=torch.uint8,
                                device=dev)
        self._s_key = key
        self._s_built = False

    def _s_check(self, state, pos, cell64):
        L.call("tsb_verlet_check", L.ptr(pos), L.ptr(self.s_ref), L.ptr(self.s_wraps),
               L.ptr(cell64), L.ptr(self.model._species(state.atomic_numbers)), state.n_atoms,
               L.dtype_code(pos.dtype), self.skin, L.ptr(self.s_expired), L.ptr(self.s_ws),
               self.s_ws.numel(), L.stream_ptr(state.device))

    def _s_build(self, state, pos):
        cell = state.cell[0].mT.to(pos.dtype).contiguous()
        while True:
            L.call("tsb_verlet_build", L.ptr(pos), L.ptr(cell), state.n_atoms,
                   L.dtype_code(pos.dtype), self.model.cutoff, self.skin, L.ptr(self.s_list),
                   L.ptr(self.s_counts), self.s_cap, L.ptr(self.s_ref), L.ptr(self.s_wraps),
                   L.ptr(self.s_status), L.ptr(self.s_ws), self.s_ws.numel(),
                   L.stream_ptr(state.device))
            st = int(self.s_status.item())
            if st == 0:
                break
            if st >= (1 << 30):
                raise ValueError("VerletListModel needs every periodic cell width >= "
                                 "cutoff + skin")
            self.s_cap = int(st * 1.2) + 8
            self.s_list = torch.empty(self.s_cap * state.n_atoms, dtype=torch.int32,
                                      device=state.device)
        self.n_builds += 1
        self._s_built = True

    def _single_forward(self, state):
        if state.dtype != self._dtype:
            raise TypeError(f"SimState dtype {state.dtype} does not match model dtype "
                            f"{self._dtype}.")
        L.require_cuda(state.positions, "state.positions")
        self._s_ensure(state)
        pos = state.positions.contiguous()
        cell64 = state.cell[0].mT.double().contiguous()
        if not self._s_built:
            self._s_build(state, pos)
            self._s_check(state, pos, cell64)
        else:
            self._s_check(state, pos, cell64)
            if int(self.s_expired.item()):
                self._s_build(state, pos)
                self._s_check(state, pos, cell64)
        dt = pos.dtype
        energy = torch.empty(1, dtype=dt, device=state.device)
        forces = torch.empty_like(pos)
        stress = (torch.empty((1, 3, 3), dtype=dt, device=state.device)
                  if self._compute_stress else None)
        flags = L.OUT_FORCES | (L.OUT_STRESS if stress is not None else 0)
        m = self.model
        L.call("tsb_verlet_forces", m.kind, L.ptr(m.table), m.n_species, L.ptr(self.s_list),
               L.ptr(self.s_counts), state.n_atoms, L.ptr(cell64), L.dtype_code(dt), m.cutoff,
               flags, L.ptr(energy), L.ptr(forces), L.ptr(stress), L.ptr(self.s_e_atom),
               L.ptr(self.s_vir_atom), L.ptr(self.s_ws), self.s_ws.numel(),
               L.stream_ptr(state.device))
        out = {"energy": energy, "forces": forces}
        if stress is not None:
            out["stress"] = stress
        return out

    # ------------------------------------------------------------------ API
    @property
    def list_counts(self) -> torch.Tensor:
        """Neighbour-list entries per atom (slot order on the batched path) of the
        engine used by the last call."""
        return self.s_counts if self._last_single else self.counts

    def forward(self, state, **_kw) -> dict[str, torch.Tensor]:
        self._last_single = self._single_ok(state)
        if self._last_single:
            return self._single_forward(state)
        dev, dt = state.positions.device, state.positions.dtype
        n, n_sys = state.n_atoms, state.n_systems
        energy = torch.empty(n_sys, dtype=dt, device=dev)
        forces = torch.empty((n, 3), dtype=dt, device=dev)
        stress = (torch.empty((n_sys, 3, 3), dtype=dt, device=dev)
                  if self._compute_stress else None)
        energies = torch.empty(n, dtype=dt, device=dev) if self.per_atom_energies else None
        stresses = (torch.empty((n, 3, 3), dtype=dt, device=dev)
                    if self.per_atom_stresses else None)
        self._run(state, energy, forces, stress, energies, stresses, None)
        out = {"energy": energy, "forces": forces}
        if stress is not None:
            out["stress"] = stress
        if energies is not None:
            out["energies"] = energies
        if stresses is not None:
            out["stresses"] = stresses
        return out

    def forward_into(self, state, *, energy, forces, stress=None, sys_active=None):
        """Write energy/forces(/stress) of the systems with ``sys_active`` != 0 into
        existing contiguous buffers; the other systems' entries are left untouched."""
        for t in (energy, forces, stress):
            if t is not None and not t.is_contiguous():
                raise ValueError("forward_into needs contiguous output buffers")
        if sys_active is None and self._single_ok(state):
            # one large system: its own kernels, results copied into the buffers
            self._last_single = True
            out = self._single_forward(state)
            energy.copy_(out["energy"])
            forces.copy_(out["forces"])
            if stress is not None and "stress" in out:
                stress.copy_(out["stress"])
            return
        self._last_single = False
        self._run(state, energy, forces, stress if self._compute_stress else None, None, None,
                  sys_active)
