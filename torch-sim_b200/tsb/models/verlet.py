"""Verlet-list model wrapper for large periodic systems.

``VerletListModel(model, skin=1.0)`` keeps the neighbour list (cutoff + skin) of
one large fully periodic system between calls and rebuilds it only when an atom
moved more than skin/2 (C ABI: tsb_verlet_build / tsb_verlet_check /
tsb_verlet_forces).  The reference rebuilds its list in every call
(torch_sim/models/pair_potential.py:168-174); the pairs within the cutoff, and
therefore energy, forces and stress, are the same.
"""

from __future__ import annotations

import torch

from .. import _lib as L
from .interface import ModelInterface
from .pair_potential import PairTableModel


class VerletListModel(ModelInterface):
    def __init__(self, model: PairTableModel, *, skin: float = 1.0, max_neighbors: int = 0):
        super().__init__()
        if not isinstance(model, PairTableModel):
            raise TypeError("VerletListModel wraps a tsb PairTableModel")
        self.model = model
        self._device, self._dtype = model.device, model.dtype
        self._compute_forces, self._compute_stress = True, model.compute_stress
        self.skin = float(skin)
        self.max_neighbors = int(max_neighbors)
        self.n_builds = 0
        self._key = None

    def _ensure(self, state):
        n = state.n_atoms
        key = (n, state.positions.dtype, state.positions.device)
        if self._key != key:
            dev = state.device
            rcs = self.model.cutoff + self.skin
            vol = float(torch.det(state.cell[0].double()).abs())
            est = int(4.2 * rcs ** 3 * n / vol * 1.35) + 16
            self.cap = max(self.max_neighbors, est)
            self.list = torch.empty(self.cap * n, dtype=torch.int32, device=dev)
            self.counts = torch.empty(n, dtype=torch.int32, device=dev)
            self.ref = torch.empty((n, 3), dtype=torch.float64, device=dev)
            self.wraps = torch.empty((n, 3), dtype=torch.int32, device=dev)
            self.status = torch.zeros(1, dtype=torch.int32, device=dev)
            self.expired = torch.zeros(1, dtype=torch.int32, device=dev)
            self.e_atom = torch.empty(n, dtype=torch.float64, device=dev)
            self.vir_atom = torch.empty((n, 6), dtype=torch.float64, device=dev)
            self.ws = torch.empty(L.load().tsb_verlet_workspace_size(n), dtype=torch.uint8,
                                  device=dev)
            self._key = key
            self._built = False

    def _check(self, state, pos, cell64):
        L.call("tsb_verlet_check", L.ptr(pos), L.ptr(self.ref), L.ptr(self.wraps),
               L.ptr(cell64), L.ptr(self.model._species(state.atomic_numbers)), state.n_atoms,
               L.dtype_code(pos.dtype), self.skin, L.ptr(self.expired), L.ptr(self.ws),
               self.ws.numel(), L.stream_ptr(state.device))

    def _build(self, state, pos):
        cell = state.cell[0].mT.to(pos.dtype).contiguous()
        while True:
            L.call("tsb_verlet_build", L.ptr(pos), L.ptr(cell), state.n_atoms,
                   L.dtype_code(pos.dtype), self.model.cutoff, self.skin, L.ptr(self.list),
                   L.ptr(self.counts), self.cap, L.ptr(self.ref), L.ptr(self.wraps),
                   L.ptr(self.status), L.ptr(self.ws), self.ws.numel(),
                   L.stream_ptr(state.device))
            st = int(self.status.item())
            if st == 0:
                break
            if st >= (1 << 30):
                raise ValueError("VerletListModel needs every cell width >= cutoff + skin")
            self.cap = int(st * 1.2) + 8
            self.list = torch.empty(self.cap * state.n_atoms, dtype=torch.int32,
                                    device=state.device)
        self.n_builds += 1
        self._built = True

    def forward(self, state, **_kw):
        if state.n_systems != 1:
            raise ValueError("VerletListModel handles one large system")
        if not bool(torch.as_tensor(state.pbc).all()):
            raise ValueError("VerletListModel needs periodic boundaries on all axes")
        if state.dtype != self._dtype:
            raise TypeError(f"SimState dtype {state.dtype} does not match model dtype "
                            f"{self._dtype}.")
        self._ensure(state)
        pos = state.positions.contiguous()
        cell64 = state.cell[0].mT.double().contiguous()
        if not self._built:
            self._build(state, pos)
            self._check(state, pos, cell64)
        else:
            self._check(state, pos, cell64)
            if int(self.expired.item()):
                self._build(state, pos)
                self._check(state, pos, cell64)
        dt = pos.dtype
        energy = torch.empty(1, dtype=dt, device=state.device)
        forces = torch.empty_like(pos)
        stress = (torch.empty((1, 3, 3), dtype=dt, device=state.device)
                  if self._compute_stress else None)
        flags = L.OUT_FORCES | (L.OUT_STRESS if stress is not None else 0)
        table = self.model.table
        L.call("tsb_verlet_forces", self.model.kind, L.ptr(table), self.model.n_species,
               L.ptr(self.list), L.ptr(self.counts), state.n_atoms, L.ptr(cell64),
               L.dtype_code(dt), self.model.cutoff, flags, L.ptr(energy), L.ptr(forces),
               L.ptr(stress), L.ptr(self.e_atom), L.ptr(self.vir_atom), L.ptr(self.ws),
               self.ws.numel(), L.stream_ptr(state.device))
        out = {"energy": energy, "forces": forces}
        if stress is not None:
            out["stress"] = stress
        return out
