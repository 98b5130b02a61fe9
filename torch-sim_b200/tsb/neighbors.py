"""Neighbour list drop-in for ``torch_sim.neighbors``.

``torchsim_nl(positions, cell, pbc, cutoff, system_idx, self_interaction=False)``
has the signature and return contract of torch_sim/neighbors/__init__.py:46-98
(and of its default backend torch_nl_linked_cell, torch_nl.py:156-215):

* ``cell`` is the ROW-vector cell, ``[S,3,3]`` or ``[3,3]``; ``pbc`` is ``[S,3]``
  or ``[3]``;
* returns ``mapping [2,P] int64`` (both (i,j) and (j,i)), ``system_mapping [P]
  int64`` and ``shifts_idx [P,3]`` (integers stored in the cell dtype) valid for
  the unwrapped input positions; empty result is ``(2,0), (0,), (0,3)``;
* ``self_interaction=True`` also returns the (i, i, 0) pairs.

The pair set is built on the GPU by ``tsb_nl_build`` (cell binning by counting
sort, cell-list search with explicit periodic images) in one count pass and one
fill pass; pairs are grouped by i in ascending order.
"""

from __future__ import annotations

import torch

from . import _lib as L
from . import ops as _ops  # noqa: F401  (registers torch.ops.tsb.*)


def _normalize(cell: torch.Tensor, pbc: torch.Tensor, n_systems: int):
    """Broadcast to [S,3,3] / [S,3] (torch_sim/neighbors/utils.py:7-34)."""
    if cell.ndim == 2:
        cell = (cell.unsqueeze(0).expand(n_systems, 3, 3) if cell.shape[0] == 3
                else cell.reshape(n_systems, 3, 3))
    pbc = torch.as_tensor(pbc, device=cell.device)
    if pbc.ndim == 0:
        pbc = pbc.reshape(1).expand(3)
    if pbc.ndim == 1:
        pbc = (pbc.unsqueeze(0).expand(n_systems, 3) if pbc.shape[0] == 3
               else pbc.reshape(n_systems, 3))
    return cell.contiguous(), pbc.to(torch.uint8).contiguous()


_capacity_hint: dict = {}


def torchsim_nl(positions: torch.Tensor, cell: torch.Tensor, pbc: torch.Tensor,
                cutoff: float, system_idx: torch.Tensor, self_interaction: bool = False,
                *, half: bool = False, n_systems: int | None = None):
    """GPU neighbour list with the torch_nl_linked_cell contract.

    ``half=True`` returns the half list that full_to_half_list would keep
    (torch_sim/models/pair_potential.py:86-127).  ``n_systems`` may be passed to
    avoid the host synchronisation that infers it from ``system_idx``.
    """
    L.require_cuda(positions, "positions")
    dev = positions.device
    dtype = positions.dtype
    n_atoms = positions.shape[0]
    if n_systems is None:
        if cell.ndim == 3:
            n_systems = cell.shape[0]
        else:
            n_systems = int(system_idx.max().item()) + 1 if n_atoms else 1
    cell_row, pbc_u8 = _normalize(cell.to(dtype), pbc, n_systems)
    pos = positions.contiguous()
    sys_idx = system_idx.to(torch.int64).contiguous()
    flags = (L.NL_SELF_INTERACTION if self_interaction else 0) | (L.NL_HALF if half else 0)
    key = (n_atoms, n_systems, float(cutoff), flags)
    cap = _capacity_hint.get(key, 0)
    mapping, sysmap, shifts = torch.ops.tsb.nl_build(pos, cell_row, pbc_u8, sys_idx,
                                                     float(cutoff), flags, n_systems, cap)
    p = mapping.shape[1]
    if p > cap:
        _capacity_hint[key] = int(p * 1.15) + 16
    return mapping, sysmap, shifts


# names of the reference backends this replaces
cell_list_nl = torchsim_nl
torch_nl_linked_cell = torchsim_nl
default_batched_nl = torchsim_nl


def full_to_half_list(mapping: torch.Tensor, system_mapping: torch.Tensor,
                      shifts_idx: torch.Tensor):
    """Keep i<j, and for i==j the copy whose first non-zero shift is positive
    (torch_sim/models/pair_potential.py:86-127), as torch ops on the device."""
    i, j = mapping[0], mapping[1]
    s = shifts_idx
    first = torch.where(s[:, 0] != 0, s[:, 0], torch.where(s[:, 1] != 0, s[:, 1], s[:, 2]))
    keep = (i < j) | ((i == j) & (first > 0))
    return mapping[:, keep], system_mapping[keep], shifts_idx[keep]
