"""Admission policy for batches: bin packing of systems by an estimated memory
cost, as the reference autobatcher does it.

* ``to_constant_volume_bins``   <- torch_sim/autobatching.py:46-144: items
  sorted by weight, heaviest first; each goes into the fullest bin that still
  has room for it, or opens a new bin.
* ``calculate_memory_scalers``  <- autobatching.py:305-420: per-system cost
  ``n_atoms`` or ``n_atoms x number density`` (atoms^2 / nm^3; for a system that
  is not periodic on every axis, the bounding box padded by 2 A on the open
  axes stands in for the cell).
* ``BinningAutoBatcher``        <- autobatching.py:475-765: packs the systems of
  a state into batches whose summed cost stays below ``max_memory_scaler`` and
  yields them as sub-states.  The reference finds that bound by probing the
  model until it runs out of memory; here the caller gives it (the tsb kernels'
  memory is known in advance: the fused kernel holds a system in shared memory
  and a batch needs O(atoms) device memory).

``tsb.integrators.run_md`` uses these to route a batch: systems that fit the
persistent fused kernel go there in bins of bounded cost, larger systems take
the per-call step functions.
"""

from __future__ import annotations

from typing import Any, Callable, Iterator

import torch

from . import _lib as L


def to_constant_volume_bins(items, max_volume: float, *, weight_pos: int | None = None,
                            key: Callable[[Any], float] | None = None,
                            lower_bound: float | None = None,
                            upper_bound: float | None = None) -> list:
    """Pack items into the fewest bins of summed weight <= max_volume (best fit,
    heaviest first).  ``items``: dict key -> weight (bins are dicts), list of
    weights (bins are lists of weights), or list of tuples/objects with
    ``weight_pos`` or ``key`` (bins are lists of the items).  Items at or below
    ``lower_bound`` or at or above ``upper_bound`` are left out.  An item heavier
    than max_volume gets a bin of its own."""
    if lower_bound is not None and upper_bound is not None and lower_bound >= upper_bound:
        raise ValueError("lower_bound is greater or equal to upper_bound")
    if not hasattr(items, "__len__"):
        raise TypeError("items must be iterable")
    if len(items) == 0:
        return []
    is_dict = isinstance(items, dict)
    if is_dict:
        pairs = [(float(w), k) for k, w in items.items()]
    elif weight_pos is not None:
        pairs = [(float(it[weight_pos]), it) for it in items]
    elif key is not None:
        pairs = [(float(key(it)), it) for it in items]
    elif isinstance(items[0], (tuple, list)):
        raise ValueError("Must provide weight_pos or key for tuple list")
    else:
        pairs = [(float(w), w) for w in items]
    if lower_bound is not None:
        pairs = [p for p in pairs if p[0] > lower_bound]
    if upper_bound is not None:
        pairs = [p for p in pairs if p[0] < upper_bound]
    # stable: equal weights keep their input order
    order = sorted(range(len(pairs)), key=lambda i: -pairs[i][0])
    loads: list[float] = []
    bins: list[list] = []
    for i in order:
        w, payload = pairs[i]
        best = -1
        for b, load in enumerate(loads):
            if load + w <= max_volume and (best < 0 or load > loads[best]):
                best = b
        if best < 0:
            loads.append(w)
            bins.append([(w, payload)])
        else:
            loads[best] += w
            bins[best].append((w, payload))
    if is_dict:
        return [{payload: w for w, payload in b} for b in bins]
    return [[payload for _, payload in b] for b in bins]


def calculate_memory_scalers(state, memory_scales_with: str = "n_atoms_x_density") -> list:
    """Per-system memory cost: ``n_atoms`` or ``n_atoms * n_atoms / volume[nm^3]``."""
    counts = torch.bincount(state.system_idx, minlength=state.n_systems).to(torch.float64)
    if memory_scales_with == "n_atoms":
        return counts.tolist()
    if memory_scales_with != "n_atoms_x_density":
        raise ValueError(f"Invalid metric: {memory_scales_with}")
    pbc = L.pbc_rows(state.pbc, state.n_systems, state.device).bool()
    vol = torch.linalg.det(state.cell.to(torch.float64)).abs() / 1000.0
    open_sys = ~pbc.all(dim=1)
    if bool(open_sys.any()):
        pos = state.positions.to(torch.float64)
        for s in torch.nonzero(open_sys).flatten().tolist():
            x = pos[state.system_idx == s]
            box = x.max(dim=0).values - x.min(dim=0).values
            box = box + 2.0 * (~pbc[s]).to(torch.float64)
            vol[s] = torch.prod(box) / 1000.0
    return torch.where(vol > 0, counts * counts / vol, counts).tolist()


class BinningAutoBatcher:
    """Batches of systems whose summed memory cost stays below a bound.

    ``load_states(state)`` packs the systems; iterating yields
    ``(sub_state, system_indices)`` per batch (systems renumbered 0..k-1 in
    ascending order of their index in ``state``); ``restore_original_order``
    puts per-batch results back in the order of the loaded state."""

    def __init__(self, model=None, *, memory_scales_with: str = "n_atoms_x_density",
                 max_memory_scaler: float | None = None) -> None:
        if max_memory_scaler is None:
            raise ValueError("max_memory_scaler must be given (no out-of-memory probing)")
        self.model = model
        self.memory_scales_with = memory_scales_with
        self.max_memory_scaler = float(max_memory_scaler)
        self.state = None
        self.batched_indices: list[list[int]] = []

    def load_states(self, state) -> float:
        self.state = state
        scalers = calculate_memory_scalers(state, self.memory_scales_with)
        bins = to_constant_volume_bins(dict(enumerate(scalers)), self.max_memory_scaler)
        self.batched_indices = [sorted(b) for b in bins]
        return max(scalers) if scalers else 0.0

    def __iter__(self) -> Iterator:
        from .state import select_systems

        if self.state is None:
            raise RuntimeError("call load_states first")
        for idx in self.batched_indices:
            yield select_systems(self.state, idx), idx

    def restore_original_order(self, batched: list) -> list:
        """Per-system results listed batch by batch -> the loaded state's order."""
        flat = [i for b in self.batched_indices for i in b]
        out = [None] * len(flat)
        for pos, item in zip(flat, batched):
            out[pos] = item
        return out
