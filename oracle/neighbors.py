"""Neighbour-list oracle (TEST INFRASTRUCTURE ONLY; never the product path).

FP64 numpy restatement of the reference's pure-torch neighbour lists:

* ``wrap_positions``   <- torch_sim/transforms.py:160-210
  (pbc_wrap_batched_and_get_lattice_shifts)
* ``cell_repeats``     <- torch_sim/transforms.py:435-467 (get_number_of_cell_repeats)
* ``neighbor_list``    <- torch_sim/neighbors/torch_nl.py:156-215 (torch_nl_linked_cell)
  with the strict cutoff of torch_nl.py:25-91 and the shift correction of
  torch_nl.py:214.  The candidate set is all image shifts in
  ``[-rep, rep]^3`` per system (rep from ``cell_repeats``), which is exactly the
  set of images the reference's linked cell replicates (transforms.py:886-899);
  the pair set is therefore identical (checked against the reference's own
  output in tests/test_oracle_golden.py).
* ``full_to_half_list`` <- torch_sim/models/pair_potential.py:86-127

Pair-set convention (torch_nl.py:214, pair_potential.py:182): a triple
``(i, j, S)`` is a neighbour when ``|r_j - r_i + S @ cell_row| < cutoff``
for the *unwrapped* positions ``r``; the unshifted self pair ``(i, i, 0)`` is
excluded unless ``self_interaction``.
"""

from __future__ import annotations

import numpy as np


def normalize_inputs(cell, pbc, n_systems):
    """Broadcast cell to [S,3,3] and pbc to [S,3] (neighbors/utils.py:7-34)."""
    cell = np.asarray(cell, dtype=np.float64)
    pbc = np.asarray(pbc, dtype=bool)
    if cell.ndim == 2:
        cell = (np.broadcast_to(cell, (n_systems, 3, 3)) if cell.shape[0] == 3
                else cell.reshape(n_systems, 3, 3))
    if pbc.ndim == 1:
        pbc = (np.broadcast_to(pbc, (n_systems, 3)) if pbc.shape[0] == 3
               else pbc.reshape(n_systems, 3))
    return np.ascontiguousarray(cell), np.ascontiguousarray(pbc)


def wrap_positions(positions, cell_row, system_idx, pbc):
    """Wrap into the primary cell; return (wrapped, integer lattice shifts).

    transforms.py:160-210: ``f = inv(cell_row.T) r``; on periodic axes of systems
    with an invertible cell and any periodic axis, ``shift = floor(f)`` and
    ``wrapped = cell_row.T (f - shift)``; other atoms are returned unchanged.
    """
    pos = np.asarray(positions, dtype=np.float64)
    cell_T = np.transpose(cell_row, (0, 2, 1))
    dets = np.linalg.det(cell_T)
    invertible = np.isfinite(dets) & (np.abs(dets) > 1e-12)
    active = pbc.any(axis=1) & invertible
    if not active.any():
        return pos.copy(), np.zeros_like(pos)
    B = np.zeros_like(cell_row)
    B[active] = np.linalg.inv(cell_T[active])
    frac = np.einsum("nij,nj->ni", B[system_idx], pos)
    mask = pbc[system_idx] & active[system_idx][:, None]
    shifts = np.where(mask, np.floor(frac), 0.0)
    wrapped = np.einsum("nij,nj->ni", cell_T[system_idx], frac - shifts)
    act = active[system_idx][:, None]
    return np.where(act, wrapped, pos), np.where(act, shifts, 0.0)


def cell_repeats(cutoff, cell_row, pbc):
    """ceil(cutoff * |row k of inv(cell)^T|) on periodic axes (transforms.py:435-467)."""
    has_pbc = pbc.any(axis=1)
    recip = np.zeros_like(cell_row)
    if has_pbc.any():
        recip[has_pbc] = np.transpose(np.linalg.inv(cell_row[has_pbc]), (0, 2, 1))
    inv_d = np.linalg.norm(recip, axis=-1)
    rep = np.ceil(cutoff * inv_d).astype(np.int64)
    return np.where(pbc, rep, 0)


def _system_offsets(system_idx, n_systems):
    counts = np.bincount(system_idx, minlength=n_systems)
    off = np.zeros(n_systems + 1, dtype=np.int64)
    off[1:] = np.cumsum(counts)
    return off


def neighbor_list(positions, cell, pbc, cutoff, system_idx, self_interaction=False,
                  chunk=256):
    """Full neighbour list (both directions) as in torch_nl.py:156-215.

    Returns ``mapping [2,P] int64, system_mapping [P] int64, shifts [P,3] float64``
    sorted lexicographically by (system, i, j, shift) so two lists compare with
    ``np.array_equal``.
    """
    system_idx = np.asarray(system_idx, dtype=np.int64)
    if system_idx.size == 0:
        return (np.zeros((2, 0), np.int64), np.zeros(0, np.int64), np.zeros((0, 3)))
    n_systems = int(system_idx.max()) + 1
    cell_row, pbc = normalize_inputs(cell, pbc, n_systems)
    wrapped, wshift = wrap_positions(positions, cell_row, system_idx, pbc)
    rep = cell_repeats(cutoff, cell_row, pbc)
    off = _system_offsets(system_idx, n_systems)
    rc2 = cutoff * cutoff
    out_i, out_j, out_s, out_sys = [], [], [], []
    for s in range(n_systems):
        a0, a1 = off[s], off[s + 1]
        n = a1 - a0
        if n == 0:
            continue
        ax = [np.arange(-r, r + 1) for r in rep[s]]
        shifts = np.stack(np.meshgrid(*ax, indexing="ij"), -1).reshape(-1, 3)
        cs = shifts.astype(np.float64) @ cell_row[s]          # [K,3]
        w = wrapped[a0:a1]
        for c0 in range(0, n, chunk):
            c1 = min(n, c0 + chunk)
            # d = w_i - w_j - S@cell   (torch_nl.py:80-86 / transforms.py:540-566)
            d = (w[c0:c1, None, None, :] - w[None, :, None, :]
                 - cs[None, None, :, :])
            d2 = np.einsum("ijkx,ijkx->ijk", d, d)
            m = d2 < rc2
            if not self_interaction:
                zero = np.all(shifts == 0, axis=1)
                ii = np.arange(c0, c1)
                m[ii - c0, ii, :] &= ~zero[None, :]
            li, lj, lk = np.nonzero(m)
            out_i.append(li + c0 + a0)
            out_j.append(lj + a0)
            out_s.append(shifts[lk])
            out_sys.append(np.full(li.shape, s, dtype=np.int64))
    if not out_i:
        return (np.zeros((2, 0), np.int64), np.zeros(0, np.int64), np.zeros((0, 3)))
    i = np.concatenate(out_i)
    j = np.concatenate(out_j)
    S = np.concatenate(out_s).astype(np.float64)
    sysm = np.concatenate(out_sys)
    # shift correction to unwrapped positions (torch_nl.py:214)
    S = S + wshift[i] - wshift[j]
    return sort_pairs(np.stack([i, j]), sysm, S)


def sort_pairs(mapping, system_mapping, shifts):
    """Canonical order for set comparison: by (system, i, j, sx, sy, sz)."""
    mapping = np.asarray(mapping, dtype=np.int64)
    shifts = np.asarray(shifts, dtype=np.float64)
    system_mapping = np.asarray(system_mapping, dtype=np.int64)
    if mapping.shape[1] == 0:
        return mapping, system_mapping, shifts.reshape(0, 3)
    si = np.rint(shifts).astype(np.int64)
    order = np.lexsort((si[:, 2], si[:, 1], si[:, 0], mapping[1], mapping[0],
                        system_mapping))
    return mapping[:, order], system_mapping[order], shifts[order]


def pair_set_digest(mapping, shifts):
    """SHA-256 of a pair set (one system) independent of its order: each pair
    (i, j, sx, sy, sz) packed into one int64 key (i, j < 2^19, |s| <= 3),
    keys sorted ascending, little-endian bytes hashed.  Test infrastructure for
    comparing pair sets too large to store (tens of millions of pairs)."""
    import hashlib

    m = np.asarray(mapping, dtype=np.int64)
    si = np.rint(np.asarray(shifts, dtype=np.float64)).astype(np.int64)
    if m.size and (m.min() < 0 or m.max() >= 1 << 19 or np.abs(si).max() > 3):
        raise ValueError("pair_set_digest: index or shift outside the packed range")
    key = (((m[0] << 19) | m[1]) << 9) | ((si[:, 0] + 4) << 6) | ((si[:, 1] + 4) << 3) | (
        si[:, 2] + 4)
    key = np.sort(key).astype("<i8")
    return hashlib.sha256(key.tobytes()).hexdigest(), int(key.size)


def full_to_half_list(mapping, system_mapping, shifts):
    """Keep i<j, and for i==j the copy whose first non-zero shift is > 0.

    pair_potential.py:86-127.
    """
    i, j = mapping
    keep = i < j
    same = i == j
    if same.any():
        s = shifts[same]
        first = np.zeros(len(s))
        resolved = np.zeros(len(s), dtype=bool)
        for d in range(3):
            nz = (s[:, d] != 0) & ~resolved
            first = np.where(nz, s[:, d], first)
            resolved |= nz
        keep = keep.copy()
        keep[same] = first > 0
    return mapping[:, keep], system_mapping[keep], shifts[keep]


def neighbor_list_cells(positions, cell_row, cutoff, self_interaction=False):
    """Full neighbour list of ONE fully periodic system by a cell list, for
    systems too large for the all-pairs restatement (tens of thousands of atoms).

    The reference's single-system linked cell (transforms.py:843-1006) bins
    atoms into cells at least ``cutoff`` wide and pairs each cell with its 27
    neighbours.  Here: positions wrapped into the cell (transforms.py:160-210),
    fractional bins of at least ``cutoff`` in every direction (n_k =
    floor(1 / (cutoff |b_k|)), b_k the reciprocal rows; requires n_k >= 3), and
    for every bin and each of the 27 neighbour offsets the distances between all
    atom pairs, with the periodic shift the offset implies.  Returns the pair set
    in the layout and order of :func:`neighbor_list` (shifts valid for the
    unwrapped input positions, torch_nl.py:214).
    """
    pos = np.asarray(positions, dtype=np.float64)
    C = np.asarray(cell_row, dtype=np.float64).reshape(3, 3)
    n = pos.shape[0]
    T = np.linalg.inv(C)                      # fractional u = r @ T (row vectors)
    u = pos @ T
    wshift = np.floor(u)
    uw = u - wshift
    wrapped = uw @ C
    recip = np.linalg.inv(C).T                # rows b_k
    nb = np.floor(1.0 / (cutoff * np.linalg.norm(recip, axis=1))).astype(int)
    if (nb < 3).any():
        raise ValueError("neighbor_list_cells needs every cell width >= 3 cutoffs")
    b = np.minimum((uw * nb).astype(int), nb - 1)
    lin = (b[:, 0] * nb[1] + b[:, 1]) * nb[2] + b[:, 2]
    order = np.argsort(lin, kind="stable")
    counts = np.bincount(lin, minlength=int(np.prod(nb)))
    start = np.concatenate([[0], np.cumsum(counts)])
    rc2 = cutoff * cutoff
    out_i, out_j, out_s = [], [], []
    offs = np.array([(a, bb, c) for a in (-1, 0, 1) for bb in (-1, 0, 1) for c in (-1, 0, 1)])
    bins3 = np.stack(np.unravel_index(np.arange(int(np.prod(nb))), nb), 1)
    for off in offs:
        nbr = bins3 + off
        shift = np.floor_divide(nbr, nb)      # lattice shift of the neighbour bin
        nbr = nbr - shift * nb
        nlin = (nbr[:, 0] * nb[1] + nbr[:, 1]) * nb[2] + nbr[:, 2]
        for bi in np.nonzero(counts)[0]:
            bj = nlin[bi]
            if counts[bj] == 0:
                continue
            ii = order[start[bi]:start[bi + 1]]
            jj = order[start[bj]:start[bj + 1]]
            s = shift[bi].astype(np.float64)
            d = wrapped[jj][None, :, :] + (s @ C)[None, None, :] - wrapped[ii][:, None, :]
            d2 = np.einsum("ijk,ijk->ij", d, d)
            m = d2 < rc2
            if not self_interaction and not s.any():
                m &= ii[:, None] != jj[None, :]
            a, c = np.nonzero(m)
            out_i.append(ii[a])
            out_j.append(jj[c])
            out_s.append(np.broadcast_to(s, (len(a), 3)))
    i = np.concatenate(out_i)
    j = np.concatenate(out_j)
    S = np.concatenate(out_s)
    # the pair (i, j, S) on wrapped positions is (i, j, S + w_i - w_j) on the inputs
    S = S + wshift[i] - wshift[j]
    return sort_pairs(np.stack([i, j]), np.zeros(len(i), np.int64), S)
