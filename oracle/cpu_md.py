"""CPU baseline driver (TEST INFRASTRUCTURE / BASELINE ONLY; never the product path).

Times the oracle port of the reference hot path -- per system: neighbour list
(oracle.neighbors, torch_nl.py:156-215), Morse energy/forces (oracle.pair,
pair_potential.py:351-464) and one BAOAB Langevin step (oracle.md,
nvt.py:144-240) -- on the host cores.  Systems are independent, so a process
pool (spawn start method) spreads them over all cores.
"""

from __future__ import annotations

import multiprocessing as mp
import os
import time

import numpy as np

from . import md as omd
from . import pair as opair

MORSE = (2.866, 0.3429, 1.3588)  # sigma, epsilon, alpha (Cu)


def _system_slices(d):
    counts = np.bincount(d["system_idx"])
    off = np.concatenate([[0], np.cumsum(counts)])
    return off


def _advance(args):
    """Advance a list of systems by n_steps of BAOAB; returns atoms processed."""
    pos, mass, cell, sysi, n_steps, dt, kT, gamma, cutoff, seed = args
    rng = np.random.default_rng(seed)
    tab = opair.single_table(opair.MORSE, *MORSE)
    sp = np.zeros(len(pos), dtype=int)
    cell_row = np.transpose(cell, (0, 2, 1))
    pbc = np.array([True] * 3)

    def fn(q):
        o = opair.pair_forward(opair.MORSE, tab, sp, q, cell_row, pbc, sysi, cutoff)
        return o["energy"], o["forces"]

    e, f = fn(pos)
    st = {"positions": pos, "momenta": np.zeros_like(pos), "masses": mass, "forces": f,
          "energy": e}
    for _ in range(n_steps):
        st = omd.nvt_langevin_step(st, fn, dt, kT, gamma, rng.standard_normal(pos.shape), sysi)
    return len(pos) * n_steps


def sample_args(d, systems, n_steps, dt, kT, gamma, cutoff):
    off = _system_slices(d)
    out = []
    for k, s in enumerate(systems):
        a, b = off[s], off[s + 1]
        out.append((d["positions"][a:b].copy(), d["masses"][a:b].copy(), d["cell"][s:s + 1],
                    np.zeros(b - a, dtype=np.int64), n_steps, dt, kT, gamma, cutoff, k))
    return out


def time_sample(d, systems, n_steps, dt, kT, gamma, cutoff, processes=1):
    """Wall time of advancing `systems` by n_steps; returns (atom_steps, seconds).

    The force evaluation at the start of each system's trajectory is the
    reference's init call and is excluded by timing two runs (n_steps and 0)."""
    args = sample_args(d, systems, n_steps, dt, kT, gamma, cutoff)
    args0 = sample_args(d, systems, 0, dt, kT, gamma, cutoff)
    if processes > 1:
        ctx = mp.get_context("spawn")
        with ctx.Pool(processes) as pool:
            pool.map(_advance, args0[:processes])  # warm the workers
            t0 = time.perf_counter()
            pool.map(_advance, args0, chunksize=1)
            t_init = time.perf_counter() - t0
            t0 = time.perf_counter()
            atom_steps = sum(pool.map(_advance, args, chunksize=1))
            t = time.perf_counter() - t0
    else:
        t0 = time.perf_counter()
        for a in args0:
            _advance(a)
        t_init = time.perf_counter() - t0
        t0 = time.perf_counter()
        atom_steps = sum(_advance(a) for a in args)
        t = time.perf_counter() - t0
    return atom_steps, max(t - t_init, 1e-9)


def cpu_count() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1
