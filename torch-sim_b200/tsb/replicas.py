"""Multi-GPU replicas: systems are independent (no pair crosses a system), so N
GPUs run N independent batches with no collective in the step.  The only
collectives are the barrier around a timed interval and the max of the
per-rank intervals (the job is as slow as its slowest rank).
"""

from __future__ import annotations

import os

import torch


def world():
    """(world_size, rank, local_rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def barrier() -> None:
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.barrier()


def max_over_ranks(seconds: float, device=None) -> float:
    """Max of a per-rank duration over all ranks (a no-op on one rank)."""
    if not (torch.distributed.is_available() and torch.distributed.is_initialized()):
        return float(seconds)
    t = torch.tensor([float(seconds)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t)


def weak_scaling_value(units_per_rank: float, seconds_max: float, world_size: int) -> float:
    """Whole-job throughput: the units all ranks processed / the slowest rank's time."""
    return units_per_rank * world_size / seconds_max


def shard_systems(counts, world_size: int, rank: int):
    """Atom-balanced assignment of whole systems to ranks (largest first, each to
    the currently lightest rank) -- the idea of the reference's
    to_constant_volume_bins (autobatching.py:46-144) applied across GPUs."""
    order = sorted(range(len(counts)), key=lambda s: -int(counts[s]))
    load = [0] * world_size
    owner = [0] * len(counts)
    for s in order:
        r = min(range(world_size), key=lambda k: (load[k], k))
        owner[s] = r
        load[r] += int(counts[s])
    return [s for s in range(len(counts)) if owner[s] == rank]
