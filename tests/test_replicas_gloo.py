"""N>1 host path on CPU: two gloo ranks agree on the max interval and the
whole-job throughput, and the system shards cover every system once."""

import os
import socket

import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world_size, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      WORLD_SIZE=str(world_size), RANK=str(rank), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    from tsb import replicas

    assert replicas.world() == (world_size, rank, rank)
    replicas.barrier()
    t = replicas.max_over_ranks(1.0 + rank)
    v = replicas.weak_scaling_value(1000.0, t, world_size)
    mine = replicas.shard_systems([5, 9, 1, 7, 3, 3, 8], world_size, rank)
    out[rank] = (t, v, mine)
    dist.destroy_process_group()


def test_two_gloo_ranks():
    import sys

    from conftest import PKG

    if PKG not in sys.path:
        sys.path.insert(0, PKG)
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    os.environ["PYTHONPATH"] = PKG + os.pathsep + os.environ.get("PYTHONPATH", "")
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert out[0][0] == out[1][0] == 2.0
    assert out[0][1] == out[1][1] == 1000.0
    shards = out[0][2] + out[1][2]
    assert sorted(shards) == list(range(7))
    loads = [sum([5, 9, 1, 7, 3, 3, 8][s] for s in out[r][2]) for r in (0, 1)]
    assert abs(loads[0] - loads[1]) <= 3
