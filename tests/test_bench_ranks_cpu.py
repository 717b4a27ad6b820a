"""The multi-GPU bench path (replicas, one process per GPU) on CPU: two gloo ranks
combine their timings the way bench.py does (slowest rank's time, sum of work)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    sec, work = bench.combine_ranks(0.5 + rank, 100.0 * (rank + 1), "cpu")
    out[rank] = (sec, work)
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_combine_like_the_bench():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        assert out[r] == (1.5, 300.0)
