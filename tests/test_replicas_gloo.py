"""The multi-GPU bench path runs independent replicas: ranks combine the
slowest rank's time and the sum of their pairs. Checked with 2 gloo ranks."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    t, p = bench.combine_ranks(10.0 + rank, 100 * (rank + 1), dist, "cpu")
    q.put((rank, t, p))
    dist.destroy_process_group()


def test_combine_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for pr in procs:
        pr.start()
    for pr in procs:
        pr.join(timeout=120)
        assert pr.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, t, p in res:
        assert t == 11.0 and p == 300


def test_combine_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.combine_ranks(5.0, 7) == (5.0, 7)
