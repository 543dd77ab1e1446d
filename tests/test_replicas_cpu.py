"""The N-GPU bench path (independent replicas, no collective on the data
path) with world size 2 on the gloo backend, on the CPU: the slowest rank's
time and the work of all ranks are what the reported figure combines."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws))
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=ws)
    try:
        t = 10.0 + rank * 5.0          # rank 1 is the slower one
        work = 100.0 * (rank + 1)
        bench.barrier(ws)
        q.put((rank, bench.max_over_ranks(ws, t), bench.sum_over_ranks(ws, work)))
        bench.barrier(ws)
    finally:
        dist.destroy_process_group()


def test_two_replicas_combine_max_time_and_total_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert out == [(0, 15.0, 300.0), (1, 15.0, 300.0)]


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(1, 3.5) == 3.5 and bench.sum_over_ranks(1, 2.0) == 2.0
