"""Multi-process plumbing of bench.py on CPU (gloo, world size 2).

The DEM path runs one independent simulation per GPU (replicas, no data
exchange), so the only collectives are the timing barrier and the
max/sum reductions over ranks; they are exercised here without a GPU.
"""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench

    bench.barrier(dist)
    mx = bench.max_over_ranks(dist, 10.0 + rank)
    sm = bench.sum_over_ranks(dist, 1.5 * (rank + 1))
    q.put((rank, mx, sm))
    dist.destroy_process_group()


def test_rank_reductions_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 11.0, 4.5), (1, 11.0, 4.5)]


def test_single_rank_helpers_are_identity():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(None, 3.0) == 3.0 and bench.sum_over_ranks(None, 2.0) == 2.0
    bench.barrier(None)
