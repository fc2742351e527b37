"""The multi-process plumbing of bench.py (one process per GPU), on CPU with gloo.

Each of two ranks reports a different step time; every rank must agree on the
maximum (the driver reads rank 0's line), and the barrier must release both.
"""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        barrier, max_over_ranks = bench.dist_helpers(dist, torch.device("cpu"))
        barrier()
        got = max_over_ranks(10.0 + 5.0 * rank)
        barrier()
        out.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_barrier_two_ranks():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert res == [(0, 15.0), (1, 15.0)]


def test_single_process_helpers_are_noops():
    import torch
    import bench
    barrier, max_over_ranks = bench.dist_helpers(None, torch.device("cpu"))
    barrier()
    assert max_over_ranks(3.5) == 3.5
