"""The multi-GPU form of bench.py (independent replicas, one per rank, no
collective on the data path) checked with two gloo ranks on the CPU: every
rank takes the same collective steps, and the reported time is the maximum
over ranks."""
import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    r, w, lr = bench.dist_env()
    dist = bench.init_dist(w, "gloo")
    bench.barrier(w)
    t = bench.max_over_ranks(10.0 + 5.0 * r, w, "cpu")
    bench.barrier(w)
    q.put((r, w, lr, t))
    dist.destroy_process_group()


def test_two_gloo_ranks_max_over_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(2))
    assert got == [(0, 2, 0, 15.0), (1, 2, 1, 15.0)]
