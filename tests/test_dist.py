"""The multi-process plumbing of bench.py (one process per GPU, replicas with
no data exchange) with two gloo ranks on the CPU: rank reductions, barrier,
and per-replica seeds."""
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


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch
    import bench
    w, r, local = bench.dist_env()
    dist = bench.dist_init(w, "gloo")
    try:
        bench.barrier(dist)
        t = bench.max_over_ranks(dist, 1.5 + rank, torch)      # slowest rank's time
        e = bench.sum_over_ranks(dist, 10.0 * (rank + 1), torch)  # whole-job edges
        seeds = bench.replica_seed(7, r)
        q.put((r, w, local, t, e, seeds))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get(timeout=10) for _ in range(2))
    assert [o[0] for o in out] == [0, 1] and all(o[1] == 2 for o in out)
    assert all(o[3] == 2.5 for o in out)   # max over ranks
    assert all(o[4] == 30.0 for o in out)  # sum over ranks
    assert out[0][5] != out[1][5]          # replicas draw different walkers


def test_single_process_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.dist_init(1, "gloo") is None
    assert bench.max_over_ranks(None, 3.0) == 3.0
    assert bench.sum_over_ranks(None, 4.0) == 4.0
