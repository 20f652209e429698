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


def test_batched_jobs_mix_matches_its_specification():
    """The 256-job mix of the batched-jobs workload: 40 % RW with L in
    [10, 100], 40 % k-hop with fanouts from the fixed list, 20 % multi-RW of
    one 2000-walker, 10,000-step continuous-time sample; sizes lognormal,
    clipped to [1, 65536]; the same jobs for the same seed."""
    import bench
    jobs = bench.mix_jobs(1 << 20)
    assert len(jobs) == 256 and jobs == bench.mix_jobs(1 << 20)
    kinds = [j["type"] for j in jobs]
    assert kinds.count(0) == 102 and kinds.count(1) == 102 and kinds.count(2) == 52
    for j in jobs:
        if j["type"] == 0:
            assert 1 <= j["count"] <= 65536 and 10 <= j["length"] <= 100
        elif j["type"] == 1:
            assert 1 <= j["count"] <= 65536 and tuple(j["fanouts"]) in map(tuple, bench.MIX_FANOUTS)
        else:
            assert (j["count"], j["walkers"], j["steps"], j["select"]) == (1, 2000, 10000, 2)
    import numpy as np
    sizes = np.array([j["count"] for j in jobs if j["type"] != 2], dtype=np.float64)
    assert 300 < np.median(sizes) < 3000  # lognormal(ln 1024, 1.5)
    assert len({j["seed"] for j in jobs}) == 256
