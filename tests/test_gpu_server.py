"""GPU tests of the serving loop: every request's result is identical to the
standalone call with the same parameters and seed, whatever batch it lands
in, under several windows, stream counts and scratch budgets; requests over
the budget and malformed requests fail with their status; the load
generator serves one trace identically batched and one-job-per-launch."""
import os
import threading

import numpy as np
import pytest

from conftest import golden_graph
import grass_b200 as G

pytestmark = pytest.mark.gpu


def _mix(n, rng, k):
    """k requests: (kind, args) with uneven sizes and parameters."""
    out = []
    for i in range(k):
        t = i % 5
        seed = 1000 + i
        if t in (0, 1):
            W = int(rng.integers(0, 700)) if t == 0 else int(rng.integers(1, 5))
            out.append(("rw", dict(starts=rng.integers(0, n, W).astype(np.uint32),
                                   length=int(rng.integers(0, 40)), seed=seed,
                                   layout=int(rng.integers(0, 2)))))
        elif t in (2, 3):
            fan = [(25, 10), (5, 5, 5), (10,), (3, 7)][i % 4]
            S = int(rng.integers(1, 200))
            out.append(("khop", dict(seeds=rng.integers(0, n, S).astype(np.uint32),
                                     fanouts=fan, seed=seed)))
        else:
            out.append(("mrw", dict(samples=int(rng.integers(1, 4)), walkers=int(rng.integers(1, 300)),
                                    steps=int(rng.integers(1, 120)), seed=seed,
                                    select=(i // 5) % 3, given=bool(i % 3 == 0))))
    return out


def _expected(torch, g, kind, a):
    if kind == "rw":
        p, e = g.rw(a["starts"], a["length"], a["seed"], layout=a["layout"])
        return [p.reshape(-1)], e
    if kind == "khop":
        outs, e = g.khop(a["seeds"], a["fanouts"], a["seed"])
        return [o.reshape(-1) for o in outs], e
    roots = a["roots"]
    src, dst, _, e = g.mrw(roots, a["steps"], a["seed"], select=a["select"])
    return [src.reshape(-1), dst.reshape(-1)], e


def _roots(torch, g, a):
    S, R = a["samples"], a["walkers"]
    if a["given"]:
        return np.random.default_rng(a["seed"]).integers(0, g.n, (S, R)).astype(np.uint32)
    d = torch.empty(S * R, dtype=torch.int32, device="cuda")
    G.mrw_roots_device(g.n, S, R, a["seed"], d)
    return d.cpu().numpy().view(np.uint32).reshape(S, R)


def _submit(srv, kind, a):
    if kind == "rw":
        return srv.submit_rw(a["starts"], a["length"], a["seed"], layout=a["layout"])
    if kind == "khop":
        return srv.submit_khop(a["seeds"], a["fanouts"], a["seed"])
    return srv.submit_mrw(a["samples"], a["walkers"], a["steps"], a["seed"], select=a["select"],
                          roots=a["roots"] if a["given"] else None)


@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("cfg", [
    dict(),                                                   # defaults
    dict(window_min_us=1, window_max_us=1, max_inflight=1),   # ~one request per batch
    dict(window_min_us=5000, window_max_us=20000, max_inflight=4,
         batch=dict(walker_tile=64, depth=2, warps_per_block=2, khop_seeds=3)),
    dict(scratch_budget=1 << 20, max_inflight=3),             # admission waits for scratch
    dict(results_on_device=1, window_min_us=50),              # outputs kept in HBM
])
def test_server_results_equal_standalone(mode, cfg):
    import torch
    d, *_ = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, mode), mode)
    rng = np.random.default_rng(11)
    reqs = _mix(g.n, rng, 60)
    for kind, a in reqs:
        if kind == "mrw":
            a["roots"] = _roots(torch, g, a)
    expect = [_expected(torch, g, kind, a) for kind, a in reqs]
    srv = G.Server(g, **cfg)
    tickets = [None] * len(reqs)

    def worker(idx):  # several client threads submit interleaved
        for i in idx:
            tickets[i] = _submit(srv, *reqs[i])

    ths = [threading.Thread(target=worker, args=(range(k, len(reqs), 3),)) for k in range(3)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    batches = set()
    for (kind, a), tk, (outs, e) in zip(reqs, tickets, expect):
        res = srv.wait(tk, timeout_ms=60000)
        assert res["status"] == G.OK
        assert res["on_device"] == bool(cfg.get("results_on_device"))
        assert res["edges"] == e, kind
        assert len(res["outputs"]) == len(outs)
        for o, r in zip(res["outputs"], outs):
            np.testing.assert_array_equal(o, r, err_msg=kind)
        assert res["submit_us"] <= res["launch_us"] <= res["done_us"]
        batches.add(res["batch"])
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["batches"] == len(batches)
    if "scratch_budget" in cfg:
        assert st["scratch_peak"] <= cfg["scratch_budget"]
        assert st["batches"] > 1
    srv.close()


def test_results_on_device_hold_budget_until_released():
    """Results kept in device memory count against the scratch budget until
    released: a request that does not fit waits, and runs after the release."""
    import time
    d, *_ = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, "LE"), "LE")
    starts = np.arange(4000, dtype=np.uint32) % g.n
    # each request: 4000 starts + 4000 x 41 path words ~ 672 KB; budget fits one
    srv = G.Server(g, results_on_device=1, scratch_budget=1 << 20, window_min_us=10)
    ta = srv.submit_rw(starts, 40, 1)
    ra = srv.wait(ta, release=False)
    assert ra["on_device"]
    tb = srv.submit_rw(starts, 40, 2)
    time.sleep(0.3)
    assert not srv.poll(tb)  # A's result still holds the budget
    G.lib.grass_server_release(srv._h, ta)
    rb = srv.wait(tb, timeout_ms=10000)
    ref, e = g.rw(starts, 40, 2)
    np.testing.assert_array_equal(rb["outputs"][0], ref.reshape(-1))
    assert rb["edges"] == e
    srv.close()


def test_server_errors_and_empty_requests():
    d, *_ = golden_graph("hub")
    g = G.Graph(os.path.join(d, "LE"), "LE")
    srv = G.Server(g, scratch_budget=1 << 20, window_min_us=10)
    with pytest.raises(G.GrassError) as ei:  # 400k walkers x 11 words > 1 MiB
        srv.submit_rw(np.zeros(400_000, np.uint32), 10, 1)
    assert ei.value.code == G.E_BUDGET
    bad = G.Request(type=7, count=1)
    with pytest.raises(G.GrassError) as ei:
        srv.submit(bad)
    assert ei.value.code == G.E_ARG
    r = G.Request(type=G.JOB_KHOP, count=1, seed=1, hops=0)  # no hops
    with pytest.raises(G.GrassError):
        srv.submit(r)
    r = G.Request(type=G.JOB_RW, count=3, seed=1, length=4)  # missing input
    with pytest.raises(G.GrassError):
        srv.submit(r)
    # Empty requests complete with empty outputs.
    t0 = srv.submit_rw(np.zeros(0, np.uint32), 10, 1)
    t1 = srv.submit_khop(np.zeros(0, np.uint32), (3, 2), 1)
    t2 = srv.submit_mrw(0, 5, 7, 1)
    for t in (t0, t1, t2):
        res = srv.wait(t)
        assert res["edges"] == 0 and all(o.size == 0 for o in res["outputs"])
    with pytest.raises(G.GrassError):
        srv.wait(12345)
    st = srv.stats()
    assert st["rejected"] == 4 and st["completed"] == 3
    srv.close()


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_loadgen_batched_equals_one_job_per_launch(mode):
    d, *_ = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, mode), mode)
    kw = dict(rate=20000.0, requests=300, seed=3, size_mu=np.log(64), size_sigma=1.0,
              size_max=2048, mrw_walkers=100, mrw_steps=200)
    a = G.loadgen(g, mode=0, **kw)
    b = G.loadgen(g, mode=1, **kw)
    for r in (a, b):
        assert r["completed"] == 300 and r["failed"] == 0 and r["rejected"] == 0
        assert 0 < r["p50_us"] <= r["p99_us"] <= r["p999_us"] <= r["max_us"]
        assert r["launches"] > 0
    assert a["edges"] == b["edges"]  # same trace, same Philox streams
    assert a["batches"] < 300        # requests were batched


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_requests_overlap_a_running_batch(mode):
    """Continuous batching: a walk request that arrives while a long multi-RW
    chain is on the GPU is admitted on another stream and completes inside the
    chain's [launch, done] interval, so its work overlapped the chain's on the
    device (one at a time, it would finish after the chain).  Both results
    equal their standalone calls."""
    import time
    d, *_ = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, mode), mode)
    srv = G.Server(g, window_min_us=50, window_max_us=200)
    # one sequential degree-proportional chain: ~2 us per step, tens of ms
    chain = dict(samples=1, walkers=2000, steps=20000, seed=77, select=1)
    t_chain = srv.submit_mrw(chain["samples"], chain["walkers"], chain["steps"], chain["seed"],
                             select=chain["select"])
    time.sleep(0.003)  # the chain's batch is on the GPU
    starts = np.random.default_rng(2).integers(0, g.n, 500).astype(np.uint32)
    t_walk = srv.submit_rw(starts, 30, 78)
    walk = srv.wait(t_walk, timeout_ms=60000)
    res = srv.wait(t_chain, timeout_ms=60000)
    assert walk["status"] == G.OK and res["status"] == G.OK
    assert walk["batch"] != res["batch"]
    assert res["launch_us"] < walk["launch_us"] and walk["done_us"] < res["done_us"], (
        res["launch_us"], res["done_us"], walk["launch_us"], walk["done_us"])
    p, e = g.rw(starts, 30, 78)
    np.testing.assert_array_equal(walk["outputs"][0], p.reshape(-1))
    assert walk["edges"] == e
    import torch  # the chain's roots were drawn on the device from its seed
    rt = torch.empty(chain["walkers"], dtype=torch.int32, device="cuda")
    G.mrw_roots_device(g.n, 1, chain["walkers"], chain["seed"], rt)
    roots = rt.cpu().numpy().view(np.uint32).reshape(1, -1)
    src, dst, _, e2 = g.mrw(roots, chain["steps"], chain["seed"], select=chain["select"])
    np.testing.assert_array_equal(res["outputs"][0], src.reshape(-1))
    np.testing.assert_array_equal(res["outputs"][1], dst.reshape(-1))
    assert res["edges"] == e2
    srv.close()


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_held_results_do_not_stall_later_requests(mode):
    """A caller holds every result while it waits for the next, and the
    results together are far larger than the pinned staging arena.  Waiting
    for releases would stall for good; the server stages the later batches
    through its fallback pool and every request finishes, with the
    standalone result."""
    d, *_ = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, mode), mode)
    n = g.n
    rng = np.random.default_rng(9)
    srv = G.Server(g, staging_bytes=1 << 20, max_inflight=2, window_min_us=1, window_max_us=1)
    reqs = []
    for i in range(12):  # each result ~160-320 KB: the 1 MiB arena holds a few at most
        starts = rng.integers(0, n, 1000 + 100 * i).astype(np.uint32)
        reqs.append((starts, 39, 500 + i, srv.submit_rw(starts, 39, 500 + i)))
    held = []
    for starts, L, seed, t in reqs:
        held.append((starts, L, seed, srv.wait(t, timeout_ms=20000, release=False)))
    for starts, L, seed, r in held:
        p, _ = g.rw(starts, L, seed)
        np.testing.assert_array_equal(r["outputs"][0], p.reshape(-1))
    assert srv.stats()["staging_fallbacks"] >= 1
    for _, _, _, t in reqs:
        G.lib.grass_server_release(srv._h, t)
    srv.close()
