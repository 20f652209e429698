"""GPU parity: output compaction through the C ABI vs the oracle's.

The samplers' fixed-shape outputs (k-hop frontiers, walk paths, multi-RW step
edges) are compacted on the device to (src, dst) edge lists; the oracle keeps
the entries whose dst is not INVALID_VERTEX, in output order.  Both must agree
exactly, and the number of edges must equal the sampler's own edge count.
"""
import os

import numpy as np
import pytest

from conftest import golden_graph
import grass_b200 as G

pytestmark = pytest.mark.gpu


def _u32(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


def _compact(torch, call, cap):
    """Runs call(src, dst, cap, count) on sentinel-filled buffers; returns the
    written prefix, the reported count and the untouched tail."""
    src = torch.full((max(cap, 1) + 64,), -7, dtype=torch.int32, device="cuda")
    dst = torch.full_like(src, -7)
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    call(src, dst, cap, cnt)
    torch.cuda.synchronize()
    n = int(cnt.item())
    k = min(n, cap)
    s, d = _u32(src), _u32(dst)
    return s[:k], d[:k], n, (s[k:], d[k:])


def _device(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint32).view(np.int32)).cuda()


@pytest.mark.parametrize("name", ["edge_cases", "hub", "rmat_s10_e8"])
@pytest.mark.parametrize("fanouts", [(25, 10), (5, 5, 5), (40,), (5000,)])
def test_khop_edges_match_oracle(oracle_mod, torch_cuda, name, fanouts):
    torch = torch_cuda
    d, rowptr, cols, meta = golden_graph(name)
    g = G.Graph(os.path.join(d, "LE"), "LE")
    S = 3 if fanouts == (5000,) else 700
    seeds = np.concatenate([oracle_mod.uniform_starts(g.n, S, 9), np.array([g.n + 3], np.uint32)])
    S = len(seeds)
    ds = _device(torch, seeds)
    outs = [torch.empty(S * w, dtype=torch.int32, device="cuda") for w in G.hop_widths(fanouts)]
    e = torch.zeros(1, dtype=torch.int64, device="cuda")
    g.khop_device(ds, S, fanouts, 13, outs, e)
    torch.cuda.synchronize()
    host = [_u32(o).reshape(S, -1) for o in outs]
    rs, rd = oracle_mod.khop_edges(seeds, host, fanouts)
    total = sum(S * w for w in G.hop_widths(fanouts))
    s, t, n, _ = _compact(torch, lambda a, b, c, k: G.khop_edges_device(
        ds, S, fanouts, outs, a, b, c, k), total)
    assert n == len(rs) == int(e.item())
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(t, rd)


@pytest.mark.parametrize("layout", [G.LAYOUT_WALK_MAJOR, G.LAYOUT_STEP_MAJOR])
@pytest.mark.parametrize("W,L", [(3000, 80), (7, 5000), (4096, 1), (1, 4095)])
def test_rw_edges_match_oracle(oracle_mod, torch_cuda, layout, W, L):
    torch = torch_cuda
    d, rowptr, cols, meta = golden_graph("edge_cases")
    g = G.Graph(os.path.join(d, "GT"), "GT")
    starts = oracle_mod.uniform_starts(g.n, W, 7)
    if W > 1:
        starts[0] = g.n + 100  # an invalid start: no edges at all
    ds = _device(torch, starts)
    paths = torch.empty(W * (L + 1), dtype=torch.int32, device="cuda")
    e = torch.zeros(1, dtype=torch.int64, device="cuda")
    g.rw_device(ds, W, L, 7, paths, e, layout=layout)
    torch.cuda.synchronize()
    hp = _u32(paths)
    hp = hp.reshape(W, L + 1) if layout == G.LAYOUT_WALK_MAJOR else hp.reshape(L + 1, W)
    rs, rd = oracle_mod.rw_edges(hp, walk_major=layout == G.LAYOUT_WALK_MAJOR)
    s, t, n, _ = _compact(torch, lambda a, b, c, k: G.rw_edges_device(
        paths, W, L, a, b, c, k, layout=layout), W * L)
    assert n == len(rs) == int(e.item())
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(t, rd)


@pytest.mark.parametrize("select", [G.SELECT_UNIFORM, G.SELECT_DEGREE, G.SELECT_DEGREE_CT])
def test_mrw_edges_match_oracle(oracle_mod, torch_cuda, select):
    torch = torch_cuda
    d, rowptr, cols, meta = golden_graph("edge_cases")
    g = G.Graph(os.path.join(d, "LE"), "LE")
    roots = oracle_mod.mrw_roots(g.n, 64, 80, 5)
    src, dst, fin, e = g.mrw(roots, 100, 19, select)
    rs, rd = oracle_mod.mrw_edges(src, dst)
    s, t, n, _ = _compact(torch, lambda a, b, c, k: G.mrw_edges_device(
        _device(torch, src), _device(torch, dst), 64, 100, a, b, c, k), 64 * 100)
    assert n == len(rs) == e
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(t, rd)


def test_capacity_truncates_and_counts_all(oracle_mod, torch_cuda):
    torch = torch_cuda
    d, rowptr, cols, meta = golden_graph("hub")
    g = G.Graph(os.path.join(d, "GT"), "GT")
    S, fan = 900, (25, 10)
    seeds = oracle_mod.uniform_starts(g.n, S, 4)
    ds = _device(torch, seeds)
    outs = [torch.empty(S * w, dtype=torch.int32, device="cuda") for w in G.hop_widths(fan)]
    g.khop_device(ds, S, fan, 17, outs)
    torch.cuda.synchronize()
    rs, rd = oracle_mod.khop_edges(seeds, [_u32(o).reshape(S, -1) for o in outs], fan)
    for cap in (0, 1, 4095, 4097, 12345, len(rs) - 1):
        s, t, n, (ts, td) = _compact(torch, lambda a, b, c, k: G.khop_edges_device(
            ds, S, fan, outs, a, b, c, k), cap)
        assert n == len(rs)
        np.testing.assert_array_equal(s, rs[:cap])
        np.testing.assert_array_equal(t, rd[:cap])
        assert (ts == np.uint32(0xFFFFFFF9)).all() and (td == np.uint32(0xFFFFFFF9)).all()


def test_empty_inputs(torch_cuda):
    torch = torch_cuda
    cnt = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    G.khop_edges_device(None, 0, (25, 10), [None, None], None, None, 0, cnt)
    torch.cuda.synchronize()
    assert int(cnt.item()) == 0
    cnt.fill_(-1)
    G.rw_edges_device(None, 0, 80, None, None, 0, cnt)
    torch.cuda.synchronize()
    assert int(cnt.item()) == 0
    paths = torch.zeros(16, dtype=torch.int32, device="cuda")
    cnt.fill_(-1)
    G.rw_edges_device(paths, 16, 0, None, None, 0, cnt)  # zero-length walks
    torch.cuda.synchronize()
    assert int(cnt.item()) == 0
    with pytest.raises(G.GrassError):
        G.rw_edges_device(paths, 16, 0, None, None, 0, None)
    with pytest.raises(G.GrassError):
        G.rw_edges_device(paths, 8, 1, None, None, 4, cnt)


def test_khop_edges_at_scale(oracle_mod, torch_cuda):
    """Size-independent property on R-MAT scale 18 with 65,536 seeds: the
    compacted list equals the oracle's compaction of the same frontiers and
    every edge is an edge of the graph."""
    torch = torch_cuda
    rp, cols = G.rmat_graph(18, 16, seed=42)
    gb, ob = G.compress(rp, cols, "LE")
    g = G.Graph.from_bytes(gb, ob, "LE")
    S, fan = 65536, (25, 10)
    seeds = oracle_mod.uniform_starts(g.n, S, 3)
    ds = _device(torch, seeds)
    outs = [torch.empty(S * w, dtype=torch.int32, device="cuda") for w in G.hop_widths(fan)]
    e = torch.zeros(1, dtype=torch.int64, device="cuda")
    g.khop_device(ds, S, fan, 5, outs, e)
    torch.cuda.synchronize()
    rs, rd = oracle_mod.khop_edges(seeds, [_u32(o).reshape(S, -1) for o in outs], fan)
    s, t, n, _ = _compact(torch, lambda a, b, c, k: G.khop_edges_device(
        ds, S, fan, outs, a, b, c, k), S * 275)
    assert n == len(rs) == int(e.item())
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(t, rd)
    key = s.astype(np.uint64) << np.uint64(32) | t.astype(np.uint64)
    edges = np.repeat(np.arange(len(rp) - 1, dtype=np.uint64), np.diff(rp).astype(np.int64))
    gkey = np.sort(edges << np.uint64(32) | cols.astype(np.uint64))
    pos = np.minimum(np.searchsorted(gkey, key), len(gkey) - 1)
    assert (gkey[pos] == key).all()
