"""GPU parity: samplers through the C ABI vs the CPU oracle, bit-exact.

Both consume the same Philox4x32-10 stream per (seed, walker, step), so paths,
k-hop frontiers and multi-RW edges must be identical; the CSR baseline must
produce the same walks as the compressed sampler.
"""
import os

import numpy as np
import pytest

from conftest import GRAPHS, golden_graph
import grass_b200 as G

pytestmark = pytest.mark.gpu


def _u32(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    assert torch.cuda.is_available()
    return torch


@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_rw_matches_oracle(oracle_mod, name, mode):
    d, rowptr, cols, meta = golden_graph(name)
    prefix = os.path.join(d, mode)
    g = G.Graph(prefix, mode)
    og = oracle_mod.OracleGraph(prefix)
    starts = np.concatenate([oracle_mod.uniform_starts(g.n, 3000, 7),
                             np.array([g.n, g.n + 100, 0, g.n - 1], np.uint32)])
    paths, e = g.rw(starts, 80, 7)
    ref, re_ = og.rw(mode, starts, 80, 7)
    np.testing.assert_array_equal(paths, ref)
    assert e == re_
    sm, e2 = g.rw(starts, 80, 7, layout=G.LAYOUT_STEP_MAJOR)
    np.testing.assert_array_equal(sm.T, ref)
    assert e2 == re_


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_rw_config1(oracle_mod, mode, tmp_path):
    """Config 1: R-MAT s16 ef16, 4096 uniform walkers x 80 steps, Philox seed 7."""
    rp, cols = G.rmat_graph(16, 16, seed=42)
    G.compress_to_files(rp, cols, mode, str(tmp_path / mode))
    g = G.Graph(str(tmp_path / mode), mode)
    og = oracle_mod.OracleGraph(str(tmp_path / mode))
    starts = oracle_mod.uniform_starts(g.n, 4096, 7)
    paths, e = g.rw(starts, 80, 7)
    ref, re_ = og.rw(mode, starts, 80, 7)
    np.testing.assert_array_equal(paths, ref)
    assert e == re_ == 4096 * 80


@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("layout", [G.LAYOUT_WALK_MAJOR, G.LAYOUT_STEP_MAJOR])
def test_rw_host_chunked_pipeline(oracle_mod, mode, layout):
    """grass_rw_host splits the walkers into 2^17-walker chunks on two streams;
    the walks must equal one launch (here: the oracle) with a ragged tail."""
    d, rowptr, cols, meta = golden_graph("hub")
    g = G.Graph(os.path.join(d, mode), mode)
    og = oracle_mod.OracleGraph(os.path.join(d, mode))
    W, L = 300_001, 12
    starts = oracle_mod.uniform_starts(g.n, W, 17)
    paths, e = g.rw(starts, L, 9, layout=layout)
    ref, re_ = og.rw(mode, starts, L, 9)
    if layout == G.LAYOUT_STEP_MAJOR:
        paths = paths.T
    np.testing.assert_array_equal(paths, ref)
    assert e == re_
    # a second call reuses the workspace
    paths2, e2 = g.rw(starts[:1000], L, 9, layout=layout)
    ref2 = ref[:1000]
    np.testing.assert_array_equal(paths2.T if layout == G.LAYOUT_STEP_MAJOR else paths2, ref2)


def test_device_starts_match_oracle(oracle_mod, torch_cuda):
    torch = torch_cuda
    out = torch.empty(10001, dtype=torch.int32, device="cuda")
    G.uniform_starts_device(46723, 10001, 7, out)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_u32(out), oracle_mod.uniform_starts(46723, 10001, 7))


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_csr_rw_equals_compressed_rw(oracle_mod, torch_cuda, mode):
    torch = torch_cuda
    d, rowptr, cols, meta = golden_graph("hub")
    g = G.Graph(os.path.join(d, mode), mode)
    c = g.csr()
    c2 = G.Csr.from_host(rowptr, cols)
    W, L = 5000, 40
    starts = torch.from_numpy(oracle_mod.uniform_starts(g.n, W, 3).view(np.int32)).cuda()
    outs = []
    for obj in (g, c, c2):
        p = torch.empty(W * (L + 1), dtype=torch.int32, device="cuda")
        e = torch.zeros(1, dtype=torch.int64, device="cuda")
        obj.rw_device(starts, W, L, 5, p, e)
        torch.cuda.synchronize()
        outs.append((_u32(p).reshape(W, L + 1), int(e.item())))
    for p, e in outs[1:]:
        np.testing.assert_array_equal(p, outs[0][0])
        assert e == outs[0][1]
    ref, re_ = oracle_mod.rw_csr(rowptr, cols, _u32(starts), L, 5)
    np.testing.assert_array_equal(outs[0][0], ref)


@pytest.mark.parametrize("name", ["edge_cases", "hub", "rmat_s10_e8"])
@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("fanouts", [(25, 10), (10, 25), (5, 5, 5), (40,)])
def test_khop_matches_oracle(oracle_mod, name, mode, fanouts):
    d, rowptr, cols, meta = golden_graph(name)
    prefix = os.path.join(d, mode)
    g = G.Graph(prefix, mode)
    og = oracle_mod.OracleGraph(prefix)
    seeds = np.concatenate([oracle_mod.uniform_starts(g.n, 700, 9), np.array([g.n + 3], np.uint32)])
    outs, e = g.khop(seeds, fanouts, 13)
    ref, re_ = og.khop(mode, seeds, fanouts, 13)
    for a, b in zip(outs, ref):
        np.testing.assert_array_equal(a, b)
    assert e == re_


def test_csr_khop_equals_compressed(oracle_mod, torch_cuda):
    torch = torch_cuda
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, "GT"), "GT")
    c = g.csr()
    S, fan = 1000, (25, 10)
    seeds = torch.from_numpy(oracle_mod.uniform_starts(g.n, S, 4).view(np.int32)).cuda()
    res = []
    for obj in (g, c):
        outs = [torch.empty(S * w, dtype=torch.int32, device="cuda") for w in G.hop_widths(fan)]
        e = torch.zeros(1, dtype=torch.int64, device="cuda")
        obj.khop_device(seeds, S, fan, 17, outs, e)
        torch.cuda.synchronize()
        res.append(([_u32(o) for o in outs], int(e.item())))
    for a, b in zip(res[0][0], res[1][0]):
        np.testing.assert_array_equal(a, b)
    assert res[0][1] == res[1][1] == S * 275


@pytest.mark.parametrize("name", ["edge_cases", "rmat_s10_e8"])
@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("select", [G.SELECT_UNIFORM, G.SELECT_DEGREE, G.SELECT_DEGREE_CT])
def test_mrw_matches_oracle(oracle_mod, name, mode, select):
    d, rowptr, cols, meta = golden_graph(name)
    prefix = os.path.join(d, mode)
    g = G.Graph(prefix, mode)
    og = oracle_mod.OracleGraph(prefix)
    # the reference's shape: 80 roots, 100 steps
    roots = oracle_mod.mrw_roots(g.n, 64, 80, 5)
    src, dst, fin, e = g.mrw(roots, 100, 19, select)
    rs, rd, rf, re_ = og.mrw(mode, roots, 100, 19, select)
    np.testing.assert_array_equal(src, rs)
    np.testing.assert_array_equal(dst, rd)
    np.testing.assert_array_equal(fin, rf)
    assert e == re_


@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("select,S,R,T", [
    (G.SELECT_DEGREE, 3, 2000, 2000),     # warp per sample, sequential steps
    (G.SELECT_DEGREE_CT, 3, 2000, 2000),  # block per sample, walkers in parallel
    (G.SELECT_DEGREE_CT, 1, 2000, 10000), # the batched-jobs shape
    (G.SELECT_DEGREE_CT, 2, 5000, 700),   # more walkers than threads x 2
    (G.SELECT_DEGREE_CT, 5, 1, 300),      # a single walker
    (G.SELECT_UNIFORM, 2, 2000, 10000),   # block per sample
    (G.SELECT_UNIFORM, 1500, 8, 50),      # many samples: warp kernel
])
def test_mrw_large_frontier(oracle_mod, mode, select, S, R, T):
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    prefix = os.path.join(d, mode)
    g = G.Graph(prefix, mode)
    og = oracle_mod.OracleGraph(prefix)
    roots = oracle_mod.mrw_roots(g.n, S, R, 8)
    src, dst, fin, e = g.mrw(roots, T, 23, select)
    rs, rd, rf, re_ = og.mrw(mode, roots, T, 23, select)
    np.testing.assert_array_equal(src, rs)
    np.testing.assert_array_equal(dst, rd)
    np.testing.assert_array_equal(fin, rf)
    assert e == re_
    ok = rd != G.INVALID  # every move is an edge
    nb = [set(cols[rowptr[v]:rowptr[v + 1]].tolist()) for v in range(len(rowptr) - 1)]
    assert all(int(b) in nb[int(a)] for a, b in zip(rs[ok][:2000], rd[ok][:2000]))


def test_rw_paths_are_edges_at_scale(torch_cuda):
    """Size-independent property at R-MAT scale 20: every step of every walk
    is an edge of the graph and every walker takes every step."""
    torch = torch_cuda
    rp, cols = G.rmat_graph(20, 16, seed=42)
    gb, ob = G.compress(rp, cols, "LE")
    g = G.Graph.from_bytes(gb, ob, "LE")
    W, L = 200_000, 20
    starts = torch.empty(W, dtype=torch.int32, device="cuda")
    G.uniform_starts_device(g.n, W, 1, starts)
    paths = torch.empty(W * (L + 1), dtype=torch.int32, device="cuda")
    e = torch.zeros(1, dtype=torch.int64, device="cuda")
    g.rw_device(starts, W, L, 2, paths, e)
    torch.cuda.synchronize()
    assert int(e.item()) == W * L
    P = _u32(paths).reshape(W, L + 1).astype(np.int64)
    u, v = P[:, :-1].ravel(), P[:, 1:].ravel()
    keys = u * (1 << 32) + v
    src = np.repeat(np.arange(len(rp) - 1, dtype=np.int64), np.diff(rp).astype(np.int64))
    edges = src * (1 << 32) + cols.astype(np.int64)
    assert np.isin(keys, edges, assume_unique=False).all()


def test_random_read_probe_counts_every_read(torch_cuda):
    """The random-read probe (the bench's random-access ceiling) reads what it
    claims: over a buffer of ones the sink equals the number of reads."""
    torch = torch_cuda
    n = 1 << 20
    buf = torch.ones(n, dtype=torch.int32, device="cuda")
    sink = torch.zeros(1, dtype=torch.int64, device="cuda")
    k = G.random_read_probe(buf, n, 1 << 22, 9, sink)
    torch.cuda.synchronize()
    assert k >= 1 << 22 and int(sink.item()) == k
    with pytest.raises(G.GrassError):
        G.random_read_probe(buf, n - 1, 1 << 10, 9, sink)
