"""CPU tests: the oracle pinned against the reference's golden fixtures.

The fixtures under tests/golden were produced by the reference's own
compressor and checked against the reference's own bcg.cuh decoder
(tests/golden/make_golden.py).  When oracle/_ref is present (a machine with
the reference sources), the reference decoder is also run live here.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, GRAPHS, golden_graph
import pyref


def test_philox_known_answers(oracle_mod):
    kat = json.load(open(os.path.join(GOLDEN, "philox_kat.json")))
    assert len(kat["cases"]) >= 40
    for c in kat["cases"]:
        key = c["key"][0] | (c["key"][1] << 32)
        assert oracle_mod.philox(key, c["ctr"]).tolist() == c["out"], c


def test_philox_zero_block(oracle_mod):
    # Random123's published Philox4x32-10 answer for a zero key and counter.
    assert oracle_mod.philox(0, [0, 0, 0, 0]).tolist() == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C,
                                                           0x9B00DBD8]


@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_oracle_decode_matches_reference_files(oracle_mod, name, mode):
    d, rowptr, cols, meta = golden_graph(name)
    g = oracle_mod.OracleGraph(os.path.join(d, mode))
    assert g.n == meta[mode]["n"]
    assert g.n_file == meta[mode]["n_file"]
    assert g.ubl == meta[mode]["ubl"]
    rp, cl = g.decode_all(mode)
    np.testing.assert_array_equal(rp, rowptr)
    np.testing.assert_array_equal(cl, cols)
    # random access equals the sequential block decode
    rng = np.random.default_rng(1)
    verts = rng.integers(0, g.n, size=min(g.n, 300))
    for v in verts:
        dv = int(rowptr[v + 1] - rowptr[v])
        assert g.degree(mode, int(v)) == dv
        for i in rng.integers(0, max(dv, 1), size=min(dv, 8)):
            assert g.get_vertex(mode, int(v), int(i)) == cols[int(rowptr[v]) + int(i)]


def test_phantom_vertex_trimmed(oracle_mod):
    d, rowptr, cols, meta = golden_graph("tiny_path7")
    for mode in ("GT", "LE"):
        g = oracle_mod.OracleGraph(os.path.join(d, mode))
        assert g.n_file == 8 and g.n == 7


@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_reference_decoder_live(oracle_mod, name, mode):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    d, rowptr, cols, meta = golden_graph(name)
    g = oracle_mod.OracleGraph(os.path.join(d, mode))
    rp, cl = oracle_mod.ref_decode_all(mode, g.words(), g.offsets())
    np.testing.assert_array_equal(rp, rowptr)
    np.testing.assert_array_equal(cl, cols)
    ob = open(os.path.join(d, mode + ".offset"), "rb").read()
    lens = oracle_mod.ref_offset_lengths(mode, ob, g.n_file)
    np.testing.assert_array_equal(lens[: g.n], np.diff(g.offsets()))


def test_malformed_offset_rejected(oracle_mod):
    d, *_ = golden_graph("rmat_s10_e8")
    gb = open(os.path.join(d, "GT.graph"), "rb").read()
    ob = bytearray(open(os.path.join(d, "GT.offset"), "rb").read())
    with pytest.raises(ValueError):
        oracle_mod.OracleGraph(graph_bytes=gb[: len(gb) // 2], offset_bytes=bytes(ob))
    ob[0] = 0
    with pytest.raises(ValueError):
        oracle_mod.OracleGraph(graph_bytes=gb, offset_bytes=bytes(ob))


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_oracle_rw_matches_python_restatement(oracle_mod, mode):
    d, rowptr, cols, meta = golden_graph("edge_cases")
    g = oracle_mod.OracleGraph(os.path.join(d, mode))
    starts = np.concatenate([oracle_mod.uniform_starts(g.n, 60, 7),
                             np.array([g.n + 5, 0, g.n - 1], np.uint32)])
    paths, tot = g.rw(mode, starts, 12, 99)
    ref = pyref.rw(oracle_mod.philox, rowptr, cols, starts, 12, 99)
    np.testing.assert_array_equal(paths, ref)
    assert tot == int(((ref[:, 1:] != pyref.INVALID)).sum())
    # same walk over the plain CSR
    p2, t2 = oracle_mod.rw_csr(rowptr, cols, starts, 12, 99)
    np.testing.assert_array_equal(p2, paths)
    assert t2 == tot


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_oracle_khop_matches_python_restatement(oracle_mod, mode):
    d, rowptr, cols, meta = golden_graph("edge_cases")
    g = oracle_mod.OracleGraph(os.path.join(d, mode))
    seeds = np.concatenate([oracle_mod.uniform_starts(g.n, 20, 5), np.array([g.n + 1], np.uint32)])
    outs, tot = g.khop(mode, seeds, [3, 4, 2], 11)
    ref = pyref.khop(oracle_mod.philox, rowptr, cols, seeds, [3, 4, 2], 11)
    for a, b in zip(outs, ref):
        np.testing.assert_array_equal(a, b)
    assert tot == sum(int((o != pyref.INVALID).sum()) for o in ref)


@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("select", [0, 1, 2])
def test_oracle_mrw_matches_python_restatement(oracle_mod, mode, select):
    d, rowptr, cols, meta = golden_graph("edge_cases")
    g = oracle_mod.OracleGraph(os.path.join(d, mode))
    roots = oracle_mod.mrw_roots(g.n, 6, 9, 3)
    src, dst, fin, tot = g.mrw(mode, roots, 40, 21, select)
    rs, rd, rf = pyref.mrw(oracle_mod.philox, rowptr, cols, roots, 40, 21, select)
    np.testing.assert_array_equal(src, rs)
    np.testing.assert_array_equal(dst, rd)
    np.testing.assert_array_equal(fin, rf)



@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_oracle_edge_compaction_matches_loops(oracle_mod, mode):
    d, rowptr, cols, meta = golden_graph("edge_cases")
    g = oracle_mod.OracleGraph(os.path.join(d, mode))
    seeds = np.concatenate([oracle_mod.uniform_starts(g.n, 20, 5), np.array([g.n + 1], np.uint32)])
    outs, tot = g.khop(mode, seeds, [3, 4, 2], 11)
    s, t = oracle_mod.khop_edges(seeds, outs, [3, 4, 2])
    rs, rt = pyref.khop_edges(seeds, outs, [3, 4, 2])
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(t, rt)
    assert len(s) == tot
    starts = np.concatenate([oracle_mod.uniform_starts(g.n, 60, 7),
                             np.array([g.n + 5, 0, g.n - 1], np.uint32)])
    paths, tot = g.rw(mode, starts, 12, 99)
    s, t = oracle_mod.rw_edges(paths)
    rs, rt = pyref.rw_edges(paths)
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(t, rt)
    assert len(s) == tot
    # the step-major layout lists the same edges in (step, walk) order
    s2, t2 = oracle_mod.rw_edges(np.ascontiguousarray(paths.T), walk_major=False)
    assert sorted(zip(s2.tolist(), t2.tolist())) == sorted(zip(s.tolist(), t.tolist()))
    roots = oracle_mod.mrw_roots(g.n, 6, 9, 3)
    src, dst, fin, tot = g.mrw(mode, roots, 40, 21, 1)
    s, t = oracle_mod.mrw_edges(src, dst)
    assert len(s) == tot
    np.testing.assert_array_equal(t, dst[dst != pyref.INVALID])

def test_det_log(oracle_mod):
    """The oracle's logarithm equals the Python restatement bit for bit and
    math.log to within a few ulp, including the ends of (0, 1)."""
    import math
    rng = np.random.default_rng(3)
    us = list(rng.random(20000)) + [2.0 ** -52 * 0.5, 1 - 2.0 ** -53, 0.5, 0.7071067811865476,
                                    0.7071067811865475, 1e-300]
    for u in us:
        if not 0 < u < 1:
            continue
        a = oracle_mod.det_log(u)
        assert a == pyref.det_log(u), u
        assert abs(a - math.log(u)) <= 4e-16 * max(1.0, abs(math.log(u))), u


def test_mrw_ct_has_the_law_of_sequential_degree_selection(oracle_mod):
    """Continuous-time selection (2) and one-block-per-step selection (1) are
    two constructions of the same process: the final walker positions and the
    vertices visited at a fixed step have the same distribution (two-sample
    chi-square over degree bins, 20,000 samples each)."""
    from scipy import stats
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    g = oracle_mod.OracleGraph(os.path.join(d, "LE"))
    deg = np.diff(rowptr)
    S, R, T = 20000, 4, 24
    roots = np.tile(oracle_mod.mrw_roots(g.n, 1, R, 77), (S, 1))
    bins = np.unique(np.quantile(deg[deg > 0], np.linspace(0, 1, 13)))
    out = []
    for sel, seed in ((1, 5), (2, 6)):
        src, dst, fin, _ = g.mrw("LE", roots, T, seed, sel)
        out.append((np.digitize(deg[fin.ravel()], bins), np.digitize(deg[dst[:, T // 2]], bins),
                    (src[:, :T // 2] == roots[:, :1]).sum(1)))
    for a, b in zip(out[0], out[1]):
        ks = np.union1d(a, b)
        table = np.array([[np.sum(a == k) for k in ks], [np.sum(b == k) for k in ks]])
        table = table[:, table.sum(0) >= 10]
        pval = stats.chi2_contingency(table)[1]
        assert pval > 0.001, (pval, table)


def test_rw_visit_distribution_chi_square(oracle_mod):
    """Visit counts after t steps follow the exact propagated distribution of
    a uniform-neighbor walk -- the distribution the reference's
    DeepWalkApp::next samples (GT/src/apps/randomwalk/randomWalks.cu:49-81)."""
    from scipy import stats
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    g = oracle_mod.OracleGraph(os.path.join(d, "LE"))
    n = g.n
    W, T = 200_000, 6
    starts = oracle_mod.uniform_starts(n, W, 1234)
    paths, _ = g.rw("LE", starts, T, 4321)
    p = np.bincount(starts, minlength=n).astype(np.float64) / W
    deg = np.diff(rowptr).astype(np.float64)
    src = np.repeat(np.arange(n), np.diff(rowptr).astype(np.int64))
    for _ in range(T):
        q = np.zeros(n)
        np.add.at(q, cols, (p / np.maximum(deg, 1))[src])
        p = q
    obs = np.bincount(paths[:, T], minlength=n).astype(np.float64)
    exp = p * W
    keep = exp >= 5
    o, e = obs[keep], exp[keep]
    if (~keep).any():
        o = np.append(o, obs[~keep].sum())
        e = np.append(e, exp[~keep].sum())
    chi2 = ((o - e) ** 2 / e).sum()
    pval = 1 - stats.chi2.cdf(chi2, len(o) - 1)
    assert pval > 0.01, (chi2, len(o), pval)


def test_config1_oracle_rw_runs(oracle_mod):
    """Config 1 (R-MAT s16 ef16, 4096 walkers x 80) through the oracle on files
    written by the byte-identical writer."""
    import tempfile
    import grass_b200 as G
    rp, cols = G.rmat_graph(16, 16, seed=42)
    with tempfile.TemporaryDirectory() as t:
        for mode in ("GT", "LE"):
            G.compress_to_files(rp, cols, mode, os.path.join(t, mode))
            g = oracle_mod.OracleGraph(os.path.join(t, mode))
            starts = oracle_mod.uniform_starts(g.n, 4096, 7)
            paths, tot = g.rw(mode, starts, 80, 7)
            p2, t2 = oracle_mod.rw_csr(rp, cols, starts, 80, 7)
            np.testing.assert_array_equal(paths, p2)
            assert tot == 4096 * 80
