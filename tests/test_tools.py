"""CPU tests: host graph tools (generator, graph_sort, GT/LE writer) against
the reference's own outputs."""
import hashlib
import json
import os
import tempfile

import numpy as np
import pytest

from conftest import GOLDEN, GRAPHS, golden_graph
import grass_b200 as G


@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_writer_byte_identical_to_reference(name, mode):
    d, rowptr, cols, meta = golden_graph(name)
    gb, ob = G.compress(rowptr, cols, mode)
    assert gb == open(os.path.join(d, mode + ".graph"), "rb").read()
    assert ob == open(os.path.join(d, mode + ".offset"), "rb").read()


def test_graph_sort_matches_reference_rmat():
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    src, dst = G.gen_rmat(10, 8, seed=42)
    rp, cl = G.graph_sort(src, dst)
    np.testing.assert_array_equal(rp, rowptr)
    np.testing.assert_array_equal(cl, cols)


def test_config1_pipeline_hashes():
    """R-MAT s16/ef16 through graph_sort + both writers reproduces, byte for
    byte, the files the reference's graph_sort + compressor produced."""
    ref = json.load(open(os.path.join(GOLDEN, "config1_sha256.json")))
    rp, cols = G.rmat_graph(16, 16, seed=42)
    assert len(rp) - 1 == ref["n"]
    assert len(cols) == ref["num_edges"]
    for mode in ("GT", "LE"):
        gb, ob = G.compress(rp, cols, mode)
        assert len(gb) == ref[f"{mode}.graph"]["bytes"]
        assert hashlib.sha256(gb).hexdigest() == ref[f"{mode}.graph"]["sha256"]
        assert hashlib.sha256(ob).hexdigest() == ref[f"{mode}.offset"]["sha256"]


def test_graph_sort_semantics_small():
    # self-loops dropped before relabelling, duplicates removed, symmetric
    src = np.array([10, 10, 20, 20, 30, 10, 5], np.uint32)
    dst = np.array([20, 10, 10, 30, 20, 20, 5], np.uint32)
    rp, cl = G.graph_sort(src, dst)
    # first appearance: 10->0, 20->1, 30->2 (5 only in a self-loop: dropped)
    assert len(rp) == 4
    assert cl.tolist() == [1, 0, 2, 1]
    rp2, cl2 = G.graph_sort(src, dst, directed=True)
    # directed: (0,1) (1,0) (1,2) (2,1) (0,1) -> deduped, no mirroring
    assert rp2.tolist() == [0, 1, 3, 4]
    assert cl2.tolist() == [1, 0, 2, 1]
    src3 = np.array([1, 2], np.uint32)
    dst3 = np.array([2, 3], np.uint32)
    rp3, cl3 = G.graph_sort(src3, dst3, directed=True)
    assert rp3.tolist() == [0, 1, 2, 2] and cl3.tolist() == [1, 2]


def test_writer_rejects_unsorted_rows():
    rp = np.array([0, 2, 2], np.uint64)
    cols = np.array([1, 0], np.uint32)
    with pytest.raises(G.GrassError) as e:
        G.compress(rp, cols, "GT")
    assert e.value.code == G.E_ARG


def test_large_ids_round_trip(oracle_mod):
    """Vertex ids above 2^24 (long gamma codes, wide rocks/heads)."""
    n = (1 << 24) + 40
    rows = {0: [1, 1 << 23, n - 1], 7: [3, 9], n - 1: [0, 5, (1 << 24) + 1],
            (1 << 24) + 1: [2, n - 1]}
    rp = np.zeros(n + 1, np.uint64)
    for v, nb in rows.items():
        rp[v + 1] = len(nb)
    rp = np.cumsum(rp).astype(np.uint64)
    cols = np.concatenate([np.array(rows[v], np.uint32) for v in sorted(rows)])
    with tempfile.TemporaryDirectory() as t:
        for mode in ("GT", "LE"):
            G.compress_to_files(rp, cols, mode, os.path.join(t, mode))
            g = oracle_mod.OracleGraph(os.path.join(t, mode))
            assert g.n == n
            for v, nb in rows.items():
                assert g.degree(mode, v) == len(nb)
                assert [g.get_vertex(mode, v, i) for i in range(len(nb))] == nb


def test_rmat_generator_deterministic():
    a = G.gen_rmat(12, 4, seed=42)
    b = G.gen_rmat(12, 4, seed=42)
    c = G.gen_rmat(12, 4, seed=43)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert not np.array_equal(a[0], c[0])
    assert a[0].max() < (1 << 12)
    # quadrant probabilities: the top bit of (u, v) is (0,0) with p = .57
    top = ((a[0] >> 11) & 1) * 2 + ((a[1] >> 11) & 1)
    frac = np.bincount(top, minlength=4) / len(top)
    np.testing.assert_allclose(frac, [0.57, 0.19, 0.19, 0.05], atol=0.01)


def test_chung_lu_degree_cap():
    src, dst = G.gen_chung_lu(20000, 2.1, 30, 2000, m=300000, seed=42)
    deg = np.bincount(np.concatenate([src, dst]), minlength=20000)
    assert deg.max() < 4000
    assert abs(deg.mean() - 30) < 1.0
