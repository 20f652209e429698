"""CPU tests of the oracle's second-order (node2vec) walk, the checker of the
GPU kernels: its stream layout, its acceptance rule and its bias."""
import os

import numpy as np
import pytest

from conftest import golden_graph

TAG_N2V = 0x4E320000


def _csr(name):
    d, rowptr, cols, _ = golden_graph(name)
    return d, np.asarray(rowptr, dtype=np.int64), np.asarray(cols, dtype=np.int64)


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_unbiased_walk_takes_each_first_candidate(oracle_mod, mode):
    # p = q = 1: every threshold is 2^32, so try 0 of every step is taken and
    # step s of walker w is N(v)[(word 0 of Philox(seed; s, w, 0, tag)) * d >> 32]
    d, rp, cols = _csr("rmat_s10_e8")
    g = oracle_mod.OracleGraph(os.path.join(d, mode))
    starts = np.arange(0, g.n, 7, dtype=np.uint32)
    L, seed = 12, 99
    paths, tot = g.node2vec(mode, starts, L, seed, 1.0, 1.0)
    edges = 0
    for w, s0 in enumerate(starts):
        v = int(s0)
        assert paths[w, 0] == v
        for s in range(L):
            deg = rp[v + 1] - rp[v] if v < g.n else 0
            if v >= g.n or deg == 0:
                v = 0xFFFFFFFF
            else:
                r = int(oracle_mod.philox(seed, [s, w, 0, TAG_N2V])[0])
                v = int(cols[rp[v] + ((r * deg) >> 32)])
                edges += 1
            assert paths[w, s + 1] == v, (w, s)
    assert tot == edges


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_return_and_outward_bias(oracle_mod, mode):
    # small p: walks return to the previous vertex; small q: they move on
    d, rp, cols = _csr("rmat_s10_e8")
    g = oracle_mod.OracleGraph(os.path.join(d, mode))
    starts = np.repeat(np.arange(g.n, dtype=np.uint32), 4)
    L = 20

    def returns(p, q):
        paths, _ = g.node2vec(mode, starts, L, 5, p, q)
        a, b = paths[:, 2:], paths[:, :-2]
        ok = a != 0xFFFFFFFF
        return float((a[ok] == b[ok]).mean())

    # (a return candidate is drawn with probability 1/d per try, so even a
    # strong return bias leaves many steps outward on vertices of high degree)
    back, uniform, out = returns(0.05, 1.0), returns(1.0, 1.0), returns(1.0, 0.05)
    assert back > 4 * uniform
    assert out < 0.5 * uniform


def test_max_tries_one_is_first_order(oracle_mod):
    # one candidate per step: the acceptance draw never matters
    d, rp, cols = _csr("rmat_s10_e8")
    g = oracle_mod.OracleGraph(os.path.join(d, "LE"))
    starts = np.arange(g.n, dtype=np.uint32)
    a, ta = g.node2vec("LE", starts, 15, 3, 0.1, 7.0, max_tries=1)
    b, tb = g.node2vec("LE", starts, 15, 3, 1.0, 1.0, max_tries=1)
    np.testing.assert_array_equal(a, b)
    assert ta == tb
