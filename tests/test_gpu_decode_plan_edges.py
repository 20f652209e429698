"""Decode sweep at the edges of its plan, on the GPU, against the input CSR.

The flat sweep cuts runs of consecutive vertices every 2048 neighbors and
splits vertices of degree >= 2048 into ranges of 2048; the staged sweep splits
vertices of degree >= 32 into ranges.  These graphs put vertices on and
around those boundaries: degrees 2047, 2048, 2049, 4096 and 4097 (an LE range
that starts at neighbor d - 1, which only the last slot's right rock holds),
long stretches of isolated vertices inside a run, runs that cross the
1024-vertex plan chunks, LE degree-1 vertices (the neighbor is in the record)
and degree-2 vertices."""
import functools

import numpy as np
import pytest

import grass_b200 as G

pytestmark = pytest.mark.gpu


def _csr(adj, n):
    rp = np.zeros(n + 1, dtype=np.uint64)
    for v, nb in adj.items():
        rp[v + 1] = len(nb)
    rp = np.cumsum(rp, dtype=np.uint64)
    cols = np.zeros(int(rp[-1]), dtype=np.uint32)
    for v, nb in adj.items():
        cols[int(rp[v]):int(rp[v + 1])] = np.sort(np.asarray(nb, dtype=np.uint32))
    return rp, cols


@functools.lru_cache(maxsize=None)
def _graph(seed):
    rng = np.random.default_rng(seed)
    n = 20000
    adj = {}
    # hubs on and around the range boundaries, scattered among the vertices
    for v, d in zip((5, 1500, 2600, 7000, 12000, 19990), (2047, 2048, 2049, 4096, 4097, 6145)):
        adj[v] = rng.choice(np.setdiff1d(np.arange(n), [v]), d, replace=False)
    # stretches of small vertices with isolated vertices in between
    for v in range(3000, 6000):
        if v % 7 == 0:
            continue  # isolated
        d = int(rng.integers(1, 40))
        adj[v] = rng.choice(np.setdiff1d(np.arange(n), [v]), d, replace=False)
    for v in range(8000, 8200):  # degree 1 and 2 only
        adj[v] = rng.choice(np.setdiff1d(np.arange(n), [v]), 1 + v % 2, replace=False)
    # one vertex of degree ~1000 every 300 vertices: runs cut inside plan chunks
    for v in range(13000, 19000, 300):
        adj[v] = rng.choice(np.setdiff1d(np.arange(n), [v]), 900 + v % 200, replace=False)
    adj[n - 1] = np.array([0, 1, 2])  # (trailing vertices with no neighbors would be trimmed)
    return _csr(adj, n)


@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("depth", [0, 1, 2])
def test_decode_plan_boundaries(mode, depth):
    rp, cols = _graph(11)
    gb, ob = G.compress(rp, cols, mode)
    g = G.Graph.from_bytes(gb, ob, mode)
    g.set_tuning(decode_stage_depth=depth)
    for _ in range(2):  # the plan is built by the first call and reused
        r, c = g.decode_all()
        np.testing.assert_array_equal(r[: len(rp)], rp)
        np.testing.assert_array_equal(c, cols)
        g.check_device_error()
