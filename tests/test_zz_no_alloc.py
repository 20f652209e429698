"""GPU test of grass_decode_all_noalloc, the decode entry point that allocates
no device memory.

It exists for callers that cannot allocate when they decode (an application
that has reserved the whole device for its own memory pool, or a loop that
must not pay for allocator calls).  Its output must equal grass_decode_all's
exactly -- decoded ids are integers -- on two calls in a row, since the
shared scratch array keeps the previous call's contents.  This file sorts
last so that a run stopping at the first failure has run every other test.
"""
import ctypes as C
import os

import numpy as np
import pytest

from conftest import golden_graph
import grass_b200 as G

pytestmark = pytest.mark.gpu


def _decode(fn, g):
    import torch
    info = g.info()
    n, E = int(info["n"]), int(info["num_edges"])
    rp = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    cl = torch.empty(max(E, 1), dtype=torch.int32, device="cuda")
    rc = fn(g.handle, C.c_void_p(rp.data_ptr()), C.c_void_p(cl.data_ptr()), None)
    assert rc == G.OK, G.last_error()
    torch.cuda.synchronize()
    return rp.cpu().numpy().view(np.uint64).copy(), cl.cpu().numpy().view(np.uint32)[:E].copy()


def _check(g, cols=None):
    # before any grass_decode_all the graph has no decode plan: the unplanned sweep
    before = [_decode(G.lib.grass_decode_all_noalloc, g) for _ in range(2)]
    ref = _decode(G.lib.grass_decode_all, g)  # builds the plan
    # two calls in a row on the shared scratch, now through the planned sweep
    after = [_decode(G.lib.grass_decode_all_noalloc, g) for _ in range(2)]
    for got in before + after:
        np.testing.assert_array_equal(got[0], ref[0])
        np.testing.assert_array_equal(got[1], ref[1])
    if cols is not None:
        np.testing.assert_array_equal(ref[1], cols)


@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("name", ["tiny_path7", "hub", "rmat_s10_e8"])
def test_noalloc_decode_equals_decode_all(mode, name):
    d, rowptr, cols, meta = golden_graph(name)
    _check(G.Graph(os.path.join(d, mode), mode), cols)


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_noalloc_decode_many_tiles(mode):
    # R-MAT scale 17: tens of 4096-vertex scan tiles in the scratch array
    rp, cols = G.rmat_graph(17, 8, seed=42)
    gb, ob = G.compress(rp, cols, mode)
    _check(G.Graph.from_bytes(gb, ob, mode), cols)
