"""GPU tests of the second-order (node2vec) walk: bit-exact against the CPU
oracle on the golden graphs in both formats and both path layouts, the CSR
sampler identical to the compressed ones, and bad parameters refused."""
import os

import numpy as np
import pytest

from conftest import golden_graph
import grass_b200 as G

pytestmark = pytest.mark.gpu

PQ = [(1.0, 1.0, 0), (0.25, 4.0, 8), (4.0, 0.25, 64), (0.5, 2.0, 1)]


def _walk(torch, obj, starts, L, seed, p, q, tries, layout):
    W = len(starts)
    d_starts = torch.from_numpy(starts.view(np.int32)).cuda()
    paths = torch.empty(W * (L + 1), dtype=torch.int32, device="cuda")
    edges = torch.zeros(1, dtype=torch.int64, device="cuda")
    obj.node2vec_device(d_starts, W, L, seed, p, q, paths, edges, max_tries=tries, layout=layout)
    torch.cuda.synchronize()
    out = paths.cpu().numpy().view(np.uint32)
    shape = (W, L + 1) if layout == G.LAYOUT_WALK_MAJOR else (L + 1, W)
    out = out.reshape(shape)
    return (out if layout == G.LAYOUT_WALK_MAJOR else out.T), int(edges.item())


@pytest.mark.parametrize("name", ["rmat_s10_e8", "hub", "edge_cases"])
@pytest.mark.parametrize("mode", ["GT", "LE"])
@pytest.mark.parametrize("pq", PQ)
def test_node2vec_equals_oracle(oracle_mod, name, mode, pq):
    import torch
    p, q, tries = pq
    d, rowptr, cols, _ = golden_graph(name)
    g = G.Graph(os.path.join(d, mode), mode)
    og = oracle_mod.OracleGraph(os.path.join(d, mode))
    rng = np.random.default_rng(3)
    starts = rng.integers(0, g.n, 3000).astype(np.uint32)
    starts[:3] = [0, g.n - 1, 0xFFFFFFFF]  # an invalid start walks nowhere
    L, seed = 30, 1234
    exp, e_exp = og.node2vec(mode, starts, L, seed, p, q, max_tries=tries)
    for layout in (G.LAYOUT_WALK_MAJOR, G.LAYOUT_STEP_MAJOR):
        got, e_got = _walk(torch, g, starts, L, seed, p, q, tries, layout)
        np.testing.assert_array_equal(got, exp)
        assert e_got == e_exp
    g.check_device_error()
    # the uncompressed sampler draws the same walks
    csr = g.csr()
    got, e_got = _walk(torch, csr, starts, L, seed, p, q, tries, G.LAYOUT_WALK_MAJOR)
    np.testing.assert_array_equal(got, exp)
    assert e_got == e_exp
    csr.close()


def test_node2vec_bad_parameters():
    import torch
    d, *_ = golden_graph("tiny_path7")
    g = G.Graph(os.path.join(d, "LE"), "LE")
    s = torch.zeros(4, dtype=torch.int32, device="cuda")
    out = torch.empty(4 * 6, dtype=torch.int32, device="cuda")
    for p, q, tries in ((0.0, 1.0, 0), (1.0, -1.0, 0), (float("nan"), 1.0, 0),
                        (1.0, float("inf"), 0), (1.0, 1.0, 65537)):
        with pytest.raises(G.GrassError):
            g.node2vec_device(s, 4, 5, 1, p, q, out, max_tries=tries)
