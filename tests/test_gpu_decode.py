"""GPU parity: loading and decoding through the C ABI vs the reference's files.

Every neighbor list decoded on the B200 must equal the adjacency the reference
compressor encoded (and the reference's own decoder reproduced when the
fixtures were made), for every vertex, in both formats.
"""
import os
import tempfile

import numpy as np
import pytest

from conftest import GRAPHS, golden_graph
import grass_b200 as G

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", GRAPHS)
@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_open_and_decode_golden(name, mode):
    d, rowptr, cols, meta = golden_graph(name)
    g = G.Graph(os.path.join(d, mode), mode)
    info = g.info()
    assert info["n"] == meta[mode]["n"]
    assert info["n_file"] == meta[mode]["n_file"]
    assert info["ubl"] == meta[mode]["ubl"]
    assert info["num_edges"] == meta[mode]["num_edges"]
    assert info["max_degree"] == int(np.diff(rowptr).max())
    rp, cl = g.decode_all()
    np.testing.assert_array_equal(rp, rowptr)
    np.testing.assert_array_equal(cl, cols)


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_open_mem_equals_open_file(mode):
    d, rowptr, cols, meta = golden_graph("hub")
    gb = open(os.path.join(d, mode + ".graph"), "rb").read()
    ob = open(os.path.join(d, mode + ".offset"), "rb").read()
    g = G.Graph.from_bytes(gb, ob, mode)
    rp, cl = g.decode_all()
    np.testing.assert_array_equal(cl, cols)


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_degrees(mode):
    import torch
    d, rowptr, cols, meta = golden_graph("edge_cases")
    g = G.Graph(os.path.join(d, mode), mode)
    deg = torch.empty(g.n, dtype=torch.int32, device="cuda")
    g.degrees_device(deg)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(deg.cpu().numpy(), np.diff(rowptr).astype(np.int32))


def test_corrupt_and_mismatched_files_rejected():
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    gb = open(os.path.join(d, "GT.graph"), "rb").read()
    ob = open(os.path.join(d, "GT.offset"), "rb").read()
    # truncated stream: lengths sum past the end
    with pytest.raises(G.GrassError) as e:
        G.Graph.from_bytes(gb[: len(gb) // 2], ob, "GT")
    assert e.value.code == G.E_FORMAT
    # damaged header of vertex 0
    bad = bytearray(gb)
    bad[0] ^= 0xFF
    with pytest.raises(G.GrassError) as e:
        G.Graph.from_bytes(bytes(bad), ob, "GT")
    assert e.value.code == G.E_FORMAT
    # a GT file opened as LE
    with pytest.raises(G.GrassError) as e:
        G.Graph.from_bytes(gb, ob, "LE")
    assert e.value.code == G.E_FORMAT
    # the library still works afterwards
    g = G.Graph.from_bytes(gb, ob, "GT")
    assert g.decode_all()[1].tolist() == cols.tolist()


@pytest.mark.parametrize("scale,ef", [(16, 16), (19, 16)])
def test_decode_round_trip_generated(scale, ef):
    """decode(compress(graph_sort(R-MAT))) == graph_sort(R-MAT) at larger sizes."""
    rp, cols = G.rmat_graph(scale, ef, seed=42)
    for mode in ("GT", "LE"):
        gb, ob = G.compress(rp, cols, mode)
        g = G.Graph.from_bytes(gb, ob, mode)
        assert g.info()["num_edges"] == len(cols)
        r2, c2 = g.decode_all()
        np.testing.assert_array_equal(r2, rp)
        np.testing.assert_array_equal(c2, cols)
        g.close()


def test_csr_from_graph_matches():
    import torch
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, "LE"), "LE")
    c = g.csr()
    assert c.info()["nnz"] == len(cols)
    assert c.info()["device_bytes"] == (len(rowptr)) * 8 + len(cols) * 4
