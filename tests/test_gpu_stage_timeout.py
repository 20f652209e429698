"""Bounded device waits: the decode sweep's staged-copy wait runs out, the
warp reports GRASS_E_TIMEOUT through the graph's error word and decodes its
slots from global memory instead, and the context stays usable.

The wait is made to run out without a GPU fault: the test build of the
library (grass_b200/lib/libgrass_b200_stagetest.so, GRASS_STAGE_NEVER_COPY)
arms the barrier for a copy it never issues -- a phase that nothing
completes, with nothing in flight -- and polls only 4096 times."""
import ctypes as C
import os

import numpy as np
import pytest

import grass_b200 as G

pytestmark = pytest.mark.gpu

TEST_LIB = os.path.join(os.path.dirname(G.LIB_PATH), "libgrass_b200_stagetest.so")


def test_staged_wait_runs_out_and_is_reported(tmp_path):
    import torch
    lib = C.CDLL(TEST_LIB)  # a second, independent copy of the library
    P = C.c_void_p
    for name, args in {"grass_open": [C.c_char_p, C.c_int, C.c_int, C.POINTER(P)],
                       "grass_decode_all": [P, P, P, P],
                       "grass_check_device_error": [P, P], "grass_close": [P],
                       "grass_set_tuning": [P, P],
                       "grass_rw": [P, P, P, C.c_uint64, P, P, P]}.items():
        getattr(lib, name).argtypes = args
        getattr(lib, name).restype = C.c_int
    # R-MAT scale 16: its vertices of degree >= 32 are decoded by the range
    # sweep, which stages their slots
    rp, cols = G.rmat_graph(16, 16, seed=42)
    G.compress_to_files(rp, cols, "LE", str(tmp_path / "LE"))
    g = P()
    assert lib.grass_open(str(tmp_path / "LE").encode(), G.MODE_LE, 0, C.byref(g)) == G.OK
    tune = G.Tuning(decode_stage_depth=2)  # the range sweep stages its slots
    assert lib.grass_set_tuning(g, C.cast(C.byref(tune), P)) == G.OK
    n, E = len(rp) - 1, len(cols)
    rp_d = torch.empty(n + 1, dtype=torch.int64, device="cuda")
    cl_d = torch.empty(E, dtype=torch.int32, device="cuda")
    for _ in range(2):
        cl_d.fill_(-1)
        assert lib.grass_decode_all(g, P(rp_d.data_ptr()), P(cl_d.data_ptr()), None) == G.OK
        assert lib.grass_check_device_error(g, None) == G.E_TIMEOUT
        assert lib.grass_check_device_error(g, None) == G.OK  # read and cleared
        np.testing.assert_array_equal(rp_d.cpu().numpy().view(np.uint64), rp.astype(np.uint64))
        np.testing.assert_array_equal(cl_d.cpu().numpy().view(np.uint32), cols)
    # the context is still usable: a walk on the same graph
    W, L = 4096, 20
    starts = torch.randint(0, n, (W,), dtype=torch.int32, device="cuda")
    paths = torch.empty(W * (L + 1), dtype=torch.int32, device="cuda")
    prm = G.RwParams(L, G.LAYOUT_WALK_MAJOR, 5)
    assert lib.grass_rw(g, C.byref(prm), P(starts.data_ptr()), W, P(paths.data_ptr()), None,
                        None) == G.OK
    assert lib.grass_check_device_error(g, None) == G.OK
    torch.cuda.synchronize()
    ref = G.Graph(str(tmp_path / "LE"), "LE")
    exp = torch.empty_like(paths)
    ref.rw_device(starts, W, L, 5, exp)
    torch.cuda.synchronize()
    assert torch.equal(paths, exp)
    assert lib.grass_close(g) == G.OK


@pytest.mark.parametrize("mode", ["LE", "GT"])
@pytest.mark.parametrize("depth", [0, 1, 2, 4])
def test_library_decode_staged_reports_no_error(mode, depth):
    """The shipped library, slots staged or not: the same CSR, no error."""
    rp, cols = G.rmat_graph(16, 16, seed=42)
    gb, ob = G.compress(rp, cols, mode)
    g = G.Graph.from_bytes(gb, ob, mode)
    g.set_tuning(decode_stage_depth=depth)
    for _ in range(2):
        r, c = g.decode_all()
        np.testing.assert_array_equal(r, rp.astype(np.uint64))
        np.testing.assert_array_equal(c, cols)
        g.check_device_error()
