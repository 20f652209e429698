"""GPU parity at R-MAT scale 20 (edge factor 16): the samplers and the decode
sweep through the C ABI against the CPU oracle, bit for bit, on a graph large
enough that every decode path runs (LE payloads in both layouts, GT long gap
runs, hub ranges split over warps).  Walkers 0..k-1 and seeds 0..k-1 draw the
same Philox streams in a full launch and in the oracle's run over those k
inputs, so a slice of a full-size launch is checked against the oracle."""
import os

import numpy as np
import pytest

import grass_b200 as G

pytestmark = pytest.mark.gpu

SCALE, EF = 20, 16


def _u32(t):
    return t.contiguous().cpu().numpy().view(np.uint32)


@pytest.fixture(scope="module")
def s20(tmp_path_factory, oracle_mod):
    import torch
    d = tmp_path_factory.mktemp("rmat_s20")
    rp, cols = G.rmat_graph(SCALE, EF, seed=42)
    out = {"torch": torch, "rowptr": rp, "cols": cols}
    for mode in ("LE", "GT"):
        prefix = str(d / mode)
        G.compress_to_files(rp, cols, mode, prefix)
        out[mode] = (G.Graph(prefix, mode), oracle_mod.OracleGraph(prefix))
    return out


@pytest.mark.parametrize("mode", ["LE", "GT"])
def test_rw_bit_exact_at_scale(s20, oracle_mod, mode):
    torch = s20["torch"]
    g, og = s20[mode]
    W, L, k = 1 << 20, 80, 65536
    starts = torch.empty(W, dtype=torch.int32, device="cuda")
    G.uniform_starts_device(g.n, W, 7, starts)
    paths = torch.empty(W * (L + 1), dtype=torch.int32, device="cuda")
    e = torch.zeros(1, dtype=torch.int64, device="cuda")
    g.rw_device(starts, W, L, 7, paths, e, layout=G.LAYOUT_STEP_MAJOR)
    torch.cuda.synchronize()
    st = _u32(starts[:k])
    np.testing.assert_array_equal(st, oracle_mod.uniform_starts(g.n, W, 7)[:k])
    ref, _ = og.rw(mode, st, L, 7)
    np.testing.assert_array_equal(_u32(paths.view(L + 1, W)[:, :k].T), ref)


@pytest.mark.parametrize("mode", ["LE", "GT"])
def test_khop_bit_exact_at_scale(s20, oracle_mod, mode):
    torch = s20["torch"]
    g, og = s20[mode]
    S, fan, k = 65536, (25, 10), 4096
    seeds = torch.empty(S, dtype=torch.int32, device="cuda")
    G.uniform_starts_device(g.n, S, 11, seeds)
    hops = [torch.empty(S * w, dtype=torch.int32, device="cuda") for w in G.hop_widths(fan)]
    g.khop_device(seeds, S, fan, 13, hops)
    torch.cuda.synchronize()
    refs, _ = og.khop(mode, _u32(seeds[:k]), fan, 13)
    for h, w in enumerate(G.hop_widths(fan)):
        np.testing.assert_array_equal(_u32(hops[h].view(S, w)[:k]), refs[h])


@pytest.mark.parametrize("mode", ["LE", "GT"])
def test_decode_sweep_bit_exact_at_scale(s20, mode):
    """Every neighbor list, against the graph the files were written from."""
    torch = s20["torch"]
    g, _ = s20[mode]
    rp, cols = s20["rowptr"], s20["cols"]
    rp_d = torch.empty(g.n + 1, dtype=torch.int64, device="cuda")
    cl_d = torch.empty(len(cols), dtype=torch.int32, device="cuda")
    for _ in range(2):  # the first sweep builds the plan, the second reuses it
        cl_d.fill_(-1)
        g.decode_all_device(rp_d, cl_d)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(rp_d.cpu().numpy().view(np.uint64), rp.astype(np.uint64))
        np.testing.assert_array_equal(_u32(cl_d), cols.astype(np.uint32))


@pytest.mark.parametrize("mode", ["LE", "GT"])
def test_batched_jobs_bit_exact_at_scale(s20, oracle_mod, mode):
    """A batched run of RW, k-hop and multi-RW jobs (every selection) against
    the oracle."""
    torch = s20["torch"]
    g, og = s20[mode]
    n = g.n
    rng = np.random.default_rng(3)
    b = G.Batch(g)
    checks = []
    alive = []  # the batch holds raw device pointers: keep every input alive

    def ints(a):
        t = torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).cuda()
        alive.append(t)
        return t

    for k, (W, L) in enumerate([(3000, 60), (40000, 12), (1, 100)]):
        st = rng.integers(0, n, W).astype(np.uint32)
        out = torch.empty(W * (L + 1), dtype=torch.int32, device="cuda")
        b.add_rw(ints(st), W, L, 50 + k, out)
        checks.append(("rw", st, (L, 50 + k), out))
    for k, fan in enumerate([(25, 10), (5, 5, 5), (15, 10)]):
        S = int(rng.integers(100, 3000))
        sd = rng.integers(0, n, S).astype(np.uint32)
        outs = [torch.empty(S * w, dtype=torch.int32, device="cuda") for w in G.hop_widths(fan)]
        b.add_khop(ints(sd), S, fan, 60 + k, outs)
        checks.append(("khop", sd, (fan, 60 + k), outs))
    for k, (R, T, sel) in enumerate([(2000, 10000, 2), (500, 3000, 1), (80, 100, 0)]):
        roots = oracle_mod.mrw_roots(n, 1, R, 70 + k)
        rt = ints(roots.ravel())
        src, dst = (torch.empty(T, dtype=torch.int32, device="cuda") for _ in range(2))
        b.add_mrw(rt, 1, R, T, 70 + k, src, dst, select=sel)
        checks.append(("mrw", roots, (T, 70 + k, sel), (src, dst, rt)))
    b.run()
    torch.cuda.synchronize()
    for kind, inp, prm, out in checks:
        if kind == "rw":
            ref, _ = og.rw(mode, inp, *prm)
            np.testing.assert_array_equal(_u32(out).reshape(len(inp), -1), ref)
        elif kind == "khop":
            refs, _ = og.khop(mode, inp, *prm)
            for o, r in zip(out, refs):
                np.testing.assert_array_equal(_u32(o).reshape(len(inp), -1), r)
        else:
            T, seed, sel = prm
            src, dst, fin, _ = og.mrw(mode, inp, T, seed, sel)
            np.testing.assert_array_equal(_u32(out[0]).reshape(1, -1), src)
            np.testing.assert_array_equal(_u32(out[1]).reshape(1, -1), dst)
            np.testing.assert_array_equal(_u32(out[2]).reshape(1, -1), fin)
    b.close()
