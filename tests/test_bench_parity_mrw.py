"""The bench's multi-RW parity check (bench.Parity.mrw) on CPU tensors: it
accepts outputs equal to the oracle's for the first k samples, and rejects an
output with one edge, or one final root, changed."""
import os
import sys

import numpy as np

from conftest import golden_graph

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def _case(oracle_mod, mode):
    import torch
    d, *_ = golden_graph("rmat_s10_e8")
    prefix = os.path.join(d, mode)
    og = oracle_mod.OracleGraph(prefix)
    S, R, T, seed = 40, 80, 100, 11
    roots0 = oracle_mod.mrw_roots(og.n, S, R, seed)
    src, dst, fin, _ = og.mrw(mode, roots0, T, seed, 0)
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a).reshape(-1).view(np.int32).copy())
    return prefix, t(roots0), t(src), t(dst), t(fin), R, T, seed


def test_equal_outputs_pass_and_changes_fail(oracle_mod):
    for mode in ("LE", "GT"):
        prefix, roots0, src, dst, fin, R, T, seed = _case(oracle_mod, mode)
        p = bench.Parity(True)
        p.mrw("ok", prefix, mode, roots0, R, T, seed, src, dst, fin, k=32)
        assert p.res["ok"]["ok"] and p.res["ok"]["samples"] == 32
        bad_dst = dst.clone()
        bad_dst[5 * T + 7] ^= 1
        p.mrw("dst", prefix, mode, roots0, R, T, seed, src, bad_dst, fin, k=32)
        assert not p.res["dst"]["ok"]
        bad_fin = fin.clone()
        bad_fin[31 * R + 79] ^= 1
        p.mrw("fin", prefix, mode, roots0, R, T, seed, src, dst, bad_fin, k=32)
        assert not p.res["fin"]["ok"]
        # a change beyond the first k samples is outside the checked slice
        late = dst.clone()
        late[35 * T] ^= 1
        p.mrw("late", prefix, mode, roots0, R, T, seed, src, late, fin, k=32)
        assert p.res["late"]["ok"]
