"""GPU parity of the batched persistent launch: every job of a mixed batch must
produce exactly what the standalone call with the same parameters produces
(which is itself bit-exact against the oracle), on every replay of the
captured graph and under every configuration the autotuner tries."""
import os

import numpy as np
import pytest

from conftest import golden_graph
import grass_b200 as G

pytestmark = pytest.mark.gpu


def _u32(t):
    return t.cpu().numpy().view(np.uint32).copy()


class Mix:
    """A batch of uneven jobs plus the standalone results to compare with."""

    def __init__(self, torch, g, n, on=None):
        """on: what the batch samples (default the graph g itself; a Csr of
        the same graph must give the same outputs)."""
        self.torch, self.g, self.n = torch, g, n
        self.dev = torch.device("cuda")
        self.batch = G.Batch(g if on is None else on)
        self.jobs = []  # (kind, outputs, expected, edges tensor, expected edges)
        rng = np.random.default_rng(5)
        for k, (W, L, lay) in enumerate([(1000, 10, 0), (37, 80, 1), (4096, 3, 1), (1, 5, 0)]):
            self._rw(rng, W, L, lay, seed=100 + k)
        for k, fan in enumerate([(25, 10), (5, 5, 5), (10,), (3, 7)]):
            self._khop(rng, int(rng.integers(1, 300)), fan, seed=200 + k)
        for k, (S, R, T, sel) in enumerate([(3, 80, 100, 0), (1, 2000, 500, 1), (2, 7, 64, 1),
                                            (2, 300, 700, 2), (1, 2000, 3000, 2),
                                            (4, 50, 20, 2)]):
            self._mrw(S, R, T, sel, seed=300 + k)

    def _ints(self, a):
        return self.torch.from_numpy(np.ascontiguousarray(a, np.uint32).view(np.int32)).to(self.dev)

    def _rw(self, rng, W, L, lay, seed):
        t = self.torch
        starts = self._ints(rng.integers(0, self.n, W))
        out = t.empty(W * (L + 1), dtype=t.int32, device=self.dev)
        ref = t.empty_like(out)
        e, re_ = t.zeros(1, dtype=t.int64, device=self.dev), t.zeros(1, dtype=t.int64, device=self.dev)
        self.g.rw_device(starts, W, L, seed, ref, re_, layout=lay)
        self.batch.add_rw(starts, W, L, seed, out, layout=lay, edges=e)
        self.jobs.append(("rw", [out], [ref], e, re_, starts))

    def _khop(self, rng, S, fan, seed):
        t = self.torch
        seeds = self._ints(rng.integers(0, self.n, S))
        outs = [t.empty(S * w, dtype=t.int32, device=self.dev) for w in G.hop_widths(fan)]
        refs = [t.empty_like(o) for o in outs]
        e, re_ = t.zeros(1, dtype=t.int64, device=self.dev), t.zeros(1, dtype=t.int64, device=self.dev)
        self.g.khop_device(seeds, S, fan, seed, refs, re_)
        self.batch.add_khop(seeds, S, fan, seed, outs, edges=e)
        self.jobs.append(("khop", outs, refs, e, re_, seeds))

    def _mrw(self, S, R, T, sel, seed):
        t = self.torch
        roots = t.empty(S * R, dtype=t.int32, device=self.dev)
        G.mrw_roots_device(self.n, S, R, seed, roots)
        ref_roots = roots.clone()
        src, dst = (t.empty(S * T, dtype=t.int32, device=self.dev) for _ in range(2))
        rsrc, rdst = t.empty_like(src), t.empty_like(dst)
        e, re_ = t.zeros(1, dtype=t.int64, device=self.dev), t.zeros(1, dtype=t.int64, device=self.dev)
        self.g.mrw_device(ref_roots, S, R, T, seed, rsrc, rdst, select=sel, edge_count=re_)
        self.batch.add_mrw(roots, S, R, T, seed, src, dst, select=sel, edges=e)
        self.jobs.append(("mrw", [src, dst, roots], [rsrc, rdst, ref_roots], e, re_, None))

    def check(self, runs=1):
        t = self.torch
        for kind, outs, refs, e, re_, _ in self.jobs:
            e.zero_()
        total = t.zeros(1, dtype=t.int64, device=self.dev)
        for _ in range(runs):
            total.zero_()
            for kind, outs, refs, e, re_, _ in self.jobs:
                e.zero_()
            self.batch.run(total=total)
            t.cuda.synchronize()
            for kind, outs, refs, e, re_, _ in self.jobs:
                for o, r in zip(outs, refs):
                    np.testing.assert_array_equal(_u32(o), _u32(r), err_msg=kind)
                assert int(e.item()) == int(re_.item()), kind
            assert int(total.item()) == sum(int(j[4].item()) for j in self.jobs)


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_batch_matches_standalone_calls(mode):
    import torch
    d, rowptr, cols, meta = golden_graph("hub")
    g = G.Graph(os.path.join(d, mode), mode)
    m = Mix(torch, g, g.n)
    info = m.batch.info()
    assert info["jobs"] == 14
    m.check(runs=2)  # graph capture, then replay (multi-RW roots restored)
    m.batch.set_config(use_graph=2)  # plain launches
    m.check()


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_batch_configs_and_autotune(mode):
    import torch
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, mode), mode)
    m = Mix(torch, g, g.n)
    for tile, depth, wpb, wpv in [(64, 1, 1, 1), (256, 4, 8, 2), (96, 2, 2, 4), (64, 1, 8, 8)]:
        m.batch.set_config(walker_tile=tile, depth=depth, warps_per_block=wpb, khop_seeds=3,
                           warps_per_vertex=wpv)
        m.check()  # k-hop seeds split over wpv warps: the same frontiers and edge counts
    best, ms = m.batch.autotune()
    assert ms > 0 and best["walker_tile"] in (64, 128, 256)
    assert best["warps_per_vertex"] in (1, 2, 4, 8)
    assert m.batch.config()["walker_tile"] == best["walker_tile"]
    assert m.batch.config()["warps_per_vertex"] == best["warps_per_vertex"]
    m.check()


@pytest.mark.parametrize("mode", ["GT", "LE"])
def test_batch_on_csr_equals_compressed(mode):
    """The batched kernel on the uncompressed CSR decoded from a graph gives
    every job the same output as the standalone compressed calls."""
    import torch
    d, rowptr, cols, meta = golden_graph("rmat_s10_e8")
    g = G.Graph(os.path.join(d, mode), mode)
    csr = g.csr()
    m = Mix(torch, g, g.n, on=csr)
    m.check(runs=2)
    m.batch.set_config(walker_tile=64, depth=2, warps_per_block=4, khop_seeds=2,
                       warps_per_vertex=4)
    m.check()
