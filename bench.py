#!/usr/bin/env python3
"""Benchmark of the compressed-graph sampling hot path on B200.

Workload (N=1 line): R-MAT scale 22, edge factor 32, a/b/c/d = .57/.19/.19/.05,
seed 42, relabelled/deduped/symmetrized with graph_sort semantics and written in
the reference's LE and GT formats (byte-identical to the reference compressor);
then
  (a) 1,048,576 uniform random walks of length 80 (Philox seed 7) -- the headline,
  (b) k-hop with fanouts (25, 10) for 65,536 uniform seeds,
  (c) a decode-only sweep of every neighbor list,
each in LE and GT modes and on an uncompressed CSR with the same RNG stream.

A "step" is one launch of the sampler over the whole batch (all walkers, all
80 steps).  `value` = sampled edges/s with inputs resident in HBM (CUDA events
on the launching stream, L2 flushed by a 256 MiB write between timed steps).
`e2e` = the same metric through the public host API (grass_rw_host) from pinned
host memory, copies of starts in and paths out inside the timed region.

After each timed region rank 0 checks what the timed launches produced
against the CPU oracle, bit for bit (`parity` key; the run exits non-zero on
a mismatch): walkers 0..65535 of each walk, seeds 0..4095 of each k-hop, the
whole decode sweep, 8 jobs of each batched run.

`--impl reference` times the reference's CPU decode+sample path -- here the
CPU oracle's restatement of the reference decoders and app logic (the
reference has no CPU sampler) -- on all host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "sampled edges/s (random walk, compressed graph)"
UNIT = "edges/s"
CACHE = os.path.join(tempfile.gettempdir(), "grass_bench_cache")
LAYOUT = 1  # GRASS_LAYOUT_STEP_MAJOR: coalesced path stores in every arm


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="grass", choices=["grass", "reference"])
    ap.add_argument("--scale", type=int, default=22)
    ap.add_argument("--edge-factor", type=int, default=32)
    ap.add_argument("--walkers", type=int, default=1 << 20)
    ap.add_argument("--mrw-samples", type=int, default=1 << 18,
                    help="multi-RW samples (80 walkers x 100 steps each) for --only mrw")
    ap.add_argument("--length", type=int, default=80)
    ap.add_argument("--khop-seeds", type=int, default=65536)
    ap.add_argument("--mode", default="LE", choices=["LE", "GT"])
    ap.add_argument("--only", default="",
                    help="comma list: rw,khop,decode,csr,e2e,cpu,batch,serve,parity,cfg5,refgpu "
                         "(cfg5, the 3B-edge Chung-Lu graph, and refgpu, the reference's own "
                         "GPU rw app, run only when named)")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--batch-scale", type=int, default=24,
                    help="R-MAT scale of the batched-jobs / serving graph (edge factor 16)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU; replicas only, no data exchange)

def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def dist_init(ws, backend):
    if ws <= 1:
        return None
    import datetime
    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return dist


def barrier(dist, dev=None):
    if dist is not None:
        if dev is not None:
            dist.barrier(device_ids=[dev])
        else:
            dist.barrier()


def _reduce(dist, x: float, op, torch):
    if dist is None:
        return x
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(dist, x: float, torch=None) -> float:
    """Slowest rank's time: every multi-GPU number is timed as the max over ranks."""
    return _reduce(dist, x, dist.ReduceOp.MAX if dist else None, torch)


def sum_over_ranks(dist, x: float, torch=None) -> float:
    """Whole-job total (edges of all replicas)."""
    return _reduce(dist, x, dist.ReduceOp.SUM if dist else None, torch)


def replica_seed(base: int, rank: int) -> int:
    """Philox seed of a replica's walks: each rank samples its own walkers."""
    return base + rank


# ---------------------------------------------------------------------------
# synthetic graph (cached per box)

def build_graph(scale, ef):
    import grass_b200 as G
    key = f"rmat_s{scale}_e{ef}_seed42"
    d = os.path.join(CACHE, key)
    done = os.path.join(d, "done.json")
    if os.path.exists(done):
        return d, json.load(open(done))
    os.makedirs(d, exist_ok=True)
    t0 = time.time()
    rp, cols = G.rmat_graph(scale, ef, seed=42)
    t1 = time.time()
    meta = {"n": int(len(rp) - 1), "num_edges": int(len(cols)), "gen_s": t1 - t0}
    for mode in ("LE", "GT"):
        t2 = time.time()
        G.compress_to_files(rp, cols, mode, os.path.join(d, mode))
        meta[f"compress_{mode}_s"] = time.time() - t2
    np.save(os.path.join(d, "rowptr.npy"), rp)
    np.save(os.path.join(d, "cols.npy"), cols)
    json.dump(meta, open(done, "w"))
    return d, meta


def build_chung_lu(n, exponent, mean_degree, max_degree, seed=42):
    """Chung-Lu graph (m = n * mean_degree / 2 generated edges), graph_sort
    (undirected), written in both formats; cached per box like build_graph."""
    import grass_b200 as G
    key = f"chunglu_n{n}_x{exponent}_d{mean_degree}_max{max_degree}_seed{seed}"
    d = os.path.join(CACHE, key)
    done = os.path.join(d, "done.json")
    if os.path.exists(done):
        return d, json.load(open(done))
    os.makedirs(d, exist_ok=True)
    t0 = time.time()
    src, dst = G.gen_chung_lu(n, exponent, mean_degree, max_degree, int(n * mean_degree // 2),
                              seed=seed)
    t1 = time.time()
    rp, cols = G.graph_sort(src, dst, directed=False)
    del src, dst
    t2 = time.time()
    meta = {"n": int(len(rp) - 1), "num_edges": int(len(cols)), "gen_s": t1 - t0,
            "sort_s": t2 - t1, "max_degree": int(np.diff(rp).max())}
    for mode in ("LE", "GT"):
        t3 = time.time()
        G.compress_to_files(rp, cols, mode, os.path.join(d, mode))
        meta[f"compress_{mode}_s"] = time.time() - t3
    np.save(os.path.join(d, "rowptr.npy"), rp)
    json.dump(meta, open(done, "w"))
    return d, meta


def cfg5_bench(G, torch, stream, flush, K, parity=None):
    """Skewed large graph: Chung-Lu n = 100M, exponent 2.1, mean degree 30,
    max degree 1M (~3B directed edges after symmetrising).  4M uniform walks
    of length 40, k-hop (15, 10) for 262,144 seeds drawn among the vertices
    of degree >= 1000, the decode sweep, and the footprints, in LE, GT and on
    the CSR decoded from the LE graph."""
    dev = torch.device("cuda", torch.cuda.current_device())
    gdir, meta = build_chung_lu(100_000_000, 2.1, 30, 1_000_000)
    n, E = meta["n"], meta["num_edges"]
    out = {"graph": meta}
    graphs = {m: G.Graph(os.path.join(gdir, m), m) for m in ("LE", "GT")}
    infos = {m: graphs[m].info() for m in graphs}
    csr = graphs["LE"].csr()
    W, L = 4 << 20, 40
    starts = torch.empty(W, dtype=torch.int32, device=dev)
    G.uniform_starts_device(n, W, 7, starts, stream=stream)
    paths = torch.empty(W * (L + 1), dtype=torch.int32, device=dev)
    ecount = torch.zeros(1, dtype=torch.int64, device=dev)
    for name, obj in [("LE", graphs["LE"]), ("GT", graphs["GT"]), ("CSR", csr)]:
        ecount.zero_()
        obj.rw_device(starts, W, L, 7, paths, ecount, layout=LAYOUT, stream=stream)
        torch.cuda.synchronize()
        e1 = int(ecount.item())
        ms, tot = timed(torch, lambda o=obj: o.rw_device(starts, W, L, 7, paths, ecount,
                                                         layout=LAYOUT, stream=stream),
                        K, 2, flush)
        out[f"rw_{name}"] = {"value": e1 * K / (tot / 1000.0), "ms_per_step": tot / K,
                             "edges_per_step": e1}
    del paths
    rp = np.load(os.path.join(gdir, "rowptr.npy"))
    hubs = np.nonzero(np.diff(rp) >= 1000)[0].astype(np.uint32)
    del rp
    if parity is not None and parity.enabled:
        # walks that start on hubs (degree >= 1000): long LE chunks, long GT runs
        Wh = 16384
        hs = torch.from_numpy(hubs[np.random.default_rng(5).integers(0, len(hubs), Wh)]
                              .view(np.int32)).to(dev)
        hp = torch.empty(Wh * (L + 1), dtype=torch.int32, device=dev)
        for m in ("LE", "GT"):
            graphs[m].rw_device(hs, Wh, L, 9, hp, layout=LAYOUT, stream=stream)
            torch.cuda.synchronize()
            parity.rw(f"cfg5_rw_hub_starts_{m}", os.path.join(gdir, m), m, hs, Wh, L, 9, hp,
                      LAYOUT)
        del hp
    S, fan = 262144, (15, 10)
    pick = np.random.default_rng(11).integers(0, len(hubs), S)
    seeds = torch.from_numpy(hubs[pick].view(np.int32)).to(dev)
    hops = [torch.empty(S * w, dtype=torch.int32, device=dev) for w in G.hop_widths(fan)]
    for name, obj in [("LE", graphs["LE"]), ("GT", graphs["GT"]), ("CSR", csr)]:
        ecount.zero_()
        obj.khop_device(seeds, S, fan, 13, hops, ecount, stream=stream)
        torch.cuda.synchronize()
        e1 = int(ecount.item())
        ms, tot = timed(torch, lambda o=obj: o.khop_device(seeds, S, fan, 13, hops, ecount,
                                                           stream=stream), K, 2, flush)
        out[f"khop_{name}"] = {"value": e1 * K / (tot / 1000.0), "ms_per_step": tot / K,
                               "seeds_with_degree_ge_1000": int(len(hubs))}
        if parity is not None and name != "CSR":
            parity.khop(f"cfg5_khop_{name}", os.path.join(gdir, name), name, seeds, S, fan, 13,
                        hops, k=1024)
    del hops
    rp_d = torch.empty(n + 1, dtype=torch.int64, device=dev)
    cl_d = torch.empty(E, dtype=torch.int32, device=dev)
    for m in ("LE", "GT"):
        ms, tot = timed(torch, lambda g=graphs[m]: g.decode_all_device(rp_d, cl_d, stream=stream),
                        K, 2, flush)
        out[f"decode_{m}"] = {"value": E * K / (tot / 1000.0), "unit": "decoded edges/s",
                              "ms_per_step": tot / K}
    del rp_d, cl_d
    csr_bytes = (n + 1) * 8 + 4 * E
    out["footprint_bytes"] = {"CSR": csr_bytes, **{m: infos[m]["device_bytes"] for m in infos},
                              **{f"ratio_{m}": csr_bytes / infos[m]["device_bytes"]
                                 for m in infos}}
    out["compressed_vs_csr"] = {m: out[f"rw_{m}"]["value"] / out["rw_CSR"]["value"]
                                for m in ("LE", "GT")}
    return out


# ---------------------------------------------------------------------------
# clocks during the timed region

_T0 = time.time()


def progress(msg: str):
    """One line per phase on stderr, with the seconds since the bench started."""
    print(f"[bench +{time.time() - _T0:7.1f}s] {msg}", file=sys.stderr, flush=True)


# host wall-clock windows of the timed regions (time.time(), start and end),
# recorded by timed() so that the clock samples taken inside them can be told apart
TIMED_WINDOWS = []


class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap,"
              "utilization.gpu,timestamp")

    def __init__(self, gpu_index: int, enabled: bool = True):
        self.p = None
        self.path = None
        if not enabled:
            return
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(gpu_index)], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict | None:
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.close()
        import datetime
        sm, mx, pw, busy, inside = [], [], [], [], []
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 11:
                continue
            try:
                c, m, w = float(parts[1]), float(parts[2]), float(parts[3])
                b = float(parts[9]) >= 50.0
                ts = datetime.datetime.strptime(parts[10], "%Y/%m/%d %H:%M:%S.%f").timestamp()
            except ValueError:
                continue
            sm.append(c)
            mx.append(m)
            pw.append(w)
            busy.append(b)
            # a sample within 50 ms of a timed region counts as taken during it
            inside.append(any(t0 - 0.05 <= ts <= t1 + 0.05 for t0, t1 in TIMED_WINDOWS))
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        # median under load: the samples taken during the timed regions, else
        # those with the GPU busy (the sampler also runs while graphs load and
        # while the host checks outputs between timed regions)
        loaded = ([c for c, t in zip(sm, inside) if t] or [c for c, b in zip(sm, busy) if b]
                  or sm)
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "samples": len(sm),
                "samples_in_timed_regions": sum(inside), "samples_under_load": sum(busy),
                "power_w_max": max(pw), "reasons": sorted(reasons)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Parity:
    """Bit-exact checks of what the timed launches produced, against the CPU
    oracle (the checker), run after each timed region and outside it.  Each
    check compares a bounded slice of a benchmarked output -- walkers and
    seeds 0..k-1 use the same Philox streams in the full launch and in the
    oracle's run over those k inputs -- or, for the decode sweep, all of it."""

    def __init__(self, enabled: bool):
        self.enabled = enabled
        self.res = {}
        self._og = {}

    def graph(self, prefix):
        import oracle
        if prefix not in self._og:
            self._og[prefix] = oracle.OracleGraph(prefix)
        return self._og[prefix]

    def put(self, key, ok, **detail):
        self.res[key] = {"ok": bool(ok), **detail}

    def rw(self, key, prefix, mode, starts, W, L, seed, paths, layout, k=65536):
        """paths: the launch's [L+1][W] (step-major) or [W][L+1] output."""
        if not self.enabled:
            return
        k = min(k, W)
        st = starts[:k].cpu().numpy().view(np.uint32)
        ref, _ = self.graph(prefix).rw(mode, st, L, seed)
        P = paths.view(L + 1, W)[:, :k].T if layout == 1 else paths.view(W, L + 1)[:k]
        got = P.contiguous().cpu().numpy().view(np.uint32)
        self.put(key, np.array_equal(got, ref), walkers=k, steps=L)

    def node2vec(self, key, prefix, mode, starts, W, L, seed, p, q, paths, layout, k=8192):
        if not self.enabled:
            return
        k = min(k, W)
        st = starts[:k].cpu().numpy().view(np.uint32)
        ref, _ = self.graph(prefix).node2vec(mode, st, L, seed, p, q)
        P = paths.view(L + 1, W)[:, :k].T if layout == 1 else paths.view(W, L + 1)[:k]
        got = P.contiguous().cpu().numpy().view(np.uint32)
        self.put(key, np.array_equal(got, ref), walkers=k, steps=L, p=p, q=q)

    def khop(self, key, prefix, mode, seeds, S, fan, seed, hops, k=4096):
        if not self.enabled:
            return
        k = min(k, S)
        sd = seeds[:k].cpu().numpy().view(np.uint32)
        refs, _ = self.graph(prefix).khop(mode, sd, fan, seed)
        ok = True
        for h, w in enumerate(np.cumprod(fan)):
            got = hops[h].view(S, int(w))[:k].cpu().numpy().view(np.uint32)
            ok = ok and np.array_equal(got, refs[h])
        self.put(key, ok, seeds=k, fanouts=list(fan))

    def mrw(self, key, prefix, mode, roots0, R, T, seed, src, dst, roots, k=256):
        """Samples 0..k-1 of a multi-RW launch: edges taken and final roots."""
        if not self.enabled:
            return
        r0 = roots0[:k * R].cpu().numpy().view(np.uint32).reshape(k, R)
        rs, rd, fin, _ = self.graph(prefix).mrw(mode, r0, T, seed, 0)
        ok = (np.array_equal(src[:k * T].cpu().numpy().view(np.uint32).reshape(k, T), rs) and
              np.array_equal(dst[:k * T].cpu().numpy().view(np.uint32).reshape(k, T), rd) and
              np.array_equal(roots[:k * R].cpu().numpy().view(np.uint32).reshape(k, R), fin))
        self.put(key, ok, samples=k, walkers=R, steps=T)

    def batch(self, key, prefix, mode, jobs, bufs, per_type=(3, 3, 2)):
        """The first per_type[t] jobs of each type of a batched run: RW paths
        (walk-major), k-hop frontiers, multi-RW edges and final roots."""
        if not self.enabled:
            return
        og = self.graph(prefix)
        u32 = lambda t: t.cpu().numpy().view(np.uint32)  # noqa: E731
        ok, picked = True, [0, 0, 0]
        for j, (inp, outs, snap) in zip(jobs, bufs):
            t = j["type"]
            if picked[t] >= per_type[t]:
                continue
            picked[t] += 1
            c = j["count"]
            if t == 0:
                ref, _ = og.rw(mode, u32(inp), j["length"], j["seed"])
                ok = ok and np.array_equal(u32(outs[0]).reshape(c, -1), ref)
            elif t == 1:
                refs, _ = og.khop(mode, u32(inp), j["fanouts"], j["seed"])
                ok = ok and all(np.array_equal(u32(o).reshape(c, -1), r)
                                for o, r in zip(outs, refs))
            else:
                roots = u32(snap).reshape(c, j["walkers"])
                src, dst, fin, _ = og.mrw(mode, roots, j["steps"], j["seed"], j["select"])
                ok = (ok and np.array_equal(u32(outs[0]).reshape(c, -1), src) and
                      np.array_equal(u32(outs[1]).reshape(c, -1), dst) and
                      np.array_equal(u32(inp).reshape(c, -1), fin))
        self.put(key, ok, jobs={"rw": picked[0], "khop": picked[1], "mrw": picked[2]})

    def decode(self, key, prefix, mode, rowptr, cols):
        if not self.enabled:
            return
        if (prefix, "decode") not in self._og:
            self._og[(prefix, "decode")] = self.graph(prefix).decode_all(mode)
        rp, cl = self._og[(prefix, "decode")]
        ok = (np.array_equal(rowptr.cpu().numpy().view(np.uint64), rp) and
              np.array_equal(cols.cpu().numpy().view(np.uint32), cl))
        self.put(key, ok, neighbors=int(len(cl)), vertices=int(len(rp) - 1))


def ncu_traffic(workload_key: str):
    """Per-launch DRAM bytes of the walk kernel from the committed ncu summary
    (profiles/traffic.json: dram__bytes_read.sum + dram__bytes_write.sum of one
    capture, scaled to a full launch by draws), and where they come from."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(p):
        return None, None
    d = json.load(open(p))
    e = d.get(workload_key)
    if not isinstance(e, dict):
        return None, None
    return e.get("bytes_per_launch"), e.get("capture")


def random_sector_ceiling(G, torch, dev, flush, K=5, W=3):
    """Uniform random 4-byte reads from a 2 GiB buffer (the library's
    random-read probe: 8 loads in flight per thread, 2048 threads per SM).
    Each read lands in its own 32-byte sector, so the rate is what HBM gives
    random sector reads with no locality at all.  Reported beside the walks'
    sector rates, which are higher: records and hub payloads are reused."""
    n = 1 << 29
    buf = torch.zeros(n, dtype=torch.int32, device=dev)
    sink = torch.zeros(1, dtype=torch.int64, device=dev)
    reads = 1 << 27
    issued = G.random_read_probe(buf, n, reads, 3, sink)
    ms, tot = timed(torch, lambda: G.random_read_probe(buf, n, reads, 3, sink), K, W, flush)
    del buf
    return {"reads_per_launch": issued, "ms_per_launch": tot / K,
            "sectors_per_s": issued * K / (tot / 1000.0),
            "method": "grass_random_read_probe: 2^27 uniform random 4-byte reads from a 2 GiB buffer"}


# ---------------------------------------------------------------------------
# timing

def timed(torch, fn, K, W, flush, dist=None, dev=None):
    """W untimed warm-up calls, then K calls each bracketed by CUDA events on
    the current stream, with an L2 flush outside the events between calls.
    Returns (per-call ms list, max over ranks of the summed device time)."""
    for _ in range(W):
        fn()
    torch.cuda.synchronize()
    barrier(dist, dev)
    torch.cuda.synchronize()
    st = torch.cuda.current_stream()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(K)]
    t_start = time.time()
    for a, b in evs:
        flush()
        a.record(st)
        fn()
        b.record(st)
    torch.cuda.synchronize()
    TIMED_WINDOWS.append((t_start, time.time()))
    barrier(dist, dev)
    torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in evs]
    return ms, max_over_ranks(dist, sum(ms), torch)


# ---------------------------------------------------------------------------
# batched uneven jobs (R-MAT s24 ef16) and the serving loop on the same graph

MIX_FANOUTS = [(10, 5), (15, 10), (25, 10), (5, 5, 5)]


def mix_jobs(n, k=256, seed=3):
    """k jobs: 40% RW (L ~ U[10,100]), 40% k-hop (fanouts from MIX_FANOUTS),
    20% multi-RW (one sample of 2000 walkers, 10,000 steps, degree-
    proportional selection in its continuous-time construction, walkers
    moving in parallel); RW walkers / k-hop seeds ~ lognormal(ln 1024, 1.5)
    clipped to [1, 65536]."""
    rng = np.random.default_rng(seed)
    n_rw, n_kh = round(0.4 * k), round(0.4 * k)
    types = [0] * n_rw + [1] * n_kh + [2] * (k - n_rw - n_kh)
    rng.shuffle(types)
    jobs = []
    for i, t in enumerate(types):
        size = int(np.clip(np.rint(rng.lognormal(np.log(1024), 1.5)), 1, 65536))
        j = {"type": int(t), "seed": 1000 + i}
        if t == 0:
            j.update(count=size, length=int(rng.integers(10, 101)))
        elif t == 1:
            j.update(count=size, fanouts=MIX_FANOUTS[int(rng.integers(0, 4))])
        else:
            j.update(count=1, walkers=2000, steps=10000, select=2)
        jobs.append(j)
    return jobs


def batch_bench(G, torch, graphs, n, stream, flush, K, W, parity=None, gdir=None):
    """One persistent captured launch over 256 uneven jobs, autotuned, against
    the plain method (one standalone launch per job, same stream).  After the
    timed runs of each compressed mode, parity checks 8 of the jobs."""
    dev = torch.device("cuda", torch.cuda.current_device())
    jobs = mix_jobs(n)
    bufs = []
    for j in jobs:
        c = j["count"]
        if j["type"] == 0:
            inp = torch.empty(c, dtype=torch.int32, device=dev)
            G.uniform_starts_device(n, c, j["seed"], inp, stream=stream)
            outs = [torch.empty(c * (j["length"] + 1), dtype=torch.int32, device=dev)]
        elif j["type"] == 1:
            inp = torch.empty(c, dtype=torch.int32, device=dev)
            G.uniform_starts_device(n, c, j["seed"], inp, stream=stream)
            outs = [torch.empty(c * w, dtype=torch.int32, device=dev)
                    for w in G.hop_widths(j["fanouts"])]
        else:
            inp = torch.empty(c * j["walkers"], dtype=torch.int32, device=dev)
            G.mrw_roots_device(n, c, j["walkers"], j["seed"], inp, stream=stream)
            outs = [torch.empty(c * j["steps"], dtype=torch.int32, device=dev)
                    for _ in range(2)]
        bufs.append((inp, outs, inp.clone()))
    total = torch.zeros(1, dtype=torch.int64, device=dev)
    draws = {0: 0, 1: 0, 2: 0}
    res = {}
    for m, g in graphs.items():
        # the multi-RW inputs are the snapshot again (the previous mode's
        # standalone chains walked them in place); a batch copies them at add
        for j, (inp, outs, snap) in zip(jobs, bufs):
            if j["type"] == 2:
                inp.copy_(snap)

        def make(types):
            b = G.Batch(g)
            for j, (inp, outs, _) in zip(jobs, bufs):
                if j["type"] not in types:
                    continue
                if j["type"] == 0:
                    b.add_rw(inp, j["count"], j["length"], j["seed"], outs[0])
                elif j["type"] == 1:
                    b.add_khop(inp, j["count"], j["fanouts"], j["seed"], outs)
                else:
                    b.add_mrw(inp, j["count"], j["walkers"], j["steps"], j["seed"], outs[0],
                              outs[1], select=j["select"])
            return b
        b = make({0, 1, 2})
        best, best_ms = b.autotune(stream=stream)
        total.zero_()
        b.run(stream=stream, total=total)
        torch.cuda.synchronize()
        edges = int(total.item())
        lc0 = G.launch_count()
        ms, tot = timed(torch, lambda: b.run(stream=stream), K, W, flush)
        launches = (G.launch_count() - lc0) / (K + W)
        if parity is not None and m in ("LE", "GT"):
            parity.batch(f"batch_{m}", os.path.join(gdir, m), m, jobs, bufs)
        short = make({0, 1})
        short.set_config(**{k: v for k, v in best.items() if k != "use_graph"})
        ms_s, tot_s = timed(torch, lambda: short.run(stream=stream), K, W, flush)

        # plain method: each job its own launch, back to back on one stream
        def plain():
            for j, (inp, outs, snap) in zip(jobs, bufs):
                if j["type"] == 0:
                    g.rw_device(inp, j["count"], j["length"], j["seed"], outs[0], stream=stream)
                elif j["type"] == 1:
                    g.khop_device(inp, j["count"], j["fanouts"], j["seed"], outs, stream=stream)
                else:
                    inp.copy_(snap)
                    g.mrw_device(inp, j["count"], j["walkers"], j["steps"], j["seed"], outs[0],
                                 outs[1], select=j["select"], stream=stream)
        if m == "CSR":  # the CSR side: the batched launch only (no standalone CSR multi-RW)
            res[m] = {"makespan_ms": tot / K, "ms_min": min(ms), "ms_max": max(ms),
                      "edges_per_run": edges, "edges_per_s": edges / (tot / K / 1000.0),
                      "launches_per_run": launches, "autotune_best": best,
                      "autotune_best_ms": best_ms, "makespan_rw_khop_only_ms": tot_s / K}
            b.close()
            short.close()
            continue
        pms, ptot = timed(torch, plain, 1, 1, flush)
        # one multi-RW sample alone (2000 walkers x 10,000 steps, degree-proportional):
        # continuous-time (walkers in parallel) and one Philox block per step (sequential)
        mj = next(k for k, j in enumerate(jobs) if j["type"] == 2)
        minp, mouts, msnap = bufs[mj]
        chain_ms = {}
        for sel in (2, 1):
            def chain(sel=sel):
                minp.copy_(msnap)
                g.mrw_device(minp, 1, 2000, 10000, jobs[mj]["seed"], mouts[0], mouts[1],
                             select=sel, stream=stream)
            cms, ctot = timed(torch, chain, 3, 1, flush)
            chain_ms[sel] = ctot / 3
        res[m] = {"makespan_ms": tot / K, "ms_min": min(ms), "ms_max": max(ms),
                  "edges_per_run": edges, "edges_per_s": edges / (tot / K / 1000.0),
                  "launches_per_run": launches, "autotune_best": best,
                  "autotune_best_ms": best_ms,
                  "makespan_rw_khop_only_ms": tot_s / K,
                  "mrw_sample_alone_ms": {"continuous_time": chain_ms[2],
                                          "sequential_steps": chain_ms[1]},
                  "plain_one_launch_per_job_ms": ptot,
                  "speedup_vs_plain": ptot / (tot / K)}
        b.close()
        short.close()
    if "CSR" in res:
        res["compressed_vs_csr"] = {m: res["CSR"]["makespan_ms"] / res[m]["makespan_ms"]
                                    for m in ("LE", "GT") if m in res}
    for j in jobs:
        t = j["type"]
        if t == 0:
            draws[0] += j["count"] * j["length"]
        elif t == 1:
            draws[1] += j["count"] * sum(G.hop_widths(j["fanouts"]))
        else:
            draws[2] += j["count"] * j["steps"]
    res["jobs"] = {"rw": sum(j["type"] == 0 for j in jobs),
                   "khop": sum(j["type"] == 1 for j in jobs),
                   "mrw": sum(j["type"] == 2 for j in jobs),
                   "max_draws_by_type": {"rw": draws[0], "khop": draws[1], "mrw": draws[2]}}
    del bufs
    return res


SERVE_KEYS = ("completed", "rejected", "failed", "batches", "p50_us", "p99_us", "p999_us",
              "mean_us", "max_us", "p50_type_us", "p99_type_us", "queue_p50_us", "queue_p99_us",
              "service_p50_us", "service_p99_us", "issue_us", "staging_alloc_us", "phase_us",
              "wall_s",
              "edges", "edges_per_s", "achieved_rate", "launches")


def serve_bench(G, g, rates=(2000, 10000, 50000), seconds=0.25, plain_cap=1000):
    """Open-loop Poisson arrivals of the batched-jobs request mix through the
    serving loop, with results copied to host memory and with results kept
    in device memory: (1) peak = the completion rate under 200k requests/s
    offered (overload), (2) latency at 80% of that peak, (3) the listed
    rates.  At each listed rate the first plain_cap requests of the same
    trace are also served one standalone launch per request (the plain
    method, results to the host)."""
    def run(rate, nreq, mode=0, **kw):
        r = G.loadgen(g, float(rate), nreq, mode=mode, seed=5, **kw)
        return {k: r[k] for k in SERVE_KEYS}
    out = {}
    for where, kw in (("host", {}), ("device", {"results_on_device": 1})):
        o = {}
        over = run(200000, 20000, **kw)
        peak = over["achieved_rate"]
        at80 = run(0.8 * peak, int(max(2000, 0.8 * peak * seconds)), **kw)
        o["peak"] = {"offered_rate": 200000, "requests": 20000, "result": over,
                     "peak_rate": peak, "peak_edges_per_s": over["edges_per_s"]}
        o["at_80pct_of_peak"] = {"offered_rate": 0.8 * peak, "result": at80,
                                 "p99_under_5ms": at80["p99_us"] < 5000.0}
        for rate in rates:
            nreq = int(max(1000, rate * seconds))
            o[str(rate)] = {"requests": nreq, "batched": run(rate, nreq, **kw)}
            if where == "host":
                o[str(rate)]["one_job_per_launch"] = run(rate, min(nreq, plain_cap), mode=1)
                o[str(rate)]["plain_requests"] = min(nreq, plain_cap)
        out["results_" + where] = o
    return out


def cpu_baseline(gdir, mode, n, length, seed, budget_s=12.0):
    import oracle
    oracle.lib()
    og = oracle.OracleGraph(os.path.join(gdir, mode))
    threads = oracle.max_threads()
    W = 8192
    best = None
    spent = 0.0
    while True:
        starts = oracle.uniform_starts(n, W, 7)
        t0 = time.perf_counter()
        _, edges = og.rw(mode, starts, length, seed, threads)
        dt = time.perf_counter() - t0
        spent += dt
        best = (W, edges, dt)
        if dt > 2.0 or spent + 3 * dt > budget_s:
            break
        W *= 4
    W, edges, dt = best
    return {"value": edges / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{W} uniform walkers x {length} steps ({mode} decode per draw) on the "
                      f"same graph; oracle restatement of the reference decoders + app next(), "
                      f"OpenMP over walkers"}


def two_sample_chi2(a, b, min_count=10):
    """Two-sample chi-square of two count vectors over the same vertices.
    Conditional on each bin's combined count c, a's share is Binomial(c, p),
    p = sum(a) / (sum(a) + sum(b)), under the null of one law.  Vertices with
    c >= min_count are bins of their own; the others are pooled in vertex
    order into bins of combined count >= 2 min_count.  Returns (stat, df, p)."""
    from scipy.stats import chi2
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    c = a + b
    big = c >= min_count
    A, Cc = [a[big]], [c[big]]
    sa, sc = a[~big], c[~big]
    if sc.size:
        cut = np.floor(np.cumsum(sc) / (2 * min_count)).astype(np.int64)
        cut = np.minimum(cut, max(int(cut[-1]) - 1, 0))  # fold a short tail into the last bin
        A.append(np.bincount(cut, weights=sa))
        Cc.append(np.bincount(cut, weights=sc))
    A, Cc = np.concatenate(A), np.concatenate(Cc)
    keep = Cc > 0
    A, Cc = A[keep], Cc[keep]
    p = a.sum() / c.sum()
    stat = float(((A - Cc * p) ** 2 / (Cc * p * (1 - p))).sum())
    df = int(A.size - 1)
    return stat, df, float(chi2.sf(stat, df))


def reference_visits(G, torch, gdir, n, positions=(1, 10, 40, 79), timeout_s=600):
    """Per-vertex visit counts of the reference's own GPU sampler against this
    library's, two-sample chi-square per position.  The reference's rw app is
    run, one walker per vertex, from baseline/_ref/rw_{gt,le}_visits (its
    sources with baseline/visit_hook.h force-included, which writes the
    transits after the chosen steps); this library walks the same starts
    (i % n) for 80 steps.  Each walker adds one visit per position, so each
    position's counts are a sample of n walkers; ended walks are not counted.
    Calibration beside it: this library against itself (two Philox seeds),
    and, for LE, whose reference states are seeded from the clock, the
    reference against itself (two runs).  The test assumes independent
    walkers; a sample whose walkers are correlated fails it even against
    itself."""
    import tempfile
    out = {"positions": list(positions), "walkers": n}
    dev = torch.device("cuda", torch.cuda.current_device())

    def ref_counts(exe, gpath):
        with tempfile.TemporaryDirectory() as td:
            env = dict(os.environ, GRASS_VISIT_DUMP=os.path.join(td, "v"),
                       GRASS_VISIT_STEPS=",".join(map(str, positions)))
            r = subprocess.run([exe, "-g", gpath, "-n", "1"], env=env, capture_output=True,
                               text=True, timeout=timeout_s)
            cnt = {}
            for pos in positions:
                f = os.path.join(td, f"v.{pos}.i32")
                if os.path.exists(f):
                    a = np.fromfile(f, dtype=np.int32)
                    cnt[pos] = np.bincount(a[(a >= 0) & (a < n)], minlength=n)
            return r.returncode, cnt

    def chi(a, b):
        stat, df, pv = two_sample_chi2(a, b)
        return {"chi2_over_df": stat / max(df, 1), "df": df, "p": pv}

    for m in ("GT", "LE"):
        exe = os.path.join(ROOT, "baseline", "_ref", f"rw_{m.lower()}_visits")
        if not os.path.exists(exe):
            out[m] = {"unavailable": f"{exe} not built"}
            continue
        gpath = os.path.join(gdir, m)
        rc, ref = ref_counts(exe, gpath)
        ref2 = ref_counts(exe, gpath)[1] if m == "LE" else None
        g = G.Graph(gpath, m)
        starts = torch.arange(n, dtype=torch.int32, device=dev)
        paths = torch.empty(n * 81, dtype=torch.int32, device=dev)
        ours = []
        for seed in (20241203, 777):
            g.rw_device(starts, n, 80, seed, paths, layout=1)
            ours.append(paths.view(81, n).cpu().numpy())
        g.close()
        res = {"rc": rc}
        for pos in positions:
            if pos not in ref:
                res[str(pos)] = {"unavailable": "no dump"}
                continue
            oc = [np.bincount(o[pos][(o[pos] >= 0) & (o[pos] < n)], minlength=n) for o in ours]
            e = {"visits_reference": int(ref[pos].sum()), "visits_grass_b200": int(oc[0].sum()),
                 "reference_vs_grass_b200": chi(ref[pos], oc[0]),
                 "grass_b200_vs_itself": chi(oc[0], oc[1])}
            if ref2 is not None and pos in ref2:
                e["reference_vs_itself"] = chi(ref[pos], ref2[pos])
            res[str(pos)] = e
        out[m] = res
    return out


def reference_gpu(gdir, n, runs=3, timeout_s=600):
    """The reference's own GPU sampler on this GPU: its unmodified `rw` app
    (baseline/_ref/rw_gt, rw_le, built from its sources for sm_100a) against
    this library's drop-in `rw` on the same files and the same workload, the
    reference app's default: one walker per vertex starting at i % n, 80
    steps (GT/src/apps/randomwalk/randomWalks.cu:4-24), `-n runs`.  Both print
    runSamplingTime (GT/src/grass.cu:2127-2130); every walker takes every step
    on these graphs (no isolated vertices), so a run samples 80 n edges."""
    out = {"workload": f"{n} walkers (one per vertex, start i % n) x 80 steps, -n {runs}",
           "edges_per_run": 80 * n}
    bins = {"reference": {"GT": os.path.join(ROOT, "baseline", "_ref", "rw_gt"),
                          "LE": os.path.join(ROOT, "baseline", "_ref", "rw_le")},
            "grass_b200": {m: os.path.join(ROOT, "grass_b200", "bin", "rw") for m in ("GT", "LE")}}
    for who, exes in bins.items():
        for m, exe in exes.items():
            if not os.path.exists(exe):
                out[f"{who}_{m}"] = {"unavailable": f"{exe} not built"}
                continue
            cmd = [exe, "-g", os.path.join(gdir, m), "-n", str(runs)]
            if who == "grass_b200":
                cmd += ["--mode", m]
            r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
            t = None
            for line in r.stdout.splitlines():
                if line.startswith("runSamplingTime:"):
                    t = float(line.split()[1])
            res = {"rc": r.returncode, "runSamplingTime_s": t}
            if t:
                res["edges_per_s"] = 80 * n * runs / t
            out[f"{who}_{m}"] = res
    for m in ("GT", "LE"):
        a, b = out.get(f"reference_{m}", {}), out.get(f"grass_b200_{m}", {})
        if a.get("edges_per_s") and b.get("edges_per_s"):
            out[f"speedup_{m}"] = b["edges_per_s"] / a["edges_per_s"]
    return out


# ---------------------------------------------------------------------------

def run_reference(args):
    ws, rank, local = dist_env()
    if rank != 0:
        return 0
    import oracle
    gdir, meta = build_graph(args.scale, args.edge_factor)
    n = meta["n"]
    og = oracle.OracleGraph(os.path.join(gdir, args.mode))
    threads = oracle.max_threads()
    # bounded sample per step: sized so one step is ~1-3 s of CPU work
    Wc = 8192
    starts = oracle.uniform_starts(n, Wc, 7)
    t0 = time.perf_counter()
    og.rw(args.mode, starts, args.length, 7, threads)
    dt = time.perf_counter() - t0
    Wc = int(min(args.walkers, max(8192, Wc * 1.5 / max(dt, 1e-3))))
    starts = oracle.uniform_starts(n, Wc, 7)
    for _ in range(args.warmup):
        og.rw(args.mode, starts, args.length, 7, threads)
    tot_e, tot_t = 0, 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, e = og.rw(args.mode, starts, args.length, 7, threads)
        tot_t += time.perf_counter() - t0
        tot_e += e
    val = tot_e / tot_t
    sample = (f"{Wc} of the {args.walkers} uniform walkers x {args.length} steps per step, "
              f"{args.mode} decode per draw")
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * tot_t / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic",
        "config": workload_config(args, meta),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": sample},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference has no CPU sampler; this is the CPU oracle's restatement of its "
                "bcg.cuh decoders and app next() with the shared Philox stream",
    }
    print(json.dumps(line), flush=True)
    return 0


def footprint_config1(G):
    """BASELINE config 1's graph (R-MAT s16 ef16, seed 42, graph_sort): the
    resident bytes of each format and of its files against the CSR."""
    gdir, meta = build_graph(16, 16)
    n, E = meta["n"], meta["num_edges"]
    csr = (n + 1) * 8 + 4 * E
    out = {"graph": f"R-MAT scale 16 edge factor 16: {n} vertices, {E} directed edges",
           "CSR": csr}
    for m in ("LE", "GT"):
        g = G.Graph(os.path.join(gdir, m), m)
        inf = g.info()
        out[m] = {"device_bytes": inf["device_bytes"], "ratio_device": csr / inf["device_bytes"],
                  "file_bytes": inf["graph_file_bytes"] + inf["offset_file_bytes"],
                  "ratio_files": csr / (inf["graph_file_bytes"] + inf["offset_file_bytes"])}
        g.close()
    return out


def workload_config(args, meta):
    return {
        "workload": f"random walk, {args.walkers} uniform walkers x L={args.length}, "
                    f"{args.mode} compressed R-MAT s{args.scale} ef{args.edge_factor}",
        "graph": f"R-MAT scale {args.scale} edge factor {args.edge_factor} "
                 f".57/.19/.19/.05 seed 42, graph_sort (undirected)",
        "vertices": meta["n"], "directed_edges": meta["num_edges"],
        "walkers": args.walkers, "length": args.length, "philox_seed": 7,
        "decode_mode": args.mode, "l2": "flushed (256 MiB write) between timed steps",
        "path_layout": "step-major [L+1][W] (both compressed and CSR arms)",
    }


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    ws, rank, local = dist_env()
    import torch
    torch.cuda.set_device(local)
    dist = dist_init(ws, "nccl")
    import grass_b200 as G

    only = set(args.only.split(",")) if args.only else {"rw", "khop", "decode", "csr", "e2e",
                                                         "cpu", "batch", "serve", "parity",
                                                         "footprint"}
    progress("graph build / cache")
    gdir, meta = build_graph(args.scale, args.edge_factor)
    n, E = meta["n"], meta["num_edges"]
    W, L = args.walkers, args.length
    dev = torch.device("cuda", local)
    progress("open graphs")
    stream = torch.cuda.current_stream()
    flush_buf = torch.empty(64 << 20, dtype=torch.int32, device=dev)

    def flush():
        flush_buf.fill_(1)

    graphs = {m: G.Graph(os.path.join(gdir, m), m, device=local) for m in ("LE", "GT")}
    infos = {m: graphs[m].info() for m in graphs}
    csr = graphs["LE"].csr() if ("csr" in only) else None

    # per-rank walker ids offset so replicas sample different walks
    starts = torch.empty(W, dtype=torch.int32, device=dev)
    G.uniform_starts_device(n, W, replica_seed(7, rank), starts, stream=stream)
    paths = torch.empty(W * (L + 1), dtype=torch.int32, device=dev)
    ecount = torch.zeros(1, dtype=torch.int64, device=dev)
    clocks = Clocks(local, enabled=not args.no_clocks)
    out = {}
    # the oracle checks the benchmarked outputs on rank 0 (outside every timed region)
    parity = Parity(rank == 0 and "parity" in only)

    def rw_fn(obj):
        return lambda: obj.rw_device(starts, W, L, replica_seed(7, rank), paths, ecount, layout=LAYOUT,
                                     stream=stream)

    progress("random walks")
    # ---- (a) random walk: headline mode first
    order = [args.mode] + [m for m in ("LE", "GT") if m != args.mode]
    launches0 = G.launch_count()
    for m in order:
        ecount.zero_()
        graphs[m].rw_device(starts, W, L, replica_seed(7, rank), paths, ecount, layout=LAYOUT, stream=stream)
        torch.cuda.synchronize()
        edges_per_step = int(ecount.item())
        lc0 = G.launch_count()
        ms, tot = timed(torch, rw_fn(graphs[m]), args.steps, args.warmup, flush, dist, local)
        lc = G.launch_count() - lc0 - args.warmup
        all_edges = sum_over_ranks(dist, edges_per_step * args.steps, torch)
        out[f"rw_{m}"] = {"value": all_edges / (tot / 1000.0), "ms_per_step": tot / args.steps,
                          "edges_per_step": edges_per_step, "launches": lc,
                          "ms_min": min(ms), "ms_max": max(ms)}
        parity.rw(f"rw_{m}", os.path.join(gdir, m), m, starts, W, L, replica_seed(7, rank),
                  paths, LAYOUT)
    if "csr" in only and csr is not None:
        ecount.zero_()
        csr.rw_device(starts, W, L, replica_seed(7, rank), paths, ecount, layout=LAYOUT, stream=stream)
        torch.cuda.synchronize()
        e1 = int(ecount.item())
        ms, tot = timed(torch, rw_fn(csr), args.steps, args.warmup, flush, dist, local)
        all_edges = sum_over_ranks(dist, e1 * args.steps, torch)
        out["rw_CSR"] = {"value": all_edges / (tot / 1000.0), "ms_per_step": tot / args.steps}

    progress("k-hop")
    # ---- (b) k-hop (25, 10)
    if "khop" in only:
        S, fan = args.khop_seeds, (25, 10)
        seeds = torch.empty(S, dtype=torch.int32, device=dev)
        G.uniform_starts_device(n, S, 11 + rank, seeds, stream=stream)
        hops = [torch.empty(S * w, dtype=torch.int32, device=dev) for w in G.hop_widths(fan)]
        for name, obj in [("LE", graphs["LE"]), ("GT", graphs["GT"])] + (
                [("CSR", csr)] if csr is not None else []):
            ecount.zero_()
            obj.khop_device(seeds, S, fan, 13, hops, ecount, stream=stream)
            torch.cuda.synchronize()
            e1 = int(ecount.item())
            ms, tot = timed(torch, lambda o=obj: o.khop_device(seeds, S, fan, 13, hops, ecount,
                                                               stream=stream),
                            args.steps, args.warmup, flush, dist, local)
            out[f"khop_{name}"] = {"value": sum_over_ranks(dist, e1 * args.steps, torch) /
                                   (tot / 1000.0), "ms_per_step": tot / args.steps}
            if name != "CSR":
                parity.khop(f"khop_{name}", os.path.join(gdir, name), name, seeds, S, fan, 13,
                            hops)
        # output compaction of the same frontiers to a (src, dst) edge list
        slots = S * sum(G.hop_widths(fan))
        csrc = torch.empty(slots, dtype=torch.int32, device=dev)
        cdst = torch.empty(slots, dtype=torch.int32, device=dev)
        ccount = torch.zeros(1, dtype=torch.int64, device=dev)

        def compact():
            G.khop_edges_device(seeds, S, fan, hops, csrc, cdst, slots, ccount, stream=stream)

        compact()
        torch.cuda.synchronize()
        kept = int(ccount.item())
        ms, tot = timed(torch, compact, args.steps, args.warmup, flush, dist, local)
        # algorithmic bytes: every slot read once, every parent slot read once,
        # every kept edge written as two words
        alg = 4 * slots + 4 * (S + S * fan[0]) + 8 * kept
        out["khop_compact"] = {
            "value": sum_over_ranks(dist, slots * args.steps, torch) / (tot / 1000.0),
            "unit": "frontier slots/s", "ms_per_step": tot / args.steps, "kept_edges": kept,
            "algorithmic_bytes": alg,
            "achieved_gbs": alg / (tot / args.steps / 1000.0) / 1e9}
        del hops, csrc, cdst

    # ---- second-order (node2vec) walk, beyond the reference: only when asked for
    if "n2v" in only:
        progress("node2vec walks")
        for name, obj in [("LE", graphs["LE"]), ("GT", graphs["GT"])] + (
                [("CSR", csr)] if csr is not None else []):
            for (p, q) in ((1.0, 0.5), (4.0, 0.25)):
                ecount.zero_()
                obj.node2vec_device(starts, W, L, replica_seed(7, rank), p, q, paths, ecount, layout=LAYOUT,
                                    stream=stream)
                torch.cuda.synchronize()
                e1 = int(ecount.item())
                ms, tot = timed(torch, lambda o=obj: o.node2vec_device(
                    starts, W, L, replica_seed(7, rank), p, q, paths, ecount, layout=LAYOUT,
                    stream=stream),
                    args.steps, args.warmup, flush, dist, local)
                out[f"node2vec_{name}_p{p:g}_q{q:g}"] = {
                    "value": sum_over_ranks(dist, e1 * args.steps, torch) / (tot / 1000.0),
                    "unit": UNIT, "ms_per_step": tot / args.steps, "edges_per_step": e1}
                if name != "CSR":
                    parity.node2vec(f"node2vec_{name}_p{p:g}_q{q:g}", os.path.join(gdir, name),
                                    name, starts, W, L, replica_seed(7, rank), p, q, paths,
                                    LAYOUT)

    # ---- multi-RW in the reference mrw app's shape, beyond the headline: only when asked for
    if "mrw" in only:
        progress("multi-RW")
        S_m, R_m, T_m = args.mrw_samples, 80, 100
        roots0 = torch.empty(S_m * R_m, dtype=torch.int32, device=dev)
        G.mrw_roots_device(n, S_m, R_m, replica_seed(11, rank), roots0, stream=stream)
        torch.cuda.synchronize()
        mroots = torch.empty_like(roots0)
        msrc = torch.empty(S_m * T_m, dtype=torch.int32, device=dev)
        mdst = torch.empty(S_m * T_m, dtype=torch.int32, device=dev)
        for name in ("LE", "GT"):
            obj = graphs[name]

            def mrun(o=obj):  # the roots are updated in place: restore them (S x R x 4 bytes)
                mroots.copy_(roots0)
                o.mrw_device(mroots, S_m, R_m, T_m, replica_seed(11, rank), msrc, mdst,
                             edge_count=ecount, stream=stream)
            ecount.zero_()
            mrun()
            torch.cuda.synchronize()
            e1 = int(ecount.item())
            ms, tot = timed(torch, mrun, args.steps, args.warmup, flush, dist, local)
            out[f"mrw_{name}"] = {
                "value": sum_over_ranks(dist, e1 * args.steps, torch) / (tot / 1000.0),
                "unit": UNIT, "ms_per_step": tot / args.steps, "edges_per_step": e1,
                "samples": S_m, "walkers": R_m, "steps": T_m}
            parity.mrw(f"mrw_{name}", os.path.join(gdir, name), name, roots0, R_m, T_m,
                       replica_seed(11, rank), msrc, mdst, mroots)
        del roots0, mroots, msrc, mdst

    progress("decode sweep")
    # ---- (c) decode-only sweep
    if "decode" in only:
        rp_d = torch.empty(n + 1, dtype=torch.int64, device=dev)
        cl_d = torch.empty(E, dtype=torch.int32, device=dev)
        for m in ("LE", "GT"):
            ms, tot = timed(torch, lambda g=graphs[m]: g.decode_all_device(rp_d, cl_d,
                                                                           stream=stream),
                            args.steps, args.warmup, flush, dist, local)
            parity.decode(f"decode_{m}", os.path.join(gdir, m), m, rp_d, cl_d)
            stream_bytes = infos[m]["device_bytes"] - 16 * n  # the resident stream
            out[f"decode_{m}"] = {
                "value": sum_over_ranks(dist, E * args.steps, torch) / (tot / 1000.0),
                "unit": "decoded edges/s", "ms_per_step": tot / args.steps,
                "algorithmic_GBps": (stream_bytes + 16 * n + 4 * E + 8 * (n + 1))
                / (tot / args.steps) / 1e6}
        # LE sweep with its chunk slots staged through shared memory (cp.async.bulk)
        for depth in (1, 2, 4):
            graphs["LE"].set_tuning(decode_stage_depth=depth)
            ms, tot = timed(torch, lambda: graphs["LE"].decode_all_device(rp_d, cl_d,
                                                                          stream=stream),
                            args.steps, args.warmup, flush, dist, local)
            parity.decode(f"decode_LE_staged{depth}", os.path.join(gdir, "LE"), "LE", rp_d, cl_d)
            out[f"decode_LE_staged{depth}"] = {"ms_per_step": tot / args.steps,
                                               "value": E * args.steps / (tot / 1000.0)}
        graphs["LE"].set_tuning()
        # the allocation-free entry point on a graph without a decode plan
        # (its unplanned sweep), then with one (the planned sweep)
        import ctypes
        fresh = G.Graph(os.path.join(gdir, "LE"), "LE")
        st_ptr = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None

        def noalloc():
            rc = G.lib.grass_decode_all_noalloc(fresh.handle, ctypes.c_void_p(rp_d.data_ptr()),
                                                ctypes.c_void_p(cl_d.data_ptr()), st_ptr)
            assert rc == G.OK, G.last_error()

        ms, tot = timed(torch, noalloc, args.steps, args.warmup, flush, dist, local)
        parity.decode("decode_LE_noalloc_unplanned", os.path.join(gdir, "LE"), "LE", rp_d, cl_d)
        out["decode_LE_noalloc_unplanned"] = {"ms_per_step": tot / args.steps,
                                              "value": E * args.steps / (tot / 1000.0)}
        fresh.close()
        del rp_d, cl_d

    clk = clocks.stop()

    progress("batched jobs and serving")
    # ---- batched uneven jobs and the serving loop (R-MAT s24 ef16), 1 GPU runs
    if ws == 1 and ({"batch", "serve"} & only):
        bdir, bmeta = build_graph(args.batch_scale, 16)
        bgraphs = {m: G.Graph(os.path.join(bdir, m), m, device=local) for m in ("LE", "GT")}
        bn = bmeta["n"]
        extra = {"graph": f"R-MAT scale {args.batch_scale} edge factor 16 seed 42, graph_sort "
                          f"(undirected): "
                          f"{bn} vertices, {bmeta['num_edges']} directed edges"}
        if "batch" in only:
            progress("batch: 256-job mix, autotune + timed runs (LE, GT, CSR)")
            bcsr = bgraphs["LE"].csr()  # uncompressed baseline of the same graph
            extra["batch"] = batch_bench(G, torch, {**bgraphs, "CSR": bcsr}, bn, stream, flush,
                                         5, 3, parity, bdir)
            bcsr.close()
            del bcsr
        if "serve" in only:
            progress("serving: peak and latency sweeps")
            extra["serve"] = serve_bench(G, bgraphs[args.mode])
        out["batched_jobs_and_serving"] = extra
        del bgraphs

    # ---- the reference's own GPU rw app on this GPU: only when asked for
    if ws == 1 and rank == 0 and "refgpu" in only:
        out["reference_gpu"] = reference_gpu(gdir, n)
        g1dir, meta1 = build_graph(16, 16)
        out["reference_gpu"]["visits_rmat_s16"] = reference_visits(G, torch, g1dir, meta1["n"])
        out["reference_gpu"]["visits_rmat_s22"] = reference_visits(G, torch, gdir, n)

    # ---- skewed large graph (Chung-Lu, ~3B edges): only when asked for
    if ws == 1 and "cfg5" in only:
        out["chung_lu_100M"] = cfg5_bench(G, torch, stream, flush, 3, parity)

    progress("roofline accounting, random-read probe")
    # ---- accounting for the roofline of the headline kernel
    acct = torch.zeros(3, dtype=torch.int64, device=dev)
    graphs[args.mode].rw_account(starts, W, L, replica_seed(7, rank), acct, stream=stream)
    torch.cuda.synchronize()
    alg_bytes, sectors, draws = [int(x) for x in acct.cpu().tolist()]
    head = out[f"rw_{args.mode}"]
    avg_s = head["ms_per_step"] / 1000.0
    peak, peak_kind = peaks()
    achieved = alg_bytes / avg_s / 1e9
    traffic, traffic_src = ncu_traffic(f"rw_{args.mode}_s{args.scale}_e{args.edge_factor}_L{L}")
    # random-access context: 32-byte sectors a walk reads per second, beside
    # the rate of uniform random 4-byte reads over 2 GiB (no locality at all)
    ceil = random_sector_ceiling(G, torch, dev, flush) if "rw" in only else None
    rand = None
    if ceil:
        rand = {"uniform_random_reads_per_s": ceil["sectors_per_s"], "probe": ceil,
                f"{args.mode}_sectors_per_draw": sectors / max(draws, 1),
                f"{args.mode}_sectors_per_s": sectors / avg_s,
                "note": "walk sectors include L2 hits (vertex records, hub payloads); "
                        "uniform random reads have no locality, so they are not a ceiling"}
        if "rw_CSR" in out:  # a CSR draw reads the row-pointer pair's sector and the column's
            rand.update({"CSR_sectors_per_draw": 2.0,
                         "CSR_sectors_per_s": 2 * draws / (out["rw_CSR"]["ms_per_step"] / 1000.0)})

    progress("e2e")
    # ---- e2e through the host API, pinned buffers, copies inside the region
    e2e = None
    if "e2e" in only:
        h_starts = torch.empty(W, dtype=torch.int32, pin_memory=True)
        h_starts.copy_(starts.cpu())
        h_paths = torch.empty(W * (L + 1), dtype=torch.int32, pin_memory=True)
        hs = h_starts.numpy().view(np.uint32)
        hp = h_paths.numpy().view(np.uint32).reshape(W, L + 1)
        gm = graphs[args.mode]
        p = G.RwParams(L, LAYOUT, replica_seed(7, rank))
        import ctypes as C
        ecnt = C.c_uint64()

        def e2e_call():
            G._check(G.lib.grass_rw_host(gm.handle, C.byref(p), G._p(hs), W, G._p(hp),
                                         C.byref(ecnt)))
        for _ in range(args.warmup):
            e2e_call()
        barrier(dist, local)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_call()
        el = time.perf_counter() - t0
        barrier(dist, local)
        el = max_over_ranks(dist, el, torch)
        e2e = {"value": sum_over_ranks(dist, int(ecnt.value) * args.steps, torch) / el,
               "unit": UNIT, "h2d_bytes_per_step": W * 4, "d2h_bytes_per_step": W * (L + 1) * 4,
               "ms_per_step": 1000 * el / args.steps, "api": "grass_rw_host (pinned host buffers)"}

    cpu = None
    progress("cpu baseline")
    if rank == 0 and "cpu" in only:
        try:
            cpu = cpu_baseline(gdir, args.mode, n, L, 7)
        except Exception as ex:  # the oracle is test infrastructure; report, don't fail
            cpu = {"error": str(ex)}

    if rank == 0:
        csr_bytes = (n + 1) * 8 + 4 * E
        line = {
            "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (R-MAT generated on the box, seed 42)",
            "config": workload_config(args, meta),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": peak_kind,
                         "traffic": traffic, "traffic_capture": traffic_src,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "sector_bytes_per_launch": sectors * 32,
                         "sector_GBps": sectors * 32 / avg_s / 1e9,
                         "draws_per_launch": draws},
            "random_access": rand,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": head["launches"],
            "clocks": clk,
            "results": out,
            "compressed_vs_csr": ({m: out[f"rw_{m}"]["value"] / out["rw_CSR"]["value"]
                                   for m in ("LE", "GT")} if "rw_CSR" in out else None),
            "footprint_bytes": {"CSR": csr_bytes,
                                **{m: infos[m]["device_bytes"] for m in infos},
                                **{f"ratio_{m}": csr_bytes / infos[m]["device_bytes"]
                                   for m in infos}},
            "load_seconds": {m: infos[m]["upload_seconds"] for m in infos},
            "footprint_files": {f"ratio_{m}": csr_bytes / (infos[m]["graph_file_bytes"] +
                                                         infos[m]["offset_file_bytes"])
                                for m in infos},
            "footprint_config1": footprint_config1(G) if "footprint" in only else None,
            "parity": ({k: v["ok"] for k, v in parity.res.items()} if parity.enabled else None),
            "parity_detail": parity.res if parity.enabled else None,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    bad = [k for k, v in parity.res.items() if not v["ok"]]
    if bad:
        print(f"parity mismatch against the oracle: {', '.join(bad)}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
