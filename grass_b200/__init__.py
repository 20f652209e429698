"""grass_b200 -- B200-native compressed-graph sampling (GraSS hot path).

Python binding over the C ABI in ``include/grass.h`` (``lib/libgrass_b200.so``).
Everything here calls into the native library; there is no Python or CPU
fallback for any sampling or decoding operation, and importing the package
raises if the library has not been built.

Reference interface mirrored (calla212/GraSS):
  * ``Graph(prefix, mode)``      -- loadGraph + transferToGPUs (GT/src/grass.cu:1126-1233)
  * ``Graph.rw / khop / mrw``    -- the rw / ks / mrw apps (GT/src/apps/*)
  * ``Graph.decode_all``         -- GlobalDecoder / BCGVertex::get_vertex (GT/src/bcg.cuh)
  * ``compress``/``graph_sort``  -- GT|LE/chunk_compress (offline tools)
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# GRASS_LIB_PATH selects an alternative build of the same library (e.g. a
# build with other compile-time options); the default is the in-tree build.
LIB_PATH = os.environ.get("GRASS_LIB_PATH") or os.path.join(HERE, "lib", "libgrass_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include", "grass.h")

OK, E_IO, E_FORMAT, E_CUDA, E_OOM, E_BUDGET, E_TIMEOUT, E_ARG, E_DATA = range(9)
MODE_GT, MODE_LE = 0, 1
MODES = {"GT": MODE_GT, "LE": MODE_LE, "gt": MODE_GT, "le": MODE_LE, 0: 0, 1: 1}
INVALID = 0xFFFFFFFF
LAYOUT_WALK_MAJOR, LAYOUT_STEP_MAJOR = 0, 1
SELECT_UNIFORM, SELECT_DEGREE, SELECT_DEGREE_CT = 0, 1, 2
MAX_HOPS = 8


class GrassError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def build() -> None:
    import subprocess
    subprocess.check_call(["make", "-s", "-j8", "-C", os.path.join(HERE, "csrc"), "all"])


class GraphInfo(C.Structure):
    _fields_ = [
        ("n", C.c_uint64), ("n_file", C.c_uint64), ("num_edges", C.c_uint64),
        ("max_degree", C.c_uint32), ("ubl", C.c_uint32), ("mode", C.c_int32),
        ("device", C.c_int32), ("graph_file_bytes", C.c_uint64),
        ("offset_file_bytes", C.c_uint64), ("device_bytes", C.c_uint64),
        ("read_seconds", C.c_double), ("upload_seconds", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class RwParams(C.Structure):
    _fields_ = [("length", C.c_uint32), ("layout", C.c_uint32), ("seed", C.c_uint64)]


class Node2vecParams(C.Structure):
    _fields_ = [("length", C.c_uint32), ("layout", C.c_uint32), ("seed", C.c_uint64),
                ("p", C.c_double), ("q", C.c_double), ("max_tries", C.c_uint32),
                ("reserved", C.c_uint32 * 3)]


class KhopParams(C.Structure):
    _fields_ = [("hops", C.c_uint32), ("fanouts", C.c_uint32 * MAX_HOPS), ("seed", C.c_uint64)]


class Tuning(C.Structure):
    _fields_ = [("rw_depth", C.c_uint32), ("rw_threads", C.c_uint32),
                ("rw_blocks_per_sm", C.c_uint32), ("l2_persist", C.c_uint32),
                ("l2_fetch_bytes", C.c_uint32), ("decode_stage_depth", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]


class MrwParams(C.Structure):
    _fields_ = [("walkers", C.c_uint32), ("steps", C.c_uint32), ("select", C.c_uint32),
                ("reserved", C.c_uint32), ("seed", C.c_uint64)]


JOB_RW, JOB_KHOP, JOB_MRW = 0, 1, 2


class Job(C.Structure):
    _fields_ = [("type", C.c_uint32), ("count", C.c_uint32), ("seed", C.c_uint64),
                ("d_input", C.c_void_p), ("d_roots", C.c_void_p), ("d_out0", C.c_void_p),
                ("d_out1", C.c_void_p), ("d_hops", C.c_void_p * MAX_HOPS),
                ("d_edges", C.c_void_p), ("length", C.c_uint32), ("layout", C.c_uint32),
                ("hops", C.c_uint32), ("fanouts", C.c_uint32 * MAX_HOPS),
                ("walkers", C.c_uint32), ("steps", C.c_uint32), ("select", C.c_uint32)]


class BatchConfig(C.Structure):
    _fields_ = [("walker_tile", C.c_uint32), ("depth", C.c_uint32),
                ("warps_per_block", C.c_uint32), ("khop_seeds", C.c_uint32),
                ("use_graph", C.c_uint32), ("warps_per_vertex", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class ServerConfig(C.Structure):
    _fields_ = [("scratch_budget", C.c_uint64), ("target_draws", C.c_uint64),
                ("staging_bytes", C.c_uint64), ("window_min_us", C.c_uint32), ("window_max_us", C.c_uint32),
                ("max_inflight", C.c_uint32), ("max_batch_jobs", C.c_uint32),
                ("batch", BatchConfig), ("results_on_device", C.c_uint32),
                ("reserved", C.c_uint32 * 3)]


class Request(C.Structure):
    _fields_ = [("type", C.c_uint32), ("count", C.c_uint32), ("seed", C.c_uint64),
                ("input", C.c_void_p), ("length", C.c_uint32), ("layout", C.c_uint32),
                ("hops", C.c_uint32), ("fanouts", C.c_uint32 * MAX_HOPS),
                ("walkers", C.c_uint32), ("steps", C.c_uint32), ("select", C.c_uint32)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("n_outputs", C.c_uint32),
                ("out", C.c_void_p * MAX_HOPS), ("out_words", C.c_uint64 * MAX_HOPS),
                ("edges", C.c_uint64), ("submit_us", C.c_double), ("launch_us", C.c_double),
                ("done_us", C.c_double), ("batch", C.c_uint64), ("on_device", C.c_uint32),
                ("reserved", C.c_uint32)]


class ServerStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("submitted", "completed", "rejected", "failed",
                                          "batches", "edges", "waiting", "running",
                                          "scratch_in_use", "scratch_peak")] + \
               [("busy_us", C.c_double), ("issue_us", C.c_double),
                ("staging_alloc_us", C.c_double), ("phase_us", C.c_double * 6),
                ("staging_fallbacks", C.c_uint64)]

    def as_dict(self):
        return {k: list(getattr(self, k)) if k == "phase_us" else getattr(self, k)
                for k, _ in self._fields_}


class LoadgenConfig(C.Structure):
    _fields_ = [("rate", C.c_double), ("requests", C.c_uint32), ("mode", C.c_uint32),
                ("seed", C.c_uint64), ("pct_rw", C.c_uint32), ("pct_khop", C.c_uint32),
                ("size_mu", C.c_double), ("size_sigma", C.c_double), ("size_max", C.c_uint32),
                ("rw_len_min", C.c_uint32), ("rw_len_max", C.c_uint32),
                ("n_fanouts", C.c_uint32), ("fanouts", (C.c_uint32 * 4) * 8),
                ("mrw_samples", C.c_uint32), ("mrw_walkers", C.c_uint32),
                ("mrw_steps", C.c_uint32), ("mrw_select", C.c_uint32),
                ("timeout_ms", C.c_uint32), ("server", ServerConfig)]


class LoadgenReport(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("rejected", C.c_uint64), ("failed", C.c_uint64),
                ("batches", C.c_uint64), ("p50_us", C.c_double), ("p99_us", C.c_double),
                ("p999_us", C.c_double), ("mean_us", C.c_double), ("max_us", C.c_double),
                ("p50_type_us", C.c_double * 3), ("p99_type_us", C.c_double * 3),
                ("queue_p50_us", C.c_double), ("queue_p99_us", C.c_double),
                ("service_p50_us", C.c_double), ("service_p99_us", C.c_double),
                ("issue_us", C.c_double), ("staging_alloc_us", C.c_double),
                ("phase_us", C.c_double * 6),
                ("wall_s", C.c_double), ("edges", C.c_double), ("edges_per_s", C.c_double),
                ("offered_rate", C.c_double), ("achieved_rate", C.c_double),
                ("launches", C.c_uint64)]

    def as_dict(self):
        d = {}
        for k, _ in self._fields_:
            v = getattr(self, k)
            d[k] = list(v) if k.endswith("type_us") or k == "phase_us" else v
        return d


def _load():
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"grass_b200 native library not built ({LIB_PATH}); run "
            "`make -C grass_b200/csrc` or __graft_entry__.build()")
    L = C.CDLL(LIB_PATH)
    P, u32, u64, i32, d = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int, C.c_double
    PP = C.POINTER(C.c_void_p)
    sig = {
        "grass_last_error": ([], C.c_char_p),
        "grass_launch_count": ([], u64),
        "grass_version": ([], C.c_char_p),
        "grass_gen_rmat": ([u32, u32, d, d, d, u64, P, P], i32),
        "grass_gen_chung_lu": ([u64, d, d, u64, u64, u64, P, P], i32),
        "grass_graph_sort": ([P, P, u64, i32, PP], i32),
        "grass_host_csr_view": ([P, P, P, PP, PP], i32),
        "grass_host_csr_free": ([P], None),
        "grass_compress": ([P, P, u64, i32, P, P, P, P], i32),
        "grass_compress_to_files": ([P, P, u64, i32, C.c_char_p], i32),
        "grass_open": ([C.c_char_p, i32, i32, PP], i32),
        "grass_open_mem": ([P, u64, P, u64, i32, i32, PP], i32),
        "grass_close": ([P], i32),
        "grass_get_info": ([P, C.POINTER(GraphInfo)], i32),
        "grass_check_device_error": ([P, P], i32),
        "grass_device_view": ([P, PP, P, PP], i32),
        "grass_set_tuning": ([P, C.POINTER(Tuning)], i32),
        "grass_get_tuning": ([P, C.POINTER(Tuning)], i32),
        "grass_csr_set_tuning": ([P, C.POINTER(Tuning)], i32),
        "grass_degrees": ([P, P, P], i32),
        "grass_decode_all": ([P, P, P, P], i32),
        "grass_decode_all_noalloc": ([P, P, P, P], i32),
        "grass_uniform_starts": ([u64, u64, u64, P, P], i32),
        "grass_rw": ([P, C.POINTER(RwParams), P, u64, P, P, P], i32),
        "grass_node2vec": ([P, C.POINTER(Node2vecParams), P, u64, P, P, P], i32),
        "grass_csr_node2vec": ([P, C.POINTER(Node2vecParams), P, u64, P, P, P], i32),
        "grass_rw_host": ([P, C.POINTER(RwParams), P, u64, P, P], i32),
        "grass_rw_account": ([P, C.POINTER(RwParams), P, u64, P, P], i32),
        "grass_random_read_probe": ([P, u64, u64, u64, P, C.POINTER(u64), P], i32),
        "grass_khop": ([P, C.POINTER(KhopParams), P, u64, P, P, P], i32),
        "grass_khop_host": ([P, C.POINTER(KhopParams), P, u64, P, P], i32),
        "grass_mrw": ([P, C.POINTER(MrwParams), P, u64, P, P, P, P], i32),
        "grass_mrw_host": ([P, C.POINTER(MrwParams), P, u64, P, P, P], i32),
        "grass_csr_from_graph": ([P, PP], i32),
        "grass_csr_from_host": ([P, P, u64, i32, PP], i32),
        "grass_csr_close": ([P], i32),
        "grass_csr_info": ([P, P, P, P], i32),
        "grass_csr_rw": ([P, C.POINTER(RwParams), P, u64, P, P, P], i32),
        "grass_csr_khop": ([P, C.POINTER(KhopParams), P, u64, P, P, P], i32),
        "grass_mrw_roots": ([u64, u64, u32, u64, P, P], i32),
        "grass_khop_edges": ([C.POINTER(KhopParams), P, u64, P, P, P, u64, P, P], i32),
        "grass_rw_edges": ([C.POINTER(RwParams), P, u64, P, P, u64, P, P], i32),
        "grass_mrw_edges": ([C.POINTER(MrwParams), u64, P, P, P, P, u64, P, P], i32),
        "grass_batch_create": ([P, PP], i32),
        "grass_batch_create_csr": ([P, PP], i32),
        "grass_batch_add": ([P, C.POINTER(Job)], i32),
        "grass_batch_clear": ([P], i32),
        "grass_batch_set_config": ([P, C.POINTER(BatchConfig)], i32),
        "grass_batch_get_config": ([P, C.POINTER(BatchConfig)], i32),
        "grass_batch_run": ([P, P, P], i32),
        "grass_batch_autotune": ([P, P, C.POINTER(BatchConfig), C.POINTER(C.c_float)], i32),
        "grass_batch_info": ([P, P, P], i32),
        "grass_batch_destroy": ([P], i32),
        "grass_server_create": ([P, C.POINTER(ServerConfig), PP], i32),
        "grass_server_submit": ([P, C.POINTER(Request), C.POINTER(u64)], i32),
        "grass_server_poll": ([P, u64, C.POINTER(i32)], i32),
        "grass_server_wait": ([P, u64, u32, C.POINTER(Result)], i32),
        "grass_server_release": ([P, u64], i32),
        "grass_server_stats_get": ([P, C.POINTER(ServerStats)], i32),
        "grass_server_destroy": ([P, u32], i32),
        "grass_loadgen_run": ([P, C.POINTER(LoadgenConfig), C.POINTER(LoadgenReport)], i32),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    return L


lib = _load()


def last_error() -> str:
    return (lib.grass_last_error() or b"").decode()


def launch_count() -> int:
    return int(lib.grass_launch_count())


def _check(rc: int):
    if rc != OK:
        raise GrassError(rc, last_error())


def _p(a: np.ndarray):
    return C.c_void_p(a.ctypes.data)


def _ptr(x):
    """Device pointer from an int, a torch tensor or None."""
    if x is None:
        return None
    if isinstance(x, int):
        return C.c_void_p(x)
    return C.c_void_p(x.data_ptr())


def _stream(s):
    if s is None:
        return None
    if isinstance(s, int):
        return C.c_void_p(s)
    return C.c_void_p(s.cuda_stream)


# ---------------------------------------------------------------------------
# Host graph tools

def gen_rmat(scale: int, edge_factor: int, a=0.57, b=0.19, c=0.19, seed: int = 42):
    m = edge_factor << scale
    src = np.empty(m, dtype=np.uint32)
    dst = np.empty(m, dtype=np.uint32)
    _check(lib.grass_gen_rmat(scale, edge_factor, a, b, c, seed, _p(src), _p(dst)))
    return src, dst


def gen_chung_lu(n: int, exponent: float, mean_degree: float, max_degree: int, m: int,
                 seed: int = 42):
    src = np.empty(m, dtype=np.uint32)
    dst = np.empty(m, dtype=np.uint32)
    _check(lib.grass_gen_chung_lu(n, exponent, mean_degree, max_degree, seed, m, _p(src),
                                  _p(dst)))
    return src, dst


def graph_sort(src: np.ndarray, dst: np.ndarray, directed: bool = False):
    """graph_sort semantics; returns (rowptr u64[n+1], cols u32[nnz])."""
    src = np.ascontiguousarray(src, dtype=np.uint32)
    dst = np.ascontiguousarray(dst, dtype=np.uint32)
    h = C.c_void_p()
    _check(lib.grass_graph_sort(_p(src), _p(dst), len(src), int(directed), C.byref(h)))
    try:
        n, nnz = C.c_uint64(), C.c_uint64()
        rp, cp = C.c_void_p(), C.c_void_p()
        _check(lib.grass_host_csr_view(h, C.byref(n), C.byref(nnz), C.byref(rp), C.byref(cp)))
        rowptr = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_uint64)),
                                       shape=(n.value + 1,)).copy()
        cols = (np.ctypeslib.as_array(C.cast(cp, C.POINTER(C.c_uint32)), shape=(nnz.value,)).copy()
                if nnz.value else np.zeros(0, np.uint32))
    finally:
        lib.grass_host_csr_free(h)
    return rowptr, cols


def compress(rowptr: np.ndarray, cols: np.ndarray, mode) -> tuple[bytes, bytes]:
    """Encode a sorted CSR in the reference's GT or LE on-disk format."""
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    n = len(rowptr) - 1
    gs, os_ = C.c_uint64(), C.c_uint64()
    m = MODES[mode]
    cptr = _p(cols) if len(cols) else None
    _check(lib.grass_compress(_p(rowptr), cptr, n, m, None, C.byref(gs), None, C.byref(os_)))
    gb = np.zeros(max(gs.value, 1), np.uint8)
    ob = np.zeros(os_.value, np.uint8)
    _check(lib.grass_compress(_p(rowptr), cptr, n, m, _p(gb), C.byref(gs), _p(ob), C.byref(os_)))
    return gb[: gs.value].tobytes(), ob.tobytes()


def compress_to_files(rowptr: np.ndarray, cols: np.ndarray, mode, prefix: str) -> None:
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    _check(lib.grass_compress_to_files(_p(rowptr), _p(cols) if len(cols) else None,
                                       len(rowptr) - 1, MODES[mode], prefix.encode()))


def rmat_graph(scale: int, edge_factor: int, seed: int = 42, a=0.57, b=0.19, c=0.19):
    """R-MAT -> graph_sort (undirected) CSR."""
    src, dst = gen_rmat(scale, edge_factor, a, b, c, seed)
    return graph_sort(src, dst, directed=False)


# ---------------------------------------------------------------------------
# Device graph

def _khop_params(fanouts, seed):
    p = KhopParams()
    fanouts = list(fanouts)
    if not 1 <= len(fanouts) <= MAX_HOPS:
        raise ValueError("1..8 hops")
    p.hops = len(fanouts)
    for i, f in enumerate(fanouts):
        p.fanouts[i] = int(f)
    p.seed = seed
    return p


def hop_widths(fanouts):
    out, w = [], 1
    for f in fanouts:
        w *= int(f)
        out.append(w)
    return out


class Graph:
    """A compressed graph resident on one GPU."""

    def __init__(self, prefix: str | None = None, mode="GT", device: int = 0, *,
                 graph_bytes: bytes | None = None, offset_bytes: bytes | None = None):
        self._h = C.c_void_p()
        m = mode if isinstance(mode, int) else MODES[mode]
        if prefix is not None:
            _check(lib.grass_open(prefix.encode(), m, device, C.byref(self._h)))
        else:
            gb = np.frombuffer(graph_bytes, np.uint8) if graph_bytes else np.zeros(1, np.uint8)
            ob = np.frombuffer(offset_bytes, np.uint8)
            _check(lib.grass_open_mem(_p(gb), len(graph_bytes or b""), _p(ob), len(ob), m, device,
                                      C.byref(self._h)))
        self.mode = m

    @classmethod
    def from_bytes(cls, graph_bytes: bytes, offset_bytes: bytes, mode="GT", device: int = 0):
        return cls(None, mode, device, graph_bytes=graph_bytes, offset_bytes=offset_bytes)

    def close(self):
        if self._h:
            lib.grass_close(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def info(self) -> dict:
        i = GraphInfo()
        _check(lib.grass_get_info(self._h, C.byref(i)))
        return i.as_dict()

    @property
    def n(self) -> int:
        return int(self.info()["n"])

    def set_tuning(self, rw_depth=0, rw_threads=0, rw_blocks_per_sm=0, l2_persist=0,
                   l2_fetch_bytes=0, decode_stage_depth=0):
        t = Tuning(rw_depth, rw_threads, rw_blocks_per_sm, l2_persist, l2_fetch_bytes,
                   decode_stage_depth)
        _check(lib.grass_set_tuning(self._h, C.byref(t)))

    def tuning(self) -> dict:
        t = Tuning()
        _check(lib.grass_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_ if k != "reserved"}

    # -- host-buffer (end-to-end) calls --
    def rw(self, starts: np.ndarray, length: int, seed: int, layout: int = LAYOUT_WALK_MAJOR):
        starts = np.ascontiguousarray(starts, dtype=np.uint32)
        W = len(starts)
        p = RwParams(length, layout, seed)
        shape = (W, length + 1) if layout == LAYOUT_WALK_MAJOR else (length + 1, W)
        paths = np.zeros(shape, dtype=np.uint32)
        e = C.c_uint64()
        _check(lib.grass_rw_host(self._h, C.byref(p), _p(starts), W, _p(paths), C.byref(e)))
        return paths, int(e.value)

    def khop(self, seeds: np.ndarray, fanouts, seed: int):
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        p = _khop_params(fanouts, seed)
        outs = [np.zeros((len(seeds), w), dtype=np.uint32) for w in hop_widths(fanouts)]
        arr = (C.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        e = C.c_uint64()
        _check(lib.grass_khop_host(self._h, C.byref(p), _p(seeds), len(seeds),
                                   C.cast(arr, C.c_void_p), C.byref(e)))
        return outs, int(e.value)

    def mrw(self, roots: np.ndarray, steps: int, seed: int, select: int = SELECT_UNIFORM):
        roots = np.array(roots, dtype=np.uint32, order="C", copy=True)
        S, R = roots.shape
        p = MrwParams(R, steps, select, 0, seed)
        src = np.zeros((S, steps), np.uint32)
        dst = np.zeros((S, steps), np.uint32)
        e = C.c_uint64()
        _check(lib.grass_mrw_host(self._h, C.byref(p), _p(roots), S, _p(src), _p(dst),
                                  C.byref(e)))
        return src, dst, roots, int(e.value)

    # -- device-buffer calls (torch tensors or raw ints) --
    def rw_device(self, starts, W: int, length: int, seed: int, paths, edge_count=None,
                  layout: int = LAYOUT_WALK_MAJOR, stream=None):
        p = RwParams(length, layout, seed)
        _check(lib.grass_rw(self._h, C.byref(p), _ptr(starts), W, _ptr(paths), _ptr(edge_count),
                            _stream(stream)))

    def node2vec_device(self, starts, W: int, length: int, seed: int, p: float, q: float,
                        paths, edge_count=None, max_tries: int = 0,
                        layout: int = LAYOUT_WALK_MAJOR, stream=None):
        prm = Node2vecParams(length, layout, seed, p, q, max_tries)
        _check(lib.grass_node2vec(self._h, C.byref(prm), _ptr(starts), W, _ptr(paths),
                                  _ptr(edge_count), _stream(stream)))

    def rw_account(self, starts, W: int, length: int, seed: int, out3, stream=None):
        """Adds [algorithmic bytes, 32B sectors, draws] of the walk to out3."""
        p = RwParams(length, 0, seed)
        _check(lib.grass_rw_account(self._h, C.byref(p), _ptr(starts), W, _ptr(out3),
                                    _stream(stream)))

    def khop_device(self, seeds, S: int, fanouts, seed: int, hop_out, edge_count=None,
                    stream=None):
        p = _khop_params(fanouts, seed)
        arr = (C.c_void_p * len(hop_out))(*[_ptr(o).value for o in hop_out])
        _check(lib.grass_khop(self._h, C.byref(p), _ptr(seeds), S, C.cast(arr, C.c_void_p),
                              _ptr(edge_count), _stream(stream)))

    def mrw_device(self, roots, S: int, walkers: int, steps: int, seed: int, src, dst,
                   select: int = SELECT_UNIFORM, edge_count=None, stream=None):
        p = MrwParams(walkers, steps, select, 0, seed)
        _check(lib.grass_mrw(self._h, C.byref(p), _ptr(roots), S, _ptr(src), _ptr(dst),
                             _ptr(edge_count), _stream(stream)))

    def check_device_error(self, stream=None):
        """Wait for the stream, then raise GrassError if a device-pointer call
        flagged an error on this graph (GRASS_E_DATA / GRASS_E_TIMEOUT)."""
        _check(lib.grass_check_device_error(self._h, _stream(stream)))

    def decode_all_device(self, rowptr, cols, stream=None):
        _check(lib.grass_decode_all(self._h, _ptr(rowptr), _ptr(cols), _stream(stream)))

    def degrees_device(self, deg, stream=None):
        _check(lib.grass_degrees(self._h, _ptr(deg), _stream(stream)))

    def decode_all(self):
        """Decode every list; returns host (rowptr, cols).  Uses torch for buffers."""
        import torch
        inf = self.info()
        n, E = int(inf["n"]), int(inf["num_edges"])
        dev = torch.device("cuda", int(inf["device"]))
        rp = torch.empty(n + 1, dtype=torch.int64, device=dev)
        cl = torch.empty(max(E, 1), dtype=torch.int32, device=dev)
        self.decode_all_device(rp, cl)
        torch.cuda.synchronize(dev)
        return (rp.cpu().numpy().view(np.uint64).copy(),
                cl.cpu().numpy().view(np.uint32)[:E].copy())

    def csr(self) -> "Csr":
        h = C.c_void_p()
        _check(lib.grass_csr_from_graph(self._h, C.byref(h)))
        return Csr(h)


def random_read_probe(buf, n_words: int, reads: int, seed: int, sink, stream=None) -> int:
    """About `reads` independent random 4-byte reads from buf[0, n_words); returns
    the number issued (the device's random-read ceiling when timed)."""
    k = C.c_uint64()
    _check(lib.grass_random_read_probe(_ptr(buf), n_words, reads, seed, _ptr(sink), C.byref(k),
                                       _stream(stream)))
    return int(k.value)


def mrw_roots_device(n: int, S: int, R: int, seed: int, out, stream=None):
    _check(lib.grass_mrw_roots(n, S, R, seed, _ptr(out), _stream(stream)))


# -- output compaction: fixed-shape sampler outputs to dense edge lists --
# Each call writes the valid edges (dst not INVALID_VERTEX) in output order to
# src/dst[0, capacity) and their total to count[0] (a device u64).

def khop_edges_device(seeds, S: int, fanouts, hop_out, src, dst, capacity: int, count,
                      stream=None):
    """k-hop edges in (hop, seed, slot) order."""
    p = _khop_params(fanouts, 0)
    arr = (C.c_void_p * len(hop_out))(*[None if o is None else _ptr(o).value for o in hop_out])
    _check(lib.grass_khop_edges(C.byref(p), _ptr(seeds), S, C.cast(arr, C.c_void_p), _ptr(src),
                                _ptr(dst), capacity, _ptr(count), _stream(stream)))


def rw_edges_device(paths, W: int, length: int, src, dst, capacity: int, count,
                    layout: int = LAYOUT_WALK_MAJOR, stream=None):
    """Walk edges in (walk, step) order (walk-major) or (step, walk) order."""
    p = RwParams(length, layout, 0)
    _check(lib.grass_rw_edges(C.byref(p), _ptr(paths), W, _ptr(src), _ptr(dst), capacity,
                              _ptr(count), _stream(stream)))


def mrw_edges_device(step_src, step_dst, S: int, steps: int, src, dst, capacity: int, count,
                     stream=None):
    """Multi-RW step edges in (sample, step) order."""
    p = MrwParams(0, steps, 0, 0, 0)
    _check(lib.grass_mrw_edges(C.byref(p), S, _ptr(step_src), _ptr(step_dst), _ptr(src),
                               _ptr(dst), capacity, _ptr(count), _stream(stream)))


class Batch:
    """Many RW / k-hop / multi-RW jobs run by one persistent, graph-captured launch."""

    def __init__(self, graph):
        """graph: a Graph (compressed) or a Csr (uncompressed baseline)."""
        self._g = graph  # keep the graph alive
        self._h = C.c_void_p()
        self._keep = []
        if isinstance(graph, Csr):
            _check(lib.grass_batch_create_csr(graph._h, C.byref(self._h)))
        else:
            _check(lib.grass_batch_create(graph.handle, C.byref(self._h)))

    def _add(self, job: Job):
        _check(lib.grass_batch_add(self._h, C.byref(job)))

    def add_rw(self, starts, count: int, length: int, seed: int, paths,
               layout: int = LAYOUT_WALK_MAJOR, edges=None):
        j = Job(type=JOB_RW, count=count, seed=seed, length=length, layout=layout)
        j.d_input, j.d_out0, j.d_edges = _ptr(starts), _ptr(paths), _ptr(edges)
        self._add(j)

    def add_khop(self, seeds, count: int, fanouts, seed: int, hop_out, edges=None):
        j = Job(type=JOB_KHOP, count=count, seed=seed, hops=len(fanouts))
        j.d_input, j.d_edges = _ptr(seeds), _ptr(edges)
        for h, f in enumerate(fanouts):
            j.fanouts[h] = int(f)
            j.d_hops[h] = _ptr(hop_out[h]).value
        self._add(j)

    def add_mrw(self, roots, count: int, walkers: int, steps: int, seed: int, src, dst,
                select: int = SELECT_UNIFORM, edges=None):
        j = Job(type=JOB_MRW, count=count, seed=seed, walkers=walkers, steps=steps, select=select)
        j.d_roots, j.d_out0, j.d_out1, j.d_edges = _ptr(roots), _ptr(src), _ptr(dst), _ptr(edges)
        self._add(j)

    def set_config(self, **kw):
        c = BatchConfig(**kw)
        _check(lib.grass_batch_set_config(self._h, C.byref(c)))

    def config(self) -> dict:
        c = BatchConfig()
        _check(lib.grass_batch_get_config(self._h, C.byref(c)))
        return c.as_dict()

    def run(self, stream=None, total=None):
        _check(lib.grass_batch_run(self._h, _stream(stream), _ptr(total)))

    def autotune(self, stream=None):
        c, ms = BatchConfig(), C.c_float()
        _check(lib.grass_batch_autotune(self._h, _stream(stream), C.byref(c), C.byref(ms)))
        return c.as_dict(), float(ms.value)

    def info(self):
        j, w = C.c_uint64(), C.c_uint64()
        _check(lib.grass_batch_info(self._h, C.byref(j), C.byref(w)))
        return {"jobs": j.value, "work_items": w.value}

    def close(self):
        if self._h:
            lib.grass_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _device_u32(ptr: int, n: int) -> np.ndarray:
    """Host copy of n uint32 at a device address (a server result kept on the GPU)."""
    import torch

    class _View:
        __cuda_array_interface__ = {"shape": (n,), "typestr": "<i4", "data": (ptr, False),
                                    "version": 3}
    return torch.as_tensor(_View(), device="cuda").cpu().numpy().view(np.uint32)


def _request(type_, count, seed, inp, **kw) -> tuple[Request, object]:
    r = Request(type=type_, count=count, seed=seed)
    keep = None
    if inp is not None:
        keep = np.ascontiguousarray(inp, dtype=np.uint32)
        r.input = keep.ctypes.data
    for k, v in kw.items():
        if k == "fanouts":
            r.hops = len(v)
            for h, f in enumerate(v):
                r.fanouts[h] = int(f)
        else:
            setattr(r, k, v)
    return r, keep


class Server:
    """Serving loop over a resident graph: submit requests from any thread,
    a dispatcher batches them into persistent launches."""

    def __init__(self, graph: "Graph", **cfg):
        self._g = graph
        self._h = C.c_void_p()
        c = ServerConfig()
        for k, v in cfg.items():
            if k == "batch":
                c.batch = BatchConfig(**v)
            else:
                setattr(c, k, v)
        _check(lib.grass_server_create(graph.handle, C.byref(c), C.byref(self._h)))

    def submit(self, r: Request) -> int:
        t = C.c_uint64()
        _check(lib.grass_server_submit(self._h, C.byref(r), C.byref(t)))
        return t.value

    def submit_rw(self, starts, length: int, seed: int, layout: int = LAYOUT_WALK_MAJOR) -> int:
        r, _ = _request(JOB_RW, len(starts), seed, starts, length=length, layout=layout)
        return self.submit(r)

    def submit_khop(self, seeds, fanouts, seed: int) -> int:
        r, _ = _request(JOB_KHOP, len(seeds), seed, seeds, fanouts=fanouts)
        return self.submit(r)

    def submit_mrw(self, samples: int, walkers: int, steps: int, seed: int,
                   select: int = SELECT_UNIFORM, roots=None) -> int:
        r, _ = _request(JOB_MRW, samples, seed, roots, walkers=walkers, steps=steps,
                        select=select)
        return self.submit(r)

    def poll(self, ticket: int) -> bool:
        d = C.c_int()
        _check(lib.grass_server_poll(self._h, ticket, C.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int, timeout_ms: int = 60000, release: bool = True) -> dict:
        """Result as {'outputs': [np.uint32 arrays], 'edges', 'submit_us', ...}."""
        res = Result()
        rc = lib.grass_server_wait(self._h, ticket, timeout_ms, C.byref(res))
        if rc == E_TIMEOUT:
            raise GrassError(rc, last_error())
        out = {"status": res.status, "edges": res.edges, "submit_us": res.submit_us,
               "launch_us": res.launch_us, "done_us": res.done_us, "batch": res.batch,
               "outputs": []}
        out["on_device"] = bool(res.on_device)
        for k in range(res.n_outputs):
            n = res.out_words[k]
            if not n:
                out["outputs"].append(np.zeros(0, np.uint32))
            elif res.on_device:  # device memory: copy out through torch
                out["outputs"].append(_device_u32(res.out[k], n))
            else:
                buf = (C.c_uint32 * n).from_address(res.out[k])
                out["outputs"].append(np.ctypeslib.as_array(buf).copy())
        if release:
            _check(lib.grass_server_release(self._h, ticket))
        _check(rc)
        return out

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib.grass_server_stats_get(self._h, C.byref(s)))
        return s.as_dict()

    def close(self, timeout_ms: int = 60000):
        if self._h:
            _check(lib.grass_server_destroy(self._h, timeout_ms))
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# Request mix of the batched-jobs workload: 40% RW with length U[10, 100],
# 40% k-hop with fanouts from {(10,5), (15,10), (25,10), (5,5,5)}, 20%
# multi-RW (one sample of 2000 walkers, 10,000 steps, degree-proportional in
# continuous time);
# RW walkers and k-hop seeds ~ lognormal(ln 1024, 1.5) clipped to [1, 65536].
MIX_FANOUTS = [(10, 5), (15, 10), (25, 10), (5, 5, 5)]


def loadgen(graph: "Graph", rate: float, requests: int, mode: int = 0, seed: int = 1,
            pct_rw: int = 40, pct_khop: int = 40, size_mu: float = math.log(1024),
            size_sigma: float = 1.5, size_max: int = 65536, rw_len=(10, 100),
            fanouts=MIX_FANOUTS, mrw_samples: int = 1, mrw_walkers: int = 2000,
            mrw_steps: int = 10000, mrw_select: int = SELECT_DEGREE_CT, timeout_ms: int = 0,
            **server) -> dict:
    """Open-loop Poisson run of the request mix; mode 0 batched server,
    mode 1 one standalone launch per request."""
    c = LoadgenConfig(rate=rate, requests=requests, mode=mode, seed=seed, pct_rw=pct_rw,
                      pct_khop=pct_khop, size_mu=size_mu, size_sigma=size_sigma,
                      size_max=size_max, rw_len_min=rw_len[0], rw_len_max=rw_len[1],
                      n_fanouts=len(fanouts), mrw_samples=mrw_samples,
                      mrw_walkers=mrw_walkers, mrw_steps=mrw_steps, mrw_select=mrw_select,
                      timeout_ms=timeout_ms)
    for i, f in enumerate(fanouts):
        for h, x in enumerate(f):
            c.fanouts[i][h] = int(x)
    for k, v in server.items():
        if k == "batch":
            c.server.batch = BatchConfig(**v)
        else:
            setattr(c.server, k, v)
    r = LoadgenReport()
    _check(lib.grass_loadgen_run(graph.handle, C.byref(c), C.byref(r)))
    return r.as_dict()


def uniform_starts_device(n: int, count: int, seed: int, out, stream=None):
    _check(lib.grass_uniform_starts(n, count, seed, _ptr(out), _stream(stream)))


class Csr:
    """Uncompressed CSR on one GPU (comparison baseline)."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_host(cls, rowptr: np.ndarray, cols: np.ndarray, device: int = 0):
        rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        h = C.c_void_p()
        _check(lib.grass_csr_from_host(_p(rowptr), _p(cols) if len(cols) else None,
                                       len(rowptr) - 1, device, C.byref(h)))
        return cls(h)

    def close(self):
        if self._h:
            lib.grass_csr_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_tuning(self, rw_depth=0, rw_threads=0, rw_blocks_per_sm=0, l2_persist=0,
                   l2_fetch_bytes=0):
        t = Tuning(rw_depth, rw_threads, rw_blocks_per_sm, l2_persist, l2_fetch_bytes)
        _check(lib.grass_csr_set_tuning(self._h, C.byref(t)))

    def info(self):
        n, nnz, b = C.c_uint64(), C.c_uint64(), C.c_uint64()
        _check(lib.grass_csr_info(self._h, C.byref(n), C.byref(nnz), C.byref(b)))
        return {"n": n.value, "nnz": nnz.value, "device_bytes": b.value}

    def node2vec_device(self, starts, W: int, length: int, seed: int, p: float, q: float,
                        paths, edge_count=None, max_tries: int = 0,
                        layout: int = LAYOUT_WALK_MAJOR, stream=None):
        prm = Node2vecParams(length, layout, seed, p, q, max_tries)
        _check(lib.grass_csr_node2vec(self._h, C.byref(prm), _ptr(starts), W, _ptr(paths),
                                      _ptr(edge_count), _stream(stream)))

    def rw_device(self, starts, W: int, length: int, seed: int, paths, edge_count=None,
                  layout: int = LAYOUT_WALK_MAJOR, stream=None):
        p = RwParams(length, layout, seed)
        _check(lib.grass_csr_rw(self._h, C.byref(p), _ptr(starts), W, _ptr(paths),
                                _ptr(edge_count), _stream(stream)))

    def khop_device(self, seeds, S: int, fanouts, seed: int, hop_out, edge_count=None,
                    stream=None):
        p = _khop_params(fanouts, seed)
        arr = (C.c_void_p * len(hop_out))(*[_ptr(o).value for o in hop_out])
        _check(lib.grass_csr_khop(self._h, C.byref(p), _ptr(seeds), S, C.cast(arr, C.c_void_p),
                                  _ptr(edge_count), _stream(stream)))


def exported_symbols() -> list[str]:
    """Function names declared in include/grass.h."""
    import re
    txt = open(INCLUDE).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(grass_[a-z0-9_]+)\s*\(", txt)))
