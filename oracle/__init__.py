"""CPU oracle for the compressed-graph sampling path -- TEST INFRASTRUCTURE ONLY.

This package is the checker.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import it; the product library never does.
It binds ``build/liboracle.so`` (a C restatement of the reference's decoders
and app ``next()`` logic, see ``grass_oracle.h``) and, where it was built,
``_ref/`` (the reference's own compressor, ``graph_sort`` and ``bcg.cuh``
decoder compiled for the host from the reference sources).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

MODE_GT = 0
MODE_LE = 1
MODES = {"GT": MODE_GT, "LE": MODE_LE, "gt": MODE_GT, "le": MODE_LE}
INVALID = 0xFFFFFFFF


def build(ref: bool = True) -> None:
    """Compile the oracle and, with ref, the reference's CPU pieces (the
    Makefile's `ref` target builds them where the reference sources are
    found, GRASS_REFERENCE, and does nothing otherwise)."""
    subprocess.check_call(["make", "-s", "-C", HERE, "all"])
    if ref:
        subprocess.check_call(["make", "-s", "-C", HERE, "ref"])


class _OgGraph(C.Structure):
    _fields_ = [
        ("words", C.POINTER(C.c_uint32)),
        ("n_words", C.c_uint64),
        ("offsets", C.POINTER(C.c_uint64)),
        ("n", C.c_uint32),
        ("n_file", C.c_uint32),
        ("ubl", C.c_uint32),
        ("graph_bits", C.c_uint64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref=False)
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        u32, u64, i32 = C.c_uint32, C.c_uint64, C.c_int
        G = C.POINTER(_OgGraph)
        L.og_load.argtypes = [C.c_char_p, G]
        L.og_load_mem.argtypes = [P, u64, P, u64, G]
        L.og_free.argtypes = [G]
        L.og_degree.argtypes = [G, i32, u32]
        L.og_degree.restype = u32
        L.og_get_vertex.argtypes = [G, i32, u32, u32]
        L.og_get_vertex.restype = u32
        L.og_degrees.argtypes = [G, i32, P, i32]
        L.og_decode_all.argtypes = [G, i32, P, P, i32]
        L.og_philox4x32_10.argtypes = [u32, u32, P, P]
        L.og_uniform_starts.argtypes = [u32, u64, u64, P]
        L.og_rw.argtypes = [G, i32, P, u64, u32, u64, P, i32]
        L.og_rw.restype = u64
        L.og_rw_csr.argtypes = [P, P, u32, P, u64, u32, u64, P, i32]
        L.og_rw_csr.restype = u64
        L.og_node2vec.argtypes = [G, i32, P, u64, u32, u64, C.c_double, C.c_double, u32, P,
                                  i32]
        L.og_node2vec.restype = u64
        L.og_khop.argtypes = [G, i32, P, u64, P, i32, u64, P, i32]
        L.og_khop.restype = u64
        L.og_mrw.argtypes = [G, i32, P, u64, u32, u32, u64, i32, P, P, i32]
        L.og_mrw.restype = u64
        L.og_mrw_roots.argtypes = [u32, u64, u32, u64, P]
        L.og_max_threads.restype = i32
        L.og_det_log.argtypes = [C.c_double]
        L.og_det_log.restype = C.c_double
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def det_log(u: float) -> float:
    """ln u for u in (0, 1) with the exact operation sequence of the device."""
    return float(lib().og_det_log(u))


def max_threads() -> int:
    return int(lib().og_max_threads())


def philox(key: int, ctr) -> np.ndarray:
    c = np.asarray(ctr, dtype=np.uint32)
    out = np.zeros(4, dtype=np.uint32)
    lib().og_philox4x32_10(key & 0xFFFFFFFF, (key >> 32) & 0xFFFFFFFF, _p(c), _p(out))
    return out


def uniform_starts(n: int, count: int, seed: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint32)
    lib().og_uniform_starts(n, count, seed, _p(out))
    return out


def mrw_roots(n: int, S: int, R: int, seed: int) -> np.ndarray:
    out = np.zeros((S, R), dtype=np.uint32)
    lib().og_mrw_roots(n, S, R, seed, _p(out))
    return out


class OracleGraph:
    """A compressed graph loaded by the oracle (reference loader semantics)."""

    def __init__(self, prefix: str | None = None, graph_bytes: bytes | None = None,
                 offset_bytes: bytes | None = None):
        self._g = _OgGraph()
        L = lib()
        if prefix is not None:
            rc = L.og_load(prefix.encode(), C.byref(self._g))
        else:
            gb = np.frombuffer(graph_bytes, dtype=np.uint8) if graph_bytes else np.zeros(1, np.uint8)
            ob = np.frombuffer(offset_bytes, dtype=np.uint8)
            rc = L.og_load_mem(_p(gb), len(graph_bytes), _p(ob), len(offset_bytes),
                               C.byref(self._g))
        if rc != 0:
            raise ValueError(f"oracle load failed (code {rc})")

    def __del__(self):
        try:
            lib().og_free(C.byref(self._g))
        except Exception:
            pass

    @property
    def n(self) -> int:
        return int(self._g.n)

    @property
    def n_file(self) -> int:
        return int(self._g.n_file)

    @property
    def ubl(self) -> int:
        return int(self._g.ubl)

    def offsets(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._g.offsets, shape=(self.n + 1,)).copy()

    def words(self) -> np.ndarray:
        return np.ctypeslib.as_array(self._g.words, shape=(int(self._g.n_words) + 2,)).copy()

    def degree(self, mode, v: int) -> int:
        return int(lib().og_degree(C.byref(self._g), MODES.get(mode, mode), v))

    def get_vertex(self, mode, v: int, i: int) -> int:
        return int(lib().og_get_vertex(C.byref(self._g), MODES.get(mode, mode), v, i))

    def degrees(self, mode, threads: int = 0) -> np.ndarray:
        out = np.zeros(self.n, dtype=np.uint32)
        rc = lib().og_degrees(C.byref(self._g), MODES.get(mode, mode), _p(out), threads)
        if rc:
            raise ValueError(f"malformed header (code {rc})")
        return out

    def decode_all(self, mode, threads: int = 0):
        m = MODES.get(mode, mode)
        rowptr = np.zeros(self.n + 1, dtype=np.uint64)
        rc = lib().og_decode_all(C.byref(self._g), m, _p(rowptr), None, threads)
        if rc:
            raise ValueError(f"decode failed (code {rc})")
        cols = np.zeros(max(int(rowptr[-1]), 1), dtype=np.uint32)
        rc = lib().og_decode_all(C.byref(self._g), m, _p(rowptr), _p(cols), threads)
        if rc:
            raise ValueError(f"decode failed (code {rc})")
        return rowptr, cols[: int(rowptr[-1])]

    def rw(self, mode, starts: np.ndarray, L: int, seed: int, threads: int = 0):
        starts = np.ascontiguousarray(starts, dtype=np.uint32)
        paths = np.zeros((len(starts), L + 1), dtype=np.uint32)
        tot = lib().og_rw(C.byref(self._g), MODES.get(mode, mode), _p(starts), len(starts), L,
                          seed, _p(paths), threads)
        return paths, int(tot)

    def node2vec(self, mode, starts: np.ndarray, L: int, seed: int, p: float, q: float,
                 max_tries: int = 0, threads: int = 0):
        starts = np.ascontiguousarray(starts, dtype=np.uint32)
        paths = np.zeros((len(starts), L + 1), dtype=np.uint32)
        tot = lib().og_node2vec(C.byref(self._g), MODES.get(mode, mode), _p(starts), len(starts),
                                L, seed, p, q, max_tries, _p(paths), threads)
        return paths, int(tot)

    def khop(self, mode, seeds: np.ndarray, fanouts, seed: int, threads: int = 0):
        seeds = np.ascontiguousarray(seeds, dtype=np.uint32)
        f = np.asarray(fanouts, dtype=np.uint32)
        outs, w = [], 1
        for fi in fanouts:
            w *= int(fi)
            outs.append(np.zeros((len(seeds), w), dtype=np.uint32))
        ptrs = (C.c_void_p * len(outs))(*[o.ctypes.data for o in outs])
        tot = lib().og_khop(C.byref(self._g), MODES.get(mode, mode), _p(seeds), len(seeds),
                            _p(f), len(fanouts), seed, C.cast(ptrs, C.c_void_p), threads)
        return outs, int(tot)

    def mrw(self, mode, roots: np.ndarray, T: int, seed: int, select: int = 0,
            threads: int = 0):
        roots = np.array(roots, dtype=np.uint32, order="C", copy=True)
        S, R = roots.shape
        src = np.zeros((S, T), dtype=np.uint32)
        dst = np.zeros((S, T), dtype=np.uint32)
        tot = lib().og_mrw(C.byref(self._g), MODES.get(mode, mode), _p(roots), S, R, T, seed,
                           select, _p(src), _p(dst), threads)
        return src, dst, roots, int(tot)


def rw_csr(rowptr: np.ndarray, cols: np.ndarray, starts: np.ndarray, L: int, seed: int,
           threads: int = 0):
    rowptr = np.ascontiguousarray(rowptr, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    starts = np.ascontiguousarray(starts, dtype=np.uint32)
    paths = np.zeros((len(starts), L + 1), dtype=np.uint32)
    tot = lib().og_rw_csr(_p(rowptr), _p(cols), len(rowptr) - 1, _p(starts), len(starts), L,
                          seed, _p(paths), threads)
    return paths, int(tot)


# ---------------------------------------------------------------------------
# Output compaction.  An entry is kept when it is not INVALID_VERTEX, the
# test the reference's frontier cut applies to its sorted transits
# (invalidVertexStartPos, GT/src/grass.cu:1085-1117); kept edges stay in
# output order.

def _kept(parent: np.ndarray, child: np.ndarray):
    m = child != INVALID
    return (np.ascontiguousarray(parent[m], dtype=np.uint32),
            np.ascontiguousarray(child[m], dtype=np.uint32))


def khop_edges(seeds: np.ndarray, hop_outs, fanouts):
    """(src, dst) of the valid k-hop edges in (hop, seed, slot) order."""
    src, dst = [], []
    prev = np.asarray(seeds, dtype=np.uint32).reshape(-1, 1)
    for h, f in enumerate(fanouts):
        cur = np.asarray(hop_outs[h], dtype=np.uint32).reshape(len(prev), -1)
        s, d = _kept(np.repeat(prev, f, axis=1), cur)
        src.append(s)
        dst.append(d)
        prev = cur
    return np.concatenate(src), np.concatenate(dst)


def rw_edges(paths: np.ndarray, walk_major: bool = True):
    """(src, dst) of the valid walk edges: (walk, step) order for [W][L+1]
    paths, (step, walk) order for [L+1][W]."""
    P = np.asarray(paths, dtype=np.uint32)
    if walk_major:
        return _kept(P[:, :-1], P[:, 1:])
    return _kept(P[:-1], P[1:])


def mrw_edges(step_src: np.ndarray, step_dst: np.ndarray):
    """(src, dst) of the multi-RW steps that took an edge, in (sample, step) order."""
    return _kept(np.asarray(step_src), np.asarray(step_dst))


# ---------------------------------------------------------------------------
# The reference's own CPU pieces, compiled from its sources into _ref/.

def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f)) for f in
               ("compressor_gt", "compressor_le", "graph_sort", "libref_bcg_gt.so",
                "libref_bcg_le.so"))


def ref_graph_sort(in_txt: str, out_txt: str, directed: bool = False) -> None:
    subprocess.check_call([os.path.join(REF_DIR, "graph_sort"), in_txt, out_txt,
                           "d" if directed else "u"], stdout=subprocess.DEVNULL)


def ref_compress(mode: str, in_txt: str, out_prefix: str) -> None:
    exe = os.path.join(REF_DIR, "compressor_gt" if mode.upper() == "GT" else "compressor_le")
    env = dict(os.environ)
    env.setdefault("OMP_NUM_THREADS", str(min(8, os.cpu_count() or 1)))
    subprocess.check_call([exe, in_txt, out_prefix], stdout=subprocess.DEVNULL, env=env)


_ref_libs: dict = {}


def ref_decoder(mode: str):
    """The reference's bcg.cuh decoder compiled for the host."""
    key = mode.upper()
    if key not in _ref_libs:
        L = C.CDLL(os.path.join(REF_DIR, f"libref_bcg_{key.lower()}.so"))
        P = C.c_void_p
        L.ref_decode_offset.argtypes = [P, C.c_uint64, C.c_uint32, P]
        L.ref_degree.argtypes = [P, P, C.c_int32]
        L.ref_degree.restype = C.c_int64
        L.ref_get_vertex.argtypes = [P, P, C.c_int32, C.c_int32]
        L.ref_get_vertex.restype = C.c_int64
        L.ref_decode_all.argtypes = [P, P, C.c_uint64, P, P]
        _ref_libs[key] = L
    return _ref_libs[key]


def ref_decode_all(mode: str, words: np.ndarray, offsets: np.ndarray):
    L = ref_decoder(mode)
    n = len(offsets) - 1
    rowptr = np.zeros(n + 1, dtype=np.uint64)
    L.ref_decode_all(_p(words), _p(offsets), n, _p(rowptr), None)
    cols = np.zeros(max(int(rowptr[-1]), 1), dtype=np.uint32)
    L.ref_decode_all(_p(words), _p(offsets), n, _p(rowptr), _p(cols))
    return rowptr, cols[: int(rowptr[-1])]


def ref_offset_lengths(mode: str, offset_file_bytes: bytes, n: int) -> np.ndarray:
    """Run the reference's decode_offset body over the .offset payload."""
    L = ref_decoder(mode)
    ubl = offset_file_bytes[0]
    payload = offset_file_bytes[1:]
    nw = (len(payload) + 3) // 4
    buf = np.zeros(nw * 4 + 16, dtype=np.uint8)
    buf[: len(payload)] = np.frombuffer(payload, dtype=np.uint8)
    words = buf.view(">u4").astype(np.uint32)
    lens = np.zeros(n, dtype=np.uint64)
    L.ref_decode_offset(_p(words), n, ubl, _p(lens))
    return lens
