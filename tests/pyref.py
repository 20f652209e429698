"""Pure-Python restatement of the sampling semantics, for small cases only.

Used to cross-check the C oracle's step logic on tiny inputs: it reads
neighbor lists from a plain CSR and draws from oracle.philox, so it shares
nothing with the C code but the Philox function (pinned separately by the
known-answer fixture).
"""
import heapq
import struct

import numpy as np

INVALID = 0xFFFFFFFF
TAG_RW = 0x52570001
TAG_KHOP = 0x4B480000
TAG_MRW = 0x4D520001
TAG_MRW_CT = 0x4D520003


def _mulhi(r, d):
    return (int(r) * int(d)) >> 32


def rw(philox, rowptr, cols, starts, L, seed):
    n = len(rowptr) - 1
    out = np.zeros((len(starts), L + 1), np.uint32)
    for w, s0 in enumerate(starts):
        v = int(s0) if s0 < n else INVALID
        out[w, 0] = s0
        for s in range(L):
            r = philox(seed, [s >> 2, w & 0xFFFFFFFF, w >> 32, TAG_RW])[s & 3]
            if v != INVALID:
                d = int(rowptr[v + 1] - rowptr[v])
                v = INVALID if d == 0 else int(cols[int(rowptr[v]) + _mulhi(r, d)])
            out[w, s + 1] = v
    return out


def khop(philox, rowptr, cols, seeds, fanouts, seed):
    n = len(rowptr) - 1
    outs = []
    for h, f in enumerate(fanouts):
        prevw = 1 if h == 0 else outs[-1].shape[1]
        o = np.zeros((len(seeds), prevw * f), np.uint32)
        for s, root in enumerate(seeds):
            for p in range(prevw):
                t = int(root) if h == 0 else int(outs[-1][s, p])
                for k in range(f):
                    j = p * f + k
                    d = int(rowptr[t + 1] - rowptr[t]) if t < n else 0
                    if d == 0:
                        o[s, j] = INVALID
                        continue
                    r = philox(seed, [j >> 2, s, 0, TAG_KHOP | h])[j & 3]
                    o[s, j] = cols[int(rowptr[t]) + _mulhi(r, d)]
        outs.append(o)
    return outs


def mrw(philox, rowptr, cols, roots, T, seed, select):
    if select == 2:
        return mrw_ct(philox, rowptr, cols, roots, T, seed)
    n = len(rowptr) - 1
    roots = np.array(roots, dtype=np.int64)
    S, R = roots.shape
    src = np.zeros((S, T), np.uint32)
    dst = np.zeros((S, T), np.uint32)

    def deg(v):
        return int(rowptr[v + 1] - rowptr[v]) if v < n else 0

    for s in range(S):
        for t in range(T):
            o = philox(seed, [t, s, 0, TAG_MRW])
            if select == 0:
                x = _mulhi(o[0], R)
            else:
                ws = [deg(int(v)) for v in roots[s]]
                W = sum(ws)
                if W == 0:
                    src[s, t] = dst[s, t] = INVALID
                    continue
                r64 = (int(o[2]) << 32) | int(o[0])
                u = (r64 * W) >> 64
                acc = 0
                for x, wv in enumerate(ws):
                    acc += wv
                    if u < acc:
                        break
            v = int(roots[s, x])
            src[s, t] = v
            d = deg(v)
            if d == 0:
                dst[s, t] = INVALID
                continue
            nv = int(cols[int(rowptr[v]) + _mulhi(o[1], d)])
            dst[s, t] = nv
            roots[s, x] = nv
    return src, dst, roots.astype(np.uint32)


# ---------------------------------------------------------------------------
# Continuous-time multi-RW (select 2), restated with Python floats (IEEE
# doubles, every operation rounded on its own -- no fused multiply-add).

_ATANH = [float.fromhex(h) for h in (
    "0x1.8618618618618p-5", "0x1.af286bca1af28p-5", "0x1.e1e1e1e1e1e1ep-5",
    "0x1.1111111111111p-4", "0x1.3b13b13b13b14p-4", "0x1.745d1745d1746p-4",
    "0x1.c71c71c71c71cp-4", "0x1.2492492492492p-3", "0x1.999999999999ap-3",
    "0x1.5555555555555p-2")]  # 1/21, 1/19, ..., 1/3
_LN2 = float.fromhex("0x1.62e42fefa39efp-1")
_SQRT2 = float.fromhex("0x1.6a09e667f3bcdp+0")


def _bits(x):
    return struct.unpack("<Q", struct.pack("<d", x))[0]


def _float(b):
    return struct.unpack("<d", struct.pack("<Q", b))[0]


def det_log(u):
    """ln u = e ln2 + 2 atanh((m-1)/(m+1)), m in [sqrt(1/2), sqrt(2))."""
    b = _bits(u)
    e = ((b >> 52) & 0x7FF) - 1023
    m = _float((b & 0xFFFFFFFFFFFFF) | 0x3FF0000000000000)
    if m > _SQRT2:
        m = m * 0.5
        e += 1
    s = (m + -1.0) / (m + 1.0)
    z = s * s
    p = _ATANH[0]
    for c in _ATANH[1:]:
        p = c + z * p
    t = s + s * (z * p)
    return float(e) * _LN2 + 2.0 * t


def _exp_variate(w0, w1):
    u52 = ((int(w0) << 20) | (int(w1) >> 12)) & ((1 << 52) - 1)
    return -det_log((float(u52) + 0.5) * 2.0 ** -52)


def _next_time(t, E, d):
    nt = t + E / float(d)
    return nt if nt > t else _float(_bits(t) + 1)


def mrw_ct(philox, rowptr, cols, roots, T, seed):
    """Walker w's k-th move: Philox(seed; k, sample, w, TAG_MRW_CT), words 0-1
    the Exp(1) holding time (divided by the degree), word 2 the neighbor; the
    output is the first T moves of all walkers in (time, walker) order."""
    n = len(rowptr) - 1
    roots = np.array(roots, dtype=np.int64)
    S, R = roots.shape
    src = np.zeros((S, T), np.uint32)
    dst = np.zeros((S, T), np.uint32)

    def deg(v):
        return int(rowptr[v + 1] - rowptr[v]) if v < n else 0

    for s in range(S):
        v = [int(x) for x in roots[s]]
        k = [0] * R
        z = [0] * R
        heap = []

        def arm(w, t0):
            d = deg(v[w])
            if d == 0:
                return
            o = philox(seed, [k[w], s, w, TAG_MRW_CT])
            z[w] = int(o[2])
            heapq.heappush(heap, (_next_time(t0, _exp_variate(o[0], o[1]), d), w))

        for w in range(R):
            arm(w, 0.0)
        for r in range(T):
            if not heap:
                src[s, r] = dst[s, r] = INVALID
                continue
            t, w = heapq.heappop(heap)
            d = deg(v[w])
            nv = int(cols[int(rowptr[v[w]]) + _mulhi(z[w], d)])
            src[s, r], dst[s, r] = v[w], nv
            v[w] = nv
            k[w] += 1
            arm(w, t)
        roots[s] = v
    return src, dst, roots.astype(np.uint32)


def khop_edges(seeds, outs, fanouts):
    """Valid k-hop edges by explicit loops, (hop, seed, slot) order."""
    src, dst = [], []
    for h, f in enumerate(fanouts):
        for s in range(len(seeds)):
            for j in range(outs[h].shape[1]):
                c = int(outs[h][s, j])
                if c == INVALID:
                    continue
                src.append(int(seeds[s]) if h == 0 else int(outs[h - 1][s, j // f]))
                dst.append(c)
    return np.array(src, np.uint32), np.array(dst, np.uint32)


def rw_edges(paths):
    """Valid edges of walk-major [W][L+1] paths, (walk, step) order."""
    src, dst = [], []
    for row in paths:
        for t in range(len(row) - 1):
            if int(row[t + 1]) != INVALID:
                src.append(int(row[t]))
                dst.append(int(row[t + 1]))
    return np.array(src, np.uint32), np.array(dst, np.uint32)
