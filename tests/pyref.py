"""Pure-Python restatement of the sampling semantics, for small cases only.

Used to cross-check the C oracle's step logic on tiny inputs: it reads
neighbor lists from a plain CSR and draws from oracle.philox, so it shares
nothing with the C code but the Philox function (pinned separately by the
known-answer fixture).
"""
import numpy as np

INVALID = 0xFFFFFFFF
TAG_RW = 0x52570001
TAG_KHOP = 0x4B480000
TAG_MRW = 0x4D520001


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
