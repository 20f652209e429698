// kernels_decode.cu -- decode-only sweep: every neighbor list into CSR.
//
// Replaces the reference's two decoders for whole lists: the block-cooperative
// GlobalDecoder (GT/src/bcg.cuh:171-345, used by the grid/thread-block
// kernels at GT/src/grass.cu:529-553, 762-786) and repeated
// BCGVertex::get_vertex calls (LE/src/bcg.cuh:195-261).
//
// Work is split over the neighbor index space, not over vertices: task t
// covers neighbors [t*C, (t+1)*C) of the CSR being written, whatever
// vertices they belong to, so a hub vertex with 10^5 neighbors is spread over
// many warps instead of serialising one.  Per task a warp
//  1. finds the vertex holding the first neighbor with a 32-ary search of
//     rowptr (one coalesced probe per level);
//  2. for each round of 32 consecutive neighbors, loads the row ends and
//     records of a window of 32 vertices (coalesced), maps every lane to its
//     vertex by a shuffle binary search and takes the header by shuffle;
//  3. decodes: LE -- each neighbor is two rocks and one signed sea
//     (independent); GT -- each lane reads its own field (block head or gap)
//     and a segmented warp scan turns gaps into ids, with the running value
//     carried from round to round (and, at a task start inside a block,
//     decoded once by lane 0);
//  4. writes its 32 ids with one coalesced store.
#include "graph.h"

namespace grass {

namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr uint32_t kTaskNeighbors = 2048;  // multiple of 32

__device__ __forceinline__ VHdr shfl_hdr(const VHdr &h, int src) {
  VHdr o;
  o.P = __shfl_sync(FULL, h.P, src);
  o.v = __shfl_sync(FULL, h.v, src);
  o.d = __shfl_sync(FULL, h.d, src);
  o.bn = __shfl_sync(FULL, h.bn, src);
  o.bl = __shfl_sync(FULL, h.bl, src);
  o.om = __shfl_sync(FULL, h.om, src);
  o.fp = __shfl_sync(FULL, h.fp, src);
  o.a = __shfl_sync(FULL, h.a, src);
  o.b = __shfl_sync(FULL, h.b, src);
  return o;
}

// 64 stream bits starting at bit `off`: three word loads, two funnel shifts
// (the sweep reads the stream in order, so these hit L1).
__device__ __forceinline__ uint64_t read_bits64(const uint32_t *w, uint64_t off) {
  const uint32_t *q = w + (off >> 5);
  const uint32_t s = (uint32_t)off & 31u;
  const uint32_t x0 = ldw(q), x1 = ldw(q + 1), x2 = ldw(q + 2);
  return ((uint64_t)__funnelshift_l(x1, x0, s) << 32) | __funnelshift_l(x2, x1, s);
}

// le_neighbor (device_common.cuh) with word reads instead of sector loads:
// the same arithmetic, LE/src/bcg.cuh:195-261.
__device__ __forceinline__ uint32_t le_neighbor_words(const uint32_t *words, const VHdr &h,
                                                      uint32_t i) {
  if (h.d == 1) return h.fp;
  uint32_t tl = h.bl + 1;
  const uint32_t split = h.om * tl;
  const bool flag = i >= split;
  const uint32_t j = flag ? i - split : i;
  if (flag) tl -= 1;
  uint32_t c = j / tl;
  const uint32_t id = j - c * tl;
  if (flag) c += h.om;
  const uint64_t rwin = read_bits64(words, h.P + (uint64_t)c * (uint64_t)h.a);
  const uint32_t r1m = (uint32_t)(rwin >> (64 - h.a));
  const uint32_t r1 = (c < h.fp) ? h.v - r1m : h.v + r1m;
  if (id == 0) return r1;
  const uint32_t r2m = (uint32_t)((rwin << h.a) >> (64 - h.a));
  const uint32_t r2 = (c + 1 < h.fp) ? h.v - r2m : h.v + r2m;
  const uint64_t spos =
      h.P + (uint64_t)(h.bn + 1) * (uint64_t)h.a +
      ((uint64_t)(h.bl - 1) * c + min(h.om, c) + id - 1) * (uint64_t)(h.b + 1);
  const uint32_t raw = (uint32_t)(read_bits64(words, spos) >> (63 - h.b));
  const uint32_t mag = raw >> 1;
  return ((r2 - r1) / tl) * id + r1 + ((raw & 1u) ? 0u - mag : mag);
}

// Largest v in [0, n) with rowptr[v] <= x, for x < rowptr[n].
__device__ __forceinline__ uint32_t warp_row_of(const uint64_t *rowptr, uint32_t n, uint64_t x) {
  const int lane = threadIdx.x & 31;
  uint64_t lo = 0, hi = n;  // rowptr[lo] <= x < rowptr[hi]
  while (hi - lo > 1) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t p = lo + (uint64_t)(lane + 1) * step;
    const bool le = p < hi && rowptr[p] <= x;
    const uint32_t c = __popc(__ballot_sync(FULL, le));
    const uint64_t nlo = lo + (uint64_t)c * step;
    hi = min(hi, lo + (uint64_t)(c + 1) * step);
    lo = nlo;
  }
  return (uint32_t)lo;
}

// Largest v in [lo, n) with rowptr[v] <= x, one thread (rare fallback).
__device__ __forceinline__ uint32_t row_of_serial(const uint64_t *rowptr, uint32_t lo, uint32_t n,
                                                  uint64_t x) {
  uint32_t hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (rowptr[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <int MODE>
__global__ void __launch_bounds__(256) decode_all_kernel(DevGraph g, const uint64_t *rowptr,
                                                           uint32_t *cols, uint64_t E,
                                                           unsigned int *err) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t tasks = (E + kTaskNeighbors - 1) / kTaskNeighbors;
  bool bad = false;
  for (uint64_t t = warp; t < tasks; t += nwarps) {
    const uint64_t g0 = t * kTaskNeighbors;
    const uint64_t g1 = min(E, g0 + kTaskNeighbors);
    uint32_t vr = warp_row_of(rowptr, g.n, g0);
    uint32_t carry = 0;
    if (MODE == 0) {
      // a task that starts inside a block needs the value of neighbor g0-1
      const uint32_t i0 = (uint32_t)(g0 - rowptr[vr]);
      if (i0 > 0) {
        uint32_t c = 0;
        if (lane == 0) {
          const VHdr h0 = header<0>(g, vr);
          if (gt_locate(h0, i0).gaps > 0) c = gt_neighbor(g, h0, i0 - 1);
        }
        carry = __shfl_sync(FULL, c, 0);
      }
    }
    // Header of the vertex that holds the whole current round (fast path),
    // kept across rounds of the same vertex.
    uint32_t cv = 0xFFFFFFFFu;
    uint64_t cstart = 0, cend = 0;
    VHdr ch{};
    bool ch_ok = false;
    for (uint64_t r = g0; r < g1; r += 32) {  // warp-uniform
      const uint64_t gl = r + lane;
      const bool act = gl < g1;
      const uint64_t rlast = min(g1, r + 32) - 1;
      if (vr != cv) {
        cv = vr;
        cstart = rowptr[vr];
        cend = rowptr[vr + 1];
        ch_ok = false;
      }
      VHdr hk;
      uint64_t startv;
      bool far = false;
      int k = 0;
      const bool single = cstart <= r && rlast < cend;  // warp-uniform
      if (single) {
        // Fast path: the round lies inside vertex vr (most rounds of a
        // skewed graph): no window, no owner search.
        if (!ch_ok) {
          ch = header<MODE>(g, vr);
          ch_ok = true;
        }
        hk = ch;
        startv = cstart;
      } else {
        // window of vertices [vr, vr + 32): row ends and headers, one per lane
        const uint32_t wv = vr + lane;
        const uint64_t base = rowptr[vr];
        const uint64_t e = wv < g.n ? rowptr[wv + 1] : ~0ull;
        VHdr hw;
        if (wv < g.n) {
          hw = header<MODE>(g, wv);
        } else {
          hw.d = 0; hw.P = 0; hw.v = 0; hw.bn = hw.bl = hw.om = hw.fp = 0; hw.a = hw.b = 0;
        }
        // owner lane k: number of window rows that end at or before gl
        // (binary lifting over 31 probes gives the exact count when it is
        // below 32)
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const uint64_t ek = __shfl_sync(FULL, e, k + step - 1);
          if (ek <= gl) k += step;
        }
        // a count of 32 means gl lies beyond the window (a run of >= 32 empty
        // rows); those lanes resolve their vertex and header on their own.
        const uint64_t e31 = __shfl_sync(FULL, e, 31);
        far = act && e31 <= gl;
        const int src = far ? 0 : k;
        const uint64_t prev_e = __shfl_sync(FULL, e, src > 0 ? src - 1 : 0);
        hk = shfl_hdr(hw, src);
        startv = src == 0 ? base : prev_e;
        if (far) {
          const uint32_t v = row_of_serial(rowptr, vr + 32, g.n, gl);
          hk = header<MODE>(g, v);
          startv = rowptr[v];
        }
      }
      const uint32_t i = (uint32_t)(gl - startv);
      uint32_t val = 0;
      if (MODE == 1) {
        if (act) val = le_neighbor_words(g.words, hk, i);
      } else {
        bool head = true;
        uint32_t x = 0;
        if (act) {
          const GtRun run = gt_locate(hk, i);
          if (far) {
            x = gt_neighbor(g, hk, i);  // complete value; starts its own segment
          } else if (run.gaps == 0) {
            const uint32_t hv = read_field(g.words, run.pos, hk.a) + 1u;
            x = run.up ? hk.v + hv : hk.v - hv;
          } else {
            head = false;
            x = read_field(g.words, run.pos + hk.a + (uint64_t)(run.gaps - 1) * hk.b, hk.b) + 1u;
          }
        }
        if (lane == 0 && !head) {
          x += carry;
          head = true;
        }
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {  // segmented inclusive scan
          const uint32_t y = __shfl_up_sync(FULL, x, o);
          const int f = __shfl_up_sync(FULL, (int)head, o);
          if (lane >= o && !head) {
            x += y;
            head = f;
          }
        }
        carry = __shfl_sync(FULL, x, 31);
        val = x;
      }
      if (act) {
        if (val >= g.n) bad = true;
        cols[gl] = val;
      }
      // next window starts at the vertex of the round's last neighbor
      if (!single) {
        const uint32_t vlast = __shfl_sync(FULL, far ? 0xFFFFFFFFu : vr + (uint32_t)k, 31);
        if (vlast != 0xFFFFFFFFu) {
          vr = vlast;
        } else {
          const uint64_t gl31 = r + 31;
          vr = gl31 < g1 ? warp_row_of(rowptr, g.n, gl31) : vr;
        }
      }
    }
  }
  if (bad && err) atomicOr(err, 1u);
}

}  // namespace

void launch_decode_all(const DevGraph &g, const uint64_t *rowptr, uint32_t *cols, uint64_t E,
                       unsigned int *err, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (!E) return;
  const uint64_t tasks = (E + kTaskNeighbors - 1) / kTaskNeighbors;
  const uint64_t blocks_needed = (tasks + 7) / 8;
  const unsigned grid = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>(blocks_needed, (uint64_t)sm_count(dev) * 8));
  if (g.mode == GRASS_MODE_GT)
    decode_all_kernel<0><<<grid, 256, 0, s>>>(g, rowptr, cols, E, err);
  else
    decode_all_kernel<1><<<grid, 256, 0, s>>>(g, rowptr, cols, E, err);
  count_launch();
}

}  // namespace grass
