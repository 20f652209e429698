// kernels_sample.cu -- random walk, k-hop and multi-RW kernels over the
// compressed graph, plus the uncompressed-CSR baselines with the same RNG.
//
// The reference runs every app step as a separate transit-parallel pass:
// sample kernel, then a global radix sort inverting sample->transit, run-
// length encoding, a scan and a kernel-type partition, with blocking syncs in
// between (GT/src/grass.cu:1573-1998).  For fanout-1 walks nothing is shared
// between walkers on the same transit, so here one launch runs all steps:
// each thread owns DEPTH walkers and interleaves them, which keeps DEPTH
// independent decode chains in flight per thread.
#include "graph.h"
#include "mrw_cta.cuh"
#include "sample_warp.cuh"

#include <mutex>

// Resident 512-thread blocks per SM each walk kernel is compiled for (its
// register budget), as measured on the 1M x 80 walk: the LE walk keeps all
// the registers it wants (79 at one walker per thread; launched as 256-thread
// blocks, three per SM, which ran 17% faster than 512-thread blocks), the GT
// walk is 23% faster at 64 registers or fewer, the CSR walk 2% faster.
#ifndef GRASS_RW_LE_MIN_BLOCKS
#define GRASS_RW_LE_MIN_BLOCKS 1
#endif
#ifndef GRASS_RW_GT_MIN_BLOCKS
#define GRASS_RW_GT_MIN_BLOCKS 2
#endif
#ifndef GRASS_RW_CSR_MIN_BLOCKS
#define GRASS_RW_CSR_MIN_BLOCKS 2
#endif

namespace grass {

namespace {

__device__ __forceinline__ void store_path(uint32_t *paths, int layout, uint64_t W, uint32_t L,
                                           uint64_t w, uint32_t s, uint32_t v) {
  if (layout == GRASS_LAYOUT_WALK_MAJOR) store_out_u32(paths + w * (uint64_t)(L + 1) + s, v);
  else store_out_u32(paths + (uint64_t)s * W + w, v);
}

// w0: walker id of starts[0] -- draws use walker id w0 + w, so a batch split
// into chunks produces the same walks as one launch.
template <int MODE, int DEPTH>
__global__ void __launch_bounds__(512, MODE == 0 ? GRASS_RW_GT_MIN_BLOCKS : GRASS_RW_LE_MIN_BLOCKS) rw_kernel(DevGraph g, const uint32_t *__restrict__ starts,
                                                 uint64_t W, uint32_t L, uint64_t seed,
                                                 uint64_t w0, int layout,
                                                 uint32_t *__restrict__ paths,
                                                 unsigned long long *edges, unsigned int *err) {
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  uint64_t cnt = 0;
  bool bad = false;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; base < W;
       base += nthreads * DEPTH) {
    uint32_t v[DEPTH];
    u32x4 r[DEPTH];
#pragma unroll
    for (int k = 0; k < DEPTH; k++) {
      const uint64_t w = base + k * nthreads;
      v[k] = INVALID_VERTEX;
      r[k] = u32x4{0, 0, 0, 0};
      if (w < W) {
        const uint32_t s0 = starts[w];
        store_path(paths, layout, W, L, w, 0, s0);
        v[k] = s0 < g.n ? s0 : INVALID_VERTEX;
      }
    }
    for (uint32_t s = 0; s < L; s++) {
#pragma unroll
      for (int k = 0; k < DEPTH; k++) {
        const uint64_t w = base + k * nthreads;
        if ((s & 3) == 0) {
          const uint64_t id = w0 + w;
          r[k] = philox4x32_10(seed, s >> 2, (uint32_t)id, (uint32_t)(id >> 32), TAG_RW);
        }
        if (v[k] != INVALID_VERTEX) {
          const VHdr h = header<MODE>(g, v[k]);
          if (h.d == 0) {
            v[k] = INVALID_VERTEX;
          } else {
            const uint32_t nv = neighbor<MODE>(g, h, mulhi_u32(pick(r[k], s & 3), h.d));
            if (nv >= g.n) {
              bad = true;
              v[k] = INVALID_VERTEX;
            } else {
              v[k] = nv;
              cnt++;
            }
          }
        }
        if (w < W) store_path(paths, layout, W, L, w, s + 1, v[k]);
      }
    }
  }
  warp_add_u64(edges, cnt);
  if (bad && err) atomicOr(err, 1u);
}

// ---------------------------------------------------------------------------
// Second-order (node2vec) walk.  One walker per thread.  Try k of step s
// draws Philox(seed; s, w, w >> 32, TAG_N2V | k): word 0 picks the candidate
// from N(v), word 1 is compared with the candidate's acceptance threshold
// (return to u, a neighbor of u, or farther).  The membership test searches
// u's sorted neighbor list (has_neighbor).
struct N2vArgs {
  uint32_t L, max_tries;
  int layout;
  uint64_t seed, w0;
  uint64_t t_ret, t_in, t_out;  // acceptance thresholds in [0, 2^32]
};

// The first neighbor of slot c (GT: its head; LE: its left rock): one field
// of at most 32 bits, read as one or two 32-bit words (the second only when
// the field crosses into it).
template <int MODE>
__device__ __forceinline__ uint32_t slot_first(const DevGraph &g, const VHdr &h, uint32_t c) {
  const uint64_t pos = slot_pos(h, c);
  const uint32_t *q = g.words + (pos >> 5);
  const uint32_t s = (uint32_t)pos & 31u, w = (uint32_t)h.a;
  const uint32_t hi = ldw(q), lo = s + w > 32u ? ldw(q + 1) : 0u;
  const uint32_t m = w ? __funnelshift_l(lo, hi, s) >> (32u - w) : 0u;
  if constexpr (MODE == 0) return c >= h.fp ? h.v + m + 1u : h.v - m - 1u;
  else return c < h.fp ? h.v - m : h.v + m;
}

// The last index in [lo, hi] whose key is <= x, given key(lo) <= x, for
// nondecreasing keys: a binary search, one probe per round.  (An 8-way
// search, seven independent probes per round, was slower: with a million
// walkers in flight latency is hidden anyway, and it loads more.)
template <class Key>
__device__ __forceinline__ uint32_t last_le(uint32_t lo, uint32_t hi, uint32_t x, Key key) {
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo + 1) / 2;
    if (key(mid) <= x) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Whether x is a neighbor of the vertex of header h.  Compressed: a search
// over the slots' first neighbors for the one slot that can hold x, then a
// search of that slot inside its sector, in registers (GT: a scan of the
// gaps; LE: a binary search of the closed-form values).  CSR: a search of
// the row.
template <int MODE>
__device__ __forceinline__ bool has_neighbor(const DevGraph &g, const VHdr &h, uint32_t x) {
  if (h.d == 0) return false;
  if constexpr (MODE == 2) {
    if (neighbor<MODE>(g, h, 0) > x) return false;
    const uint32_t i = last_le(0u, h.d - 1, x, [&](uint32_t k) { return neighbor<MODE>(g, h, k); });
    return neighbor<MODE>(g, h, i) == x;
  } else {
    if (MODE == 1 && h.d == 1) return h.fp == x;
    if (slot_first<MODE>(g, h, 0) > x) return false;
    const uint32_t c = last_le(0u, h.bn - 1, x, [&](uint32_t k) { return slot_first<MODE>(g, h, k); });
    // slot c holds indices c bl .. c bl + last
    const uint32_t last = c + 1 == h.bn ? h.d - 1 - c * h.bl : h.bl - 1;
    const uint64_t pos = slot_pos(h, c);
    const Sec A = load_sector(g.words, pos >> 8);
    const uint32_t off = (uint32_t)pos & 255u;
    if constexpr (MODE == 0) {
      const uint32_t hv = (uint32_t)sec1_field(A, off, h.a) + 1u;
      uint32_t y = c >= h.fp ? h.v + hv : h.v - hv;
      uint32_t p = off + (uint32_t)h.a;
      for (uint32_t t = 0; y < x && t < last; t++, p += (uint32_t)h.b)
        y += (h.b ? (uint32_t)sec1_field(A, p, h.b) : 0u) + 1u;
      return y == x;
    } else {
      const uint32_t L = min(h.bl, h.d - 1 - c * h.bl);
      const uint32_t id = last_le(0u, last, x, [&](uint32_t k) { return le_slot_value(A, off, h, c, k, L); });
      return le_slot_value(A, off, h, c, id, L) == x;
    }
  }
}

// Resident 256-thread blocks per SM the node2vec kernels are compiled for.
// The walk is latency-bound (dependent sector reads, divergent tries), so
// resident warps matter more than registers: on the 1M x 80 walk the
// compressed kernels at 4 blocks (64 registers) ran 1.6x faster than at 118
// registers (2 blocks; unbounded builds also came out at 134, 1 block), 1.2x
// faster than at 3 blocks, and 1.1-1.2x faster than at 5 or 6, where spills
// grow.  The CSR kernel needs no cap (69 registers, 3 blocks).
#ifndef GRASS_N2V_MIN_BLOCKS
#define GRASS_N2V_MIN_BLOCKS 4
#endif
#ifndef GRASS_N2V_CSR_MIN_BLOCKS
#define GRASS_N2V_CSR_MIN_BLOCKS 1
#endif

template <int MODE>
__global__ void __launch_bounds__(256, MODE == 2 ? GRASS_N2V_CSR_MIN_BLOCKS : GRASS_N2V_MIN_BLOCKS) n2v_kernel(DevGraph g, const uint32_t *__restrict__ starts,
                                                  uint64_t W, N2vArgs a,
                                                  uint32_t *__restrict__ paths,
                                                  unsigned long long *edges, unsigned int *err) {
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  const uint64_t t_lo = min(a.t_in, a.t_out), t_hi = max(a.t_in, a.t_out);
  uint64_t cnt = 0;
  bool bad = false;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < W; w += nthreads) {
    const uint64_t id = a.w0 + w;
    const uint32_t s0 = starts[w];
    store_path(paths, a.layout, W, a.L, w, 0, s0);
    uint32_t v = s0 < g.n ? s0 : INVALID_VERTEX, u = INVALID_VERTEX;
    VHdr hu;  // the previous vertex's header (kept from the step that left it)
    hu.d = 0;
    for (uint32_t s = 0; s < a.L; s++) {
      if (v != INVALID_VERTEX) {
        const VHdr h = header<MODE>(g, v);
        if (h.d == 0) {
          v = INVALID_VERTEX;
        } else {
          uint32_t x = INVALID_VERTEX;
          for (uint32_t k = 0; k < a.max_tries; k++) {
            const u32x4 r =
                philox4x32_10(a.seed, s, (uint32_t)id, (uint32_t)(id >> 32), TAG_N2V | k);
            x = neighbor<MODE>(g, h, mulhi_u32(r.x, h.d));
            if (s == 0 || k + 1 == a.max_tries) break;  // first step: uniform
            const uint64_t y = r.y;
            if (x == u) {
              if (y < a.t_ret) break;
              continue;
            }
            // below both thresholds the candidate is taken, at or above both it
            // is not, whether or not it is a neighbor of u: only in between does
            // the membership search run (never when t_in == t_out, i.e. q = 1)
            if (y < t_lo) break;
            if (y >= t_hi) continue;
            if (y < (has_neighbor<MODE>(g, hu, x) ? a.t_in : a.t_out)) break;
          }
          if (x >= g.n) {
            bad = true;
            v = INVALID_VERTEX;
          } else {
            u = v;
            hu = h;
            v = x;
            cnt++;
          }
        }
      }
      store_path(paths, a.layout, W, a.L, w, s + 1, v);
    }
  }
  warp_add_u64(edges, cnt);
  if (bad && err) atomicOr(err, 1u);
}

// Stream bits a draw of neighbor i reads (the payload fields; the header is
// in the vertex record), and the 32-byte sectors those reads span.
template <int MODE>
__device__ __forceinline__ void draw_footprint(const DevGraph &g, const VHdr &h, uint32_t i,
                                               uint64_t &bits, uint64_t &sectors) {
  (void)g;
  sectors = 1;  // a chunk slot never crosses a sector
  if (MODE == 0) {  // the slot's head and the gaps up to neighbor i
    bits = (uint64_t)h.a + (uint64_t)(i % h.bl) * h.b;
  } else if (h.d > 1) {  // the left rock; for an inner neighbor the right rock and a sea
    uint32_t c, id, L;
    le_locate(h, i, c, id, L);
    bits = id == 0 ? (uint64_t)h.a : id == L ? 2ull * h.a : 2ull * h.a + h.b + 1;
  } else {  // LE degree 1: the neighbor is in the record
    bits = 0;
    sectors = 0;
  }
}

// Replays a walk (same stream as rw_kernel) and sums, per draw, the
// algorithmic bytes 16 (vertex record) + ceil(payload bits read / 8) + 4
// (path entry) and the 32-byte sectors the reads span (+1 for the record).
// out[0] = bytes, out[1] = sectors, out[2] = draws.  Start entries add 4
// bytes each.
// Independent random 4-byte reads: each thread draws xorshift64 indices into
// buf[0, mask] and keeps 8 loads in flight; the sum goes to *sink so the loads
// are not dropped.  Used to measure the device's random-read ceiling.
__global__ void __launch_bounds__(256) random_read_kernel(const uint32_t *__restrict__ buf,
                                                          uint64_t mask, uint64_t per_thread,
                                                          uint64_t seed,
                                                          unsigned long long *sink) {
  const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  uint64_t x = (seed + 1) * 0x9E3779B97F4A7C15ull ^ (tid + 1) * 0xBF58476D1CE4E5B9ull;
  uint32_t acc = 0;
  for (uint64_t r = 0; r < per_thread; r += 8) {
    uint32_t v[8];
#pragma unroll
    for (int k = 0; k < 8; k++) {
      x ^= x << 13;
      x ^= x >> 7;
      x ^= x << 17;
      v[k] = __ldg(buf + (x & mask));
    }
#pragma unroll
    for (int k = 0; k < 8; k++) acc += v[k];
  }
  acc = __reduce_add_sync(0xFFFFFFFFu, acc);
  if ((threadIdx.x & 31) == 0) atomicAdd(sink, (unsigned long long)acc);
}

template <int MODE>
__global__ void __launch_bounds__(256) rw_account_kernel(DevGraph g,
                                                         const uint32_t *__restrict__ starts,
                                                         uint64_t W, uint32_t L, uint64_t seed,
                                                         unsigned long long *out) {
  uint64_t bytes = 0, sect = 0, draws = 0;
  for (uint64_t w = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; w < W;
       w += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t v = starts[w];
    bytes += 4;
    if (v >= g.n) v = INVALID_VERTEX;
    u32x4 r{0, 0, 0, 0};
    for (uint32_t s = 0; s < L; s++) {
      if ((s & 3) == 0) r = philox4x32_10(seed, s >> 2, (uint32_t)w, (uint32_t)(w >> 32), TAG_RW);
      bytes += 4;
      if (v == INVALID_VERTEX) continue;
      const VHdr h = header<MODE>(g, v);
      if (h.d == 0) {
        v = INVALID_VERTEX;
        continue;
      }
      const uint32_t i = mulhi_u32(pick(r, s & 3), h.d);
      uint64_t b, sc;
      draw_footprint<MODE>(g, h, i, b, sc);
      bytes += 16 + (b + 7) / 8;
      sect += 1 + sc;
      draws++;
      const uint32_t nv = neighbor<MODE>(g, h, i);
      v = nv < g.n ? nv : INVALID_VERTEX;
    }
  }
  warp_add_u64(&out[0], bytes);
  warp_add_u64(&out[1], sect);
  warp_add_u64(&out[2], draws);
}

template <int DEPTH>
__global__ void __launch_bounds__(512, GRASS_RW_CSR_MIN_BLOCKS) rw_csr_kernel(DevCsr c, const uint32_t *__restrict__ starts,
                                                     uint64_t W, uint32_t L, uint64_t seed,
                                                     uint64_t w0, int layout,
                                                     uint32_t *__restrict__ paths,
                                                     unsigned long long *edges) {
  const uint64_t nthreads = (uint64_t)gridDim.x * blockDim.x;
  uint64_t cnt = 0;
  for (uint64_t base = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; base < W;
       base += nthreads * DEPTH) {
    uint32_t v[DEPTH];
    u32x4 r[DEPTH];
#pragma unroll
    for (int k = 0; k < DEPTH; k++) {
      const uint64_t w = base + k * nthreads;
      v[k] = INVALID_VERTEX;
      r[k] = u32x4{0, 0, 0, 0};
      if (w < W) {
        const uint32_t s0 = starts[w];
        store_path(paths, layout, W, L, w, 0, s0);
        v[k] = s0 < c.n ? s0 : INVALID_VERTEX;
      }
    }
    for (uint32_t s = 0; s < L; s++) {
#pragma unroll
      for (int k = 0; k < DEPTH; k++) {
        const uint64_t w = base + k * nthreads;
        if ((s & 3) == 0) {
          const uint64_t id = w0 + w;
          r[k] = philox4x32_10(seed, s >> 2, (uint32_t)id, (uint32_t)(id >> 32), TAG_RW);
        }
        if (v[k] != INVALID_VERTEX) {
          uint64_t b, e;
          csr_row(c.rowptr, v[k], b, e);
          const uint64_t d = e - b;
          if (d == 0) {
            v[k] = INVALID_VERTEX;
          } else {
            v[k] = load_cold_u32(c.cols + b + mulhi_u32(pick(r[k], s & 3), (uint32_t)d));
            cnt++;
          }
        }
        if (w < W) store_path(paths, layout, W, L, w, s + 1, v[k]);
      }
    }
  }
  warp_add_u64(edges, cnt);
}

// ---------------------------------------------------------------------------
// Draws a lane of the standalone k-hop has in flight at once (the batched
// kernel keeps one: its register budget is shared with the walks), and the
// k-hop kernels' resident blocks per SM (256 threads each).  Measured on
// R-MAT s22 ef32, 65,536 seeds x (25, 10): (2, 4) beat (4, 2), (4, 3), (2, 3)
// and (1, 4) for GT, LE and the CSR.
#ifndef GRASS_KHOP_INFLIGHT
#define GRASS_KHOP_INFLIGHT 2
#endif
#ifndef GRASS_KHOP_MIN_BLOCKS
#define GRASS_KHOP_MIN_BLOCKS 4
#endif
// Words of a warp's draw-staging buffers (dynamic shared memory).
constexpr uint32_t kKhopBufWords = GRASS_KHOP_INFLIGHT * 32 * kDrawBufWords;

// k-hop.  One warp per seed (khop_seed_warp).

template <int MODE>
__global__ void __launch_bounds__(256, GRASS_KHOP_MIN_BLOCKS) khop_kernel(DevGraph g, const uint32_t *__restrict__ seeds,
                                                   uint64_t S, KhopArgs A,
                                                   unsigned long long *edges, unsigned int *err) {
  __shared__ SmemHdr sh[8];
  extern __shared__ __align__(16) uint32_t khop_dbuf[];  // 8 warps x kKhopBufWords
  SmemHdr &my = sh[threadIdx.x >> 5];
  uint32_t *dbuf = khop_dbuf + (threadIdx.x >> 5) * kKhopBufWords;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  uint64_t cnt = 0;
  bool bad = false;
  for (uint64_t s = warp; s < S; s += nwarps)
    khop_seed_warp<MODE, GRASS_KHOP_INFLIGHT>(g, seeds, A, s, my, dbuf, cnt, bad);
  warp_add_u64(edges, cnt);
  if (bad && err) atomicOr(err, 1u);
}

// The CSR twin of khop_kernel: the same warp routine and draws, one column
// load per draw.
__global__ void __launch_bounds__(256, GRASS_KHOP_MIN_BLOCKS) khop_csr_kernel(DevCsr c, const uint32_t *__restrict__ seeds,
                                                       uint64_t S, KhopArgs A,
                                                       unsigned long long *edges) {
  __shared__ SmemHdr sh[8];
  SmemHdr &my = sh[threadIdx.x >> 5];
  DevGraph g{};
  g.n = c.n;
  g.mode = GRASS_MODE_CSR_INTERNAL;
  g.rowptr = c.rowptr;
  g.cols = c.cols;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  uint64_t cnt = 0;
  bool bad = false;
  for (uint64_t s = warp; s < S; s += nwarps)
    khop_seed_warp<2, GRASS_KHOP_INFLIGHT>(g, seeds, A, s, my, nullptr, cnt, bad);
  warp_add_u64(edges, cnt);
}

// ---------------------------------------------------------------------------
// Multi random walk.  One warp per sample; the walkers' vertices, degrees and
// a Fenwick tree of degrees (degree-proportional selection) live in shared
// memory; lane 0 runs the step chain, which is sequential by definition.

// Shared-memory state of one sample: vertices (16-byte padded) + records.
struct MrwLayout {
  uint32_t R;
  __host__ __device__ size_t vtx_bytes() const { return ((size_t)R * 4 + 15) / 16 * 16; }
  __host__ __device__ size_t bytes_per_warp() const { return vtx_bytes() + (size_t)R * 16; }
};

// Multi random walk, one sample per warp, the sample's state in shared memory.
// Resident 256-thread blocks per SM it is compiled for: each warp's step chain
// waits on dependent record and sector reads, so resident warps pay.  On
// 262,144 samples of 80 walkers x 100 steps (R-MAT s22 ef32) 4 blocks (64
// registers) ran 1.6x (LE) and 1.7x (GT) faster than the unbounded build
// (110-113 registers, 2 blocks), 1.25x faster than 3 blocks, and 1.1-1.2x
// faster than 5 or 6 (48 / 40 registers).
#ifndef GRASS_MRW_MIN_BLOCKS
#define GRASS_MRW_MIN_BLOCKS 4
#endif

template <int MODE>
__global__ void __launch_bounds__(256, GRASS_MRW_MIN_BLOCKS) mrw_kernel(DevGraph g, uint32_t *__restrict__ roots,
                                                  uint64_t S, uint32_t R, uint32_t T, int select,
                                                  uint64_t seed, uint32_t *__restrict__ src,
                                                  uint32_t *__restrict__ dst,
                                                  unsigned long long *edges, unsigned int *err) {
  extern __shared__ __align__(16) unsigned char smem[];
  const MrwLayout lay{R};
  const int lane = threadIdx.x & 31;
  unsigned char *base = smem + (threadIdx.x >> 5) * lay.bytes_per_warp();
  uint32_t *vtx = reinterpret_cast<uint32_t *>(base);
  uint4 *rec = reinterpret_cast<uint4 *>(base + lay.vtx_bytes());
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  uint64_t cnt = 0;
  bool bad = false;
  for (uint64_t s = warp; s < S; s += nwarps) {
    uint32_t *rt = roots + s * R;
    for (uint32_t i = lane; i < R; i += 32) vtx[i] = rt[i];
    __syncwarp();
    mrw_warp<MODE>(g, vtx, rec, R, T, select, seed, s, src, dst, cnt, bad);
    __syncwarp();
    for (uint32_t i = lane; i < R; i += 32) rt[i] = vtx[i];
    __syncwarp();
  }
  warp_add_u64(edges, cnt);
  if (bad && err) atomicOr(err, 1u);
}

// Same with the state in global memory (roots in place, rec = S*R records of
// scratch): any number of walkers per sample.
template <int MODE>
__global__ void __launch_bounds__(256) mrw_global_kernel(DevGraph g, uint32_t *__restrict__ roots,
                                                         uint4 *__restrict__ rec, uint64_t S,
                                                         uint32_t R, uint32_t T, int select,
                                                         uint64_t seed, uint32_t *__restrict__ src,
                                                         uint32_t *__restrict__ dst,
                                                         unsigned long long *edges,
                                                         unsigned int *err) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  uint64_t cnt = 0;
  bool bad = false;
  for (uint64_t s = warp; s < S; s += nwarps)
    mrw_warp<MODE>(g, roots + s * R, rec + s * R, R, T, select, seed, s, src, dst, cnt, bad);
  warp_add_u64(edges, cnt);
  if (bad && err) atomicOr(err, 1u);
}

// Multi random walk, one block per sample, walkers in parallel (mrw_cta.cuh);
// scratch holds `stride` bytes per block, reused for its samples.
template <int MODE>
__global__ void __launch_bounds__(512) mrw_cta_kernel(DevGraph g, uint32_t *__restrict__ roots,
                                                      uint64_t S, uint32_t R, uint32_t T,
                                                      uint32_t select, uint64_t seed,
                                                      uint32_t *__restrict__ src,
                                                      uint32_t *__restrict__ dst,
                                                      unsigned char *scratch, uint64_t stride,
                                                      unsigned long long *edges,
                                                      unsigned int *err) {
  __shared__ CtaSmem<16> sm;
  unsigned char *scr = scratch + blockIdx.x * stride;
  uint64_t cnt = 0;
  bool bad = false;
  for (uint64_t s = blockIdx.x; s < S; s += gridDim.x)
    mrw_cta_sample<MODE, 16>(g, roots + s * R, src + s * T, dst + s * T, R, T, select, seed, s,
                             scr, sm, cnt, bad);
  warp_add_u64(edges, cnt);
  if (bad && err) atomicOr(err, 1u);
}

__global__ void starts_kernel(uint64_t n, uint64_t count, uint64_t seed, uint32_t tag,
                              uint32_t *out) {
  const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; q * 4 < count; q += nt) {
    const u32x4 r = philox4x32_10(seed, (uint32_t)q, 0, 0, tag);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint64_t i = q * 4 + k;
      if (i < count) out[i] = mulhi_u32(pick(r, k), (uint32_t)n);
    }
  }
}

unsigned grid_warps(uint64_t units, int units_per_block, int device, int per_sm) {
  const uint64_t need = (units + units_per_block - 1) / units_per_block;
  const uint64_t cap = (uint64_t)sm_count(device) * per_sm;
  return (unsigned)std::max<uint64_t>(1, std::min(need, cap));
}

int cur_dev() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

}  // namespace

void launch_uniform_starts(uint64_t n, uint64_t count, uint64_t seed, uint32_t *out,
                           cudaStream_t s, bool mrw_roots) {
  if (!count) return;
  starts_kernel<<<grid_warps((count + 3) / 4, 256, cur_dev(), 8), 256, 0, s>>>(
      n, count, seed, mrw_roots ? TAG_MRW_ROOT : TAG_START, out);
  count_launch();
}

// Launch through cudaLaunchKernelEx so the L2 window is a per-launch
// attribute: the caller's stream keeps its own access policy.
template <class... ExpTypes, class... ActTypes>
static void launch_with_window(void (*kern)(ExpTypes...), unsigned grid, unsigned block,
                               cudaStream_t s, const L2Window &win, ActTypes &&...args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  if (win.on()) {
    attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
    attr[0].val.accessPolicyWindow.base_ptr = const_cast<void *>(win.base);
    attr[0].val.accessPolicyWindow.num_bytes = win.bytes;
    attr[0].val.accessPolicyWindow.hitRatio = win.hit_ratio;
    attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  cudaLaunchKernelEx(&cfg, kern, std::forward<ActTypes>(args)...);
}

int apply_tuning(int device, const grass_tuning &t, const void *base, size_t bytes,
                 L2Window &win) {
  win = L2Window();
  if (t.l2_fetch_bytes) {
    cudaError_t e = cudaDeviceSetLimit(cudaLimitMaxL2FetchGranularity, t.l2_fetch_bytes);
    if (e != cudaSuccess) return cuda_fail(e, "cudaLimitMaxL2FetchGranularity");
  }
  if (t.l2_persist && base && bytes) {
    int max_persist = 0, max_window = 0;
    cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, device);
    cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, device);
    if (max_persist > 0 && max_window > 0) {
      const size_t carve = std::min<size_t>((size_t)max_persist, bytes);
      cudaError_t e = cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, carve);
      if (e != cudaSuccess) return cuda_fail(e, "cudaLimitPersistingL2CacheSize");
      size_t got = 0;
      cudaDeviceGetLimit(&got, cudaLimitPersistingL2CacheSize);
      win.base = base;
      win.bytes = std::min<size_t>(bytes, (size_t)max_window);
      win.hit_ratio = (float)std::min(1.0, (double)got / (double)win.bytes);
    }
  }
  return GRASS_OK;
}

// Defaults measured on B200 (R-MAT s22 ef32, 1M walkers x 80, step-major
// paths): the LE walk is 2% faster with one walker per thread than with two
// or four (3.60 / 3.67 / 3.68 ms), the CSR walk 0.5% faster with four; GT,
// whose warps synchronise every step, is 11% faster with one than with two.
grass_tuning resolve_tuning(const grass_tuning &t, int kind) {
  grass_tuning r = t;
  if (!r.rw_depth) r.rw_depth = kind == 2 ? 4 : 1;
  if (!r.rw_threads) r.rw_threads = 256;
  return r;  // rw_blocks_per_sm == 0: as many as are resident
}

// Grid for a grid-stride kernel: the requested blocks per SM, capped by
// what the occupancy calculator says is resident, times the SM count, and
// no more blocks than there is work for.
template <class K>
static unsigned resident_grid(K kern, int threads, uint32_t want_per_sm, uint64_t units,
                              uint64_t units_per_block) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0);
  if (per_sm < 1) per_sm = 1;
  if (want_per_sm && (int)want_per_sm < per_sm) per_sm = (int)want_per_sm;
  const uint64_t need = (units + units_per_block - 1) / units_per_block;
  const uint64_t cap = (uint64_t)sm_count(cur_dev()) * per_sm;
  return (unsigned)std::max<uint64_t>(1, std::min(need, cap));
}

template <int MODE, int DEPTH>
static void rw_launch_depth(const DevGraph &g, const grass_rw_params &p, const uint32_t *starts,
                            uint64_t W, uint32_t *paths, unsigned long long *edges,
                            unsigned int *err, cudaStream_t s, const grass_tuning &t,
                            const L2Window &win, uint64_t w0) {
  auto kern = rw_kernel<MODE, DEPTH>;
  const unsigned grid =
      resident_grid(kern, (int)t.rw_threads, t.rw_blocks_per_sm, W, (uint64_t)t.rw_threads * DEPTH);
  launch_with_window(kern, grid, t.rw_threads, s, win, g, starts, W, p.length, p.seed, w0,
                     (int)p.layout, paths, edges, err);
}

template <int MODE>
static void rw_dispatch(const DevGraph &g, const grass_rw_params &p, const uint32_t *starts,
                        uint64_t W, uint32_t *paths, unsigned long long *edges,
                        unsigned int *err, cudaStream_t s, const grass_tuning &t,
                        const L2Window &win, uint64_t w0) {
  switch (t.rw_depth) {
    case 1: rw_launch_depth<MODE, 1>(g, p, starts, W, paths, edges, err, s, t, win, w0); break;
    case 4: rw_launch_depth<MODE, 4>(g, p, starts, W, paths, edges, err, s, t, win, w0); break;
    default: rw_launch_depth<MODE, 2>(g, p, starts, W, paths, edges, err, s, t, win, w0);
  }
}

void launch_rw(const DevGraph &g, const grass_rw_params &p, const uint32_t *starts, uint64_t W,
               uint32_t *paths, unsigned long long *edges, unsigned int *err, cudaStream_t s,
               const grass_tuning &tin, const L2Window &win, uint64_t w0) {
  if (!W) return;
  const grass_tuning t = resolve_tuning(tin, g.mode);
  if (g.mode == GRASS_MODE_GT) rw_dispatch<0>(g, p, starts, W, paths, edges, err, s, t, win, w0);
  else rw_dispatch<1>(g, p, starts, W, paths, edges, err, s, t, win, w0);
  count_launch();
}

uint64_t launch_random_read(const uint32_t *buf, uint64_t n_words, uint64_t reads, uint64_t seed,
                            unsigned long long *sink, cudaStream_t s) {
  const unsigned grid = (unsigned)sm_count(cur_dev()) * 8;
  const uint64_t threads = (uint64_t)grid * 256;
  const uint64_t per_thread = ((reads + threads - 1) / threads + 7) / 8 * 8;
  random_read_kernel<<<grid, 256, 0, s>>>(buf, n_words - 1, per_thread, seed, sink);
  count_launch();
  return per_thread * threads;
}

void launch_rw_account(const DevGraph &g, const grass_rw_params &p, const uint32_t *starts,
                       uint64_t W, unsigned long long *out, cudaStream_t s) {
  if (!W) return;
  const unsigned grid = grid_warps(W, 256, cur_dev(), 8);
  if (g.mode == GRASS_MODE_GT)
    rw_account_kernel<0><<<grid, 256, 0, s>>>(g, starts, W, p.length, p.seed, out);
  else
    rw_account_kernel<1><<<grid, 256, 0, s>>>(g, starts, W, p.length, p.seed, out);
  count_launch();
}

void launch_rw_csr(const DevCsr &c, const grass_rw_params &p, const uint32_t *starts,
                   uint64_t W, uint32_t *paths, unsigned long long *edges, cudaStream_t s,
                   const grass_tuning &tin, const L2Window &win, uint64_t w0) {
  if (!W) return;
  const grass_tuning t = resolve_tuning(tin, 2);
  const uint32_t L = p.length;
  const int lay = (int)p.layout;
  const int T = (int)t.rw_threads;
  switch (t.rw_depth) {
    case 1: {
      const unsigned grid = resident_grid(rw_csr_kernel<1>, T, t.rw_blocks_per_sm, W, T);
      launch_with_window(rw_csr_kernel<1>, grid, T, s, win, c, starts, W, L, p.seed, w0, lay,
                         paths, edges);
      break;
    }
    case 4: {
      const unsigned grid = resident_grid(rw_csr_kernel<4>, T, t.rw_blocks_per_sm, W, T * 4);
      launch_with_window(rw_csr_kernel<4>, grid, T, s, win, c, starts, W, L, p.seed, w0, lay,
                         paths, edges);
      break;
    }
    default: {
      const unsigned grid = resident_grid(rw_csr_kernel<2>, T, t.rw_blocks_per_sm, W, T * 2);
      launch_with_window(rw_csr_kernel<2>, grid, T, s, win, c, starts, W, L, p.seed, w0, lay,
                         paths, edges);
    }
  }
  count_launch();
}

static KhopArgs khop_args(const grass_khop_params &p, uint32_t *const *hop_out) {
  KhopArgs A{};
  A.hops = p.hops;
  uint64_t w = 1;
  for (uint32_t h = 0; h < p.hops; h++) {
    A.fan[h] = p.fanouts[h];
    w *= p.fanouts[h];
    A.width[h] = w;
    A.out[h] = hop_out[h];
  }
  A.seed = p.seed;
  return A;
}

void launch_khop(const DevGraph &g, const grass_khop_params &p, const uint32_t *seeds,
                 uint64_t S, uint32_t *const *hop_out, unsigned long long *edges,
                 unsigned int *err, cudaStream_t s) {
  if (!S) return;
  const KhopArgs A = khop_args(p, hop_out);
  const unsigned grid = grid_warps(S, 8, cur_dev(), 8);
  const uint32_t smem = 8 * kKhopBufWords * 4;
  static std::once_flag once;  // opt in to more than 48 KB of shared memory
  std::call_once(once, [&] {
    cudaFuncSetAttribute(khop_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaFuncSetAttribute(khop_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  if (g.mode == GRASS_MODE_GT)
    khop_kernel<0><<<grid, 256, smem, s>>>(g, seeds, S, A, edges, err);
  else
    khop_kernel<1><<<grid, 256, smem, s>>>(g, seeds, S, A, edges, err);
  count_launch();
}

void launch_node2vec(const DevGraph &g, const grass_node2vec_params &p, const uint64_t t[3],
                     const uint32_t *starts, uint64_t W, uint32_t *paths,
                     unsigned long long *edges, unsigned int *err, cudaStream_t s, uint64_t w0) {
  if (!W) return;
  N2vArgs a;
  a.L = p.length;
  a.max_tries = p.max_tries;
  a.layout = (int)p.layout;
  a.seed = p.seed;
  a.w0 = w0;
  a.t_ret = t[0];
  a.t_in = t[1];
  a.t_out = t[2];
  const unsigned grid = grid_warps(W, 256, cur_dev(), 8);
  if (g.mode == GRASS_MODE_GT) n2v_kernel<0><<<grid, 256, 0, s>>>(g, starts, W, a, paths, edges, err);
  else if (g.mode == GRASS_MODE_LE) n2v_kernel<1><<<grid, 256, 0, s>>>(g, starts, W, a, paths, edges, err);
  else n2v_kernel<2><<<grid, 256, 0, s>>>(g, starts, W, a, paths, edges, err);
  count_launch();
}

void launch_khop_csr(const DevCsr &c, const grass_khop_params &p, const uint32_t *seeds,
                     uint64_t S, uint32_t *const *hop_out, unsigned long long *edges,
                     cudaStream_t s) {
  if (!S) return;
  const KhopArgs A = khop_args(p, hop_out);
  khop_csr_kernel<<<grid_warps(S, 8, cur_dev(), 8), 256, 0, s>>>(c, seeds, S, A, edges);
  count_launch();
}

int launch_mrw(const DevGraph &g, const grass_mrw_params &p, uint32_t *roots, uint64_t S,
               uint32_t *src, uint32_t *dst, unsigned long long *edges, unsigned int *err,
               cudaStream_t s) {
  if (!S || !p.steps) return GRASS_OK;
  // Block per sample (walkers in parallel) for continuous-time selection, and
  // for uniform selection when there are few samples or long chains (same
  // output as the warp kernels).
  if (p.select == GRASS_SELECT_DEGREE_CT ||
      (p.select == GRASS_SELECT_UNIFORM &&
       (p.steps >= 1024 || S < (uint64_t)sm_count(cur_dev()) * 8))) {
    const int threads = (int)std::min<uint64_t>(
        512, std::max<uint64_t>(128, ((uint64_t)p.walkers / 2 + 31) / 32 * 32));
    auto kern = g.mode == GRASS_MODE_GT ? mrw_cta_kernel<0> : mrw_cta_kernel<1>;
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, 0);
    const uint64_t grid =
        std::min<uint64_t>(S, (uint64_t)sm_count(cur_dev()) * std::max(per_sm, 1));
    const uint64_t stride = mrw_sample_scratch(p.walkers, p.steps, p.select);
    unsigned char *scr = nullptr;
    cudaError_t e = scratch_alloc(reinterpret_cast<void **>(&scr), grid * stride, s);
    if (e != cudaSuccess) return cuda_fail(e, "multi-RW scratch");
    kern<<<(unsigned)grid, threads, 0, s>>>(g, roots, S, p.walkers, p.steps, p.select, p.seed, src,
                                            dst, scr, stride, edges, err);
    count_launch();
    scratch_free(scr, s);
    return GRASS_OK;
  }
  const MrwLayout lay{p.walkers};
  const size_t per_warp = lay.bytes_per_warp();
  if (per_warp > 48 * 1024) {
    // Too many walkers for shared memory: the state lives in global scratch.
    uint4 *rec = nullptr;
    cudaError_t e =
        scratch_alloc(reinterpret_cast<void **>(&rec), S * (uint64_t)p.walkers * sizeof(uint4), s);
    if (e != cudaSuccess) return cuda_fail(e, "multi-RW scratch");
    auto kern = g.mode == GRASS_MODE_GT ? mrw_global_kernel<0> : mrw_global_kernel<1>;
    kern<<<grid_warps(S, 8, cur_dev(), 8), 256, 0, s>>>(g, roots, rec, S, p.walkers, p.steps,
                                                        (int)p.select, p.seed, src, dst, edges,
                                                        err);
    count_launch();
    scratch_free(rec, s);
    return GRASS_OK;
  }
  const size_t budget = 200 * 1024;
  const int warps = (int)std::min<size_t>(8, budget / per_warp);
  const size_t smem = per_warp * warps;
  auto kern = g.mode == GRASS_MODE_GT ? mrw_kernel<0> : mrw_kernel<1>;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const unsigned grid = grid_warps(S, warps, cur_dev(), 8);
  kern<<<grid, warps * 32, smem, s>>>(g, roots, S, p.walkers, p.steps, (int)p.select, p.seed,
                                       src, dst, edges, err);
  count_launch();
  return GRASS_OK;
}

}  // namespace grass
