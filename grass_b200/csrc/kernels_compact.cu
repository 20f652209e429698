// kernels_compact.cu -- output compaction: fixed-shape sampler outputs to a
// dense (src, dst) edge list.
//
// The reference cuts invalid walkers out of each step's frontier: it radix
// sorts the (transit, sample) pairs, finds the first INVALID_VERTEX with a
// binary search kernel (invalidVertexStartPos, GT/src/grass.cu:1085-1117,
// launched :1641) and truncates there.  The samplers here never sort; they
// write fixed-shape outputs with GRASS_INVALID_VERTEX in the slots that a dead
// end leaves empty.  Compaction is a separate, order-preserving pass for
// callers that want only the sampled edges:
//   1. count: one valid-entry count per tile of 4096 entries (ballot/popc);
//   2. one exclusive scan over the tile counts;
//   3. fill: each warp owns 512 consecutive entries of a tile; a valid entry
//      is ranked inside its warp with __ballot_sync and __popc, among the
//      warps by a prefix over the eight warp counts, and written at tile
//      offset + rank -- the output keeps the input order.
// Parent indices advance incrementally (32 / div and 32 % div per step), so a
// lane divides once per tile, not once per entry.
#include <atomic>

#include "graph.h"

namespace grass {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kPer = 16;                     // slots per lane per tile
constexpr uint32_t kWarpSlots = 32 * kPer;   // a warp's contiguous chunk
constexpr uint32_t kTileEntries = kThreads * kPer;

// A segment as the kernels see it: adv_q / adv_r = 32 / div and 32 % div,
// the step of the (parent, slot) pair between a lane's consecutive slots.
struct KSeg {
  const uint32_t *parent;
  const uint32_t *child;
  uint64_t n, tile0;
  uint32_t div, adv_q, adv_r;
};

struct Plan {
  KSeg seg[kCompactMaxSegs];
  uint32_t nseg;
  uint64_t tiles;
};

// Slot cursor of one lane: slot e = q * div + r of its segment.
struct Cursor {
  uint64_t e, q, r;
};

// Finds the tile's segment and starts the lane at slot
// e0 + warp * kWarpSlots + lane.
__device__ __forceinline__ Cursor start(const Plan &pl, uint64_t tile, const KSeg *&sg) {
  uint32_t k = 0;
  while (k + 1 < pl.nseg && tile >= pl.seg[k + 1].tile0) k++;
  sg = &pl.seg[k];
  const uint32_t div = sg->div;
  const uint64_t e0 = (tile - sg->tile0) * kTileEntries;
  const uint32_t off = (threadIdx.x >> 5) * kWarpSlots + (threadIdx.x & 31);
  Cursor c;
  c.e = e0 + off;
  c.q = c.e / div;
  c.r = c.e - c.q * div;
  return c;
}

__device__ __forceinline__ void advance(Cursor &c, const KSeg &sg) {
  c.e += 32;
  c.q += sg.adv_q;
  c.r += sg.adv_r;
  if (c.r >= sg.div) {
    c.r -= sg.div;
    c.q++;
  }
}

// Child and parent indices of the slot under the cursor.
template <int KIND>
__device__ __forceinline__ uint64_t child_index(const Cursor &c, const KSeg &sg) {
  if constexpr (KIND == kCompactFan) return c.e;
  else return c.q * ((uint64_t)sg.div + 1) + c.r + 1;  // walk-major path
}
template <int KIND>
__device__ __forceinline__ uint64_t parent_index(const Cursor &c, const KSeg &sg) {
  if constexpr (KIND == kCompactFan) return c.q;
  else return c.q * ((uint64_t)sg.div + 1) + c.r;
}

template <int KIND>
__global__ void __launch_bounds__(kThreads) compact_count_kernel(Plan pl, uint32_t *counts) {
  __shared__ uint32_t wsum[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint64_t tile = blockIdx.x; tile < pl.tiles; tile += gridDim.x) {
    const KSeg *sg;
    Cursor c = start(pl, tile, sg);
    const uint64_t n = sg->n;
    uint32_t v[kPer];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      v[k] = c.e < n ? __ldg(sg->child + child_index<KIND>(c, *sg)) : GRASS_INVALID_VERTEX;
      advance(c, *sg);
    }
    uint32_t cnt = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++)
      cnt += __popc(__ballot_sync(0xffffffffu, v[k] != GRASS_INVALID_VERTEX));
    if (lane == 0) wsum[warp] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t s = 0;
#pragma unroll
      for (int w = 0; w < kWarps; w++) s += wsum[w];
      counts[tile] = s;
    }
    __syncthreads();
  }
}

// Each warp owns kWarpSlots consecutive slots of the tile: it ranks its valid
// slots with one ballot per 32, learns the counts of the warps before it
// through shared memory (the tile's only barrier), and writes in slot order.
// Resident 256-thread blocks per SM for the fill kernel: 4 (64 registers,
// with 40-148 bytes of spill).  On the k-hop (25, 10) frontiers of 65,536
// seeds (R-MAT s22 ef32) the whole compaction took 0.103 ms, against 0.118-
// 0.123 ms unbounded (96 / 76 registers, 2-3 blocks) and 0.111 ms at 3.
#ifndef GRASS_COMPACT_MIN_BLOCKS
#define GRASS_COMPACT_MIN_BLOCKS 4
#endif

template <int KIND>
__global__ void __launch_bounds__(kThreads, GRASS_COMPACT_MIN_BLOCKS)
    compact_fill_kernel(Plan pl, const uint64_t *offs, uint32_t *src, uint32_t *dst, uint64_t cap) {
  __shared__ uint32_t wsum[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t below = (1u << lane) - 1;
  for (uint64_t tile = blockIdx.x; tile < pl.tiles; tile += gridDim.x) {
    const KSeg *sg;
    Cursor c = start(pl, tile, sg);
    const uint64_t n = sg->n;
    uint32_t cv[kPer], pv[kPer];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      const bool in = c.e < n;
      cv[k] = in ? __ldg(sg->child + child_index<KIND>(c, *sg)) : GRASS_INVALID_VERTEX;
      pv[k] = in ? __ldg(sg->parent + parent_index<KIND>(c, *sg)) : GRASS_INVALID_VERTEX;
      advance(c, *sg);
    }
    uint32_t m[kPer], total = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      m[k] = __ballot_sync(0xffffffffu, cv[k] != GRASS_INVALID_VERTEX);
      total += __popc(m[k]);
    }
    if (lane == 0) wsum[warp] = total;
    __syncthreads();
    uint64_t pos = offs[tile];
#pragma unroll
    for (int w = 0; w < kWarps; w++) pos += w < warp ? wsum[w] : 0u;
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      const uint64_t at = pos + __popc(m[k] & below);
      if (((m[k] >> lane) & 1u) && at < cap) {
        store_out_u32(src + at, pv[k]);
        store_out_u32(dst + at, cv[k]);
      }
      pos += __popc(m[k]);
    }
    __syncthreads();
  }
}

template <int KIND>
void launch_kind(const Plan &pl, uint32_t *counts, uint64_t *offs, uint64_t *tmp, uint32_t *src,
                 uint32_t *dst, uint64_t cap, cudaStream_t s) {
  // resident blocks per SM, queried once (every device here is the same part)
  static std::atomic<int> cached{0};
  int per_sm = cached.load(std::memory_order_relaxed);
  if (!per_sm) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, compact_fill_kernel<KIND>, kThreads, 0);
    per_sm = std::max(per_sm, 1);
    cached.store(per_sm, std::memory_order_relaxed);
  }
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t resident = (uint64_t)sm_count(dev) * (uint64_t)per_sm * 4;
  const unsigned grid = (unsigned)std::min<uint64_t>(pl.tiles, resident);
  compact_count_kernel<KIND><<<grid, kThreads, 0, s>>>(pl, counts);
  launch_scan_u32(counts, pl.tiles, offs, tmp, s);
  compact_fill_kernel<KIND><<<grid, kThreads, 0, s>>>(pl, offs, src, dst, cap);
  count_launch(2);
}

}  // namespace

int launch_compact(const CompactSeg *segs, uint32_t nseg, uint32_t *src, uint32_t *dst,
                   uint64_t cap, unsigned long long *count, cudaStream_t s) {
  if (nseg == 0 || nseg > kCompactMaxSegs) return set_error(GRASS_E_ARG, "compaction: bad segment count");
  Plan pl{};
  pl.nseg = nseg;
  uint64_t tiles = 0;
  for (uint32_t k = 0; k < nseg; k++) {
    if (segs[k].kind != segs[0].kind) return set_error(GRASS_E_ARG, "compaction: mixed segment kinds");
    KSeg &q = pl.seg[k];
    q.parent = segs[k].parent;
    q.child = segs[k].child;
    q.n = segs[k].n;
    q.div = segs[k].div ? segs[k].div : 1u;
    q.adv_q = 32u / q.div;
    q.adv_r = 32u % q.div;
    q.tile0 = tiles;
    tiles += (segs[k].n + kTileEntries - 1) / kTileEntries;
  }
  pl.tiles = tiles;
  if (tiles == 0) {
    cudaError_t e = cudaMemsetAsync(count, 0, sizeof(unsigned long long), s);
    return e == cudaSuccess ? GRASS_OK : cuda_fail(e, "compaction count");
  }
  const uint64_t cnt_words = (tiles + 1) / 2;  // u32 counts in u64 words
  const uint64_t words = cnt_words + (tiles + 1) + scan_tmp_words(tiles);
  uint64_t *scr = nullptr;
  cudaError_t e = scratch_alloc(reinterpret_cast<void **>(&scr), words * sizeof(uint64_t), s);
  if (e != cudaSuccess) return cuda_fail(e, "compaction scratch");
  uint32_t *counts = reinterpret_cast<uint32_t *>(scr);
  uint64_t *offs = scr + cnt_words;
  uint64_t *tmp = offs + tiles + 1;
  if (segs[0].kind == kCompactFan) launch_kind<kCompactFan>(pl, counts, offs, tmp, src, dst, cap, s);
  else launch_kind<kCompactPath>(pl, counts, offs, tmp, src, dst, cap, s);
  e = cudaMemcpyAsync(count, offs + tiles, sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
  scratch_free(scr, s);
  return e == cudaSuccess ? GRASS_OK : cuda_fail(e, "compaction count");
}

}  // namespace grass
