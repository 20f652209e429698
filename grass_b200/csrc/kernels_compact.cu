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
//   3. fill: each valid entry is ranked inside its warp with __ballot_sync and
//      __popc, inside the block by a prefix over the eight warp counts, and
//      written at tile offset + rank -- the output keeps the input order.
#include "graph.h"

namespace grass {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kPer = 16;
constexpr uint32_t kTileEntries = kThreads * kPer;

struct Plan {
  CompactSeg seg[kCompactMaxSegs];
  uint32_t nseg;
  uint64_t tiles;
};

// q0 + r / div, r % div for r = r0 + off, with r0 < div and off < kTileEntries:
// the quotient step is 0 or 1 unless div is below the tile size, where r fits
// 32 bits.
__device__ __forceinline__ void step_div(uint64_t r, uint32_t div, uint64_t &qa, uint32_t &rem) {
  if (r < div) {
    qa = 0;
    rem = (uint32_t)r;
  } else if (div >= kTileEntries) {
    qa = 1;
    rem = (uint32_t)(r - div);
  } else {
    const uint32_t rr = (uint32_t)r;
    qa = rr / div;
    rem = rr - (uint32_t)qa * div;
  }
}

struct TilePos {
  const CompactSeg *sg;
  uint64_t e0, q0;
  uint32_t r0;
};

__device__ __forceinline__ TilePos locate(const Plan &pl, uint64_t tile) {
  uint32_t k = 0;
  while (k + 1 < pl.nseg && tile >= pl.seg[k + 1].tile0) k++;
  TilePos t;
  t.sg = &pl.seg[k];
  t.e0 = (tile - t.sg->tile0) * kTileEntries;
  t.q0 = t.e0 / t.sg->div;
  t.r0 = (uint32_t)(t.e0 - t.q0 * t.sg->div);
  return t;
}

// Index of entry e0 + off's child; *pidx receives its parent's index.
__device__ __forceinline__ uint64_t entry_index(const TilePos &t, uint32_t off, uint64_t *pidx) {
  uint64_t qa;
  uint32_t rem;
  step_div((uint64_t)t.r0 + off, t.sg->div, qa, rem);
  const uint64_t q = t.q0 + qa;
  if (t.sg->kind == kCompactFan) {
    *pidx = q;
    return t.e0 + off;
  }
  // walk-major paths: edge (q, rem) joins path[q][rem] -> path[q][rem + 1]
  const uint64_t i = q * ((uint64_t)t.sg->div + 1) + rem;
  *pidx = i;
  return i + 1;
}

__global__ void __launch_bounds__(kThreads) compact_count_kernel(Plan pl, uint32_t *counts) {
  __shared__ uint32_t wsum[kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint64_t tile = blockIdx.x; tile < pl.tiles; tile += gridDim.x) {
    const TilePos t = locate(pl, tile);
    const uint64_t n = t.sg->n;
    uint32_t v[kPer];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      const uint32_t off = k * kThreads + threadIdx.x;
      uint64_t pi;
      const uint64_t ci = entry_index(t, off, &pi);
      v[k] = t.e0 + off < n ? __ldg(t.sg->child + ci) : GRASS_INVALID_VERTEX;
    }
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kPer; k++) c += __popc(__ballot_sync(0xffffffffu, v[k] != GRASS_INVALID_VERTEX));
    if (lane == 0) wsum[warp] = c;
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

__global__ void __launch_bounds__(kThreads)
    compact_fill_kernel(Plan pl, const uint64_t *offs, uint32_t *src, uint32_t *dst, uint64_t cap) {
  __shared__ uint32_t wcnt[2][kWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t below = (1u << lane) - 1;
  for (uint64_t tile = blockIdx.x; tile < pl.tiles; tile += gridDim.x) {
    const TilePos t = locate(pl, tile);
    const uint64_t n = t.sg->n;
    uint32_t cv[kPer], pv[kPer];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      const uint32_t off = k * kThreads + threadIdx.x;
      uint64_t pi;
      const uint64_t ci = entry_index(t, off, &pi);
      const bool in = t.e0 + off < n;
      cv[k] = in ? __ldg(t.sg->child + ci) : GRASS_INVALID_VERTEX;
      pv[k] = in ? __ldg(t.sg->parent + pi) : GRASS_INVALID_VERTEX;
    }
    uint64_t base = offs[tile];
#pragma unroll
    for (int k = 0; k < kPer; k++) {
      const bool ok = cv[k] != GRASS_INVALID_VERTEX;
      const uint32_t m = __ballot_sync(0xffffffffu, ok);
      // wcnt[k & 1] is rewritten at round k + 2, after every thread passed the
      // barrier of round k + 1, so one barrier per round suffices.
      if (lane == 0) wcnt[k & 1][warp] = __popc(m);
      __syncthreads();
      uint32_t before = 0, total = 0;
#pragma unroll
      for (int w = 0; w < kWarps; w++) {
        const uint32_t c = wcnt[k & 1][w];
        before += w < warp ? c : 0;
        total += c;
      }
      const uint64_t pos = base + before + __popc(m & below);
      if (ok && pos < cap) {
        store_out_u32(src + pos, pv[k]);
        store_out_u32(dst + pos, cv[k]);
      }
      base += total;
    }
    __syncthreads();
  }
}

}  // namespace

int launch_compact(const CompactSeg *segs, uint32_t nseg, uint32_t *src, uint32_t *dst,
                   uint64_t cap, unsigned long long *count, cudaStream_t s) {
  if (nseg == 0 || nseg > kCompactMaxSegs) return set_error(GRASS_E_ARG, "compaction: bad segment count");
  Plan pl{};
  pl.nseg = nseg;
  uint64_t tiles = 0;
  for (uint32_t k = 0; k < nseg; k++) {
    pl.seg[k] = segs[k];
    if (pl.seg[k].div == 0) pl.seg[k].div = 1;
    pl.seg[k].tile0 = tiles;
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
  cudaError_t e = cudaMallocAsync(&scr, words * sizeof(uint64_t), s);
  if (e != cudaSuccess) return cuda_fail(e, "compaction scratch");
  uint32_t *counts = reinterpret_cast<uint32_t *>(scr);
  uint64_t *offs = scr + cnt_words;
  uint64_t *tmp = offs + tiles + 1;
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)sm_count(dev) * 8);
  compact_count_kernel<<<grid, kThreads, 0, s>>>(pl, counts);
  launch_scan_u32(counts, tiles, offs, tmp, s);
  compact_fill_kernel<<<grid, kThreads, 0, s>>>(pl, offs, src, dst, cap);
  count_launch(2);
  e = cudaMemcpyAsync(count, offs + tiles, sizeof(uint64_t), cudaMemcpyDeviceToDevice, s);
  cudaFreeAsync(scr, s);
  return e == cudaSuccess ? GRASS_OK : cuda_fail(e, "compaction count");
}

}  // namespace grass
