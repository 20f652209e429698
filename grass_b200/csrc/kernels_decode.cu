// kernels_decode.cu -- decode-only sweep: every neighbor list into CSR.
//
// Replaces the reference's two decoders for whole lists: the block-cooperative
// GlobalDecoder (GT/src/bcg.cuh:171-345, used by the grid/thread-block
// kernels at GT/src/grass.cu:529-553, 762-786) and repeated
// BCGVertex::get_vertex calls (LE/src/bcg.cuh:195-261).
//
// Layout of the work: one warp takes a tile of 32 consecutive vertices.
//  1. Each lane decodes the gamma header of one vertex (variable-length codes,
//     so lanes work on independent vertices).
//  2. A warp prefix sum of the degrees maps the tile's neighbor lists onto
//     one contiguous index space; each round, lane j takes neighbor r*32+j,
//     finds its vertex by a shuffle binary search and reads its own field.
//  3. GT: the fields are heads and gaps, so a segmented warp scan (segments =
//     blocks; a carry crosses rounds) turns gaps into ids.  LE: each neighbor
//     is two rocks plus one signed sea, no scan.
//  4. Stores are coalesced: the tile's output is contiguous in cols.
#include "graph.h"

namespace grass {

namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;

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

template <int MODE>
__global__ void __launch_bounds__(256) decode_all_kernel(DevGraph g, const uint64_t *rowptr,
                                                           uint32_t *cols, unsigned int *err) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t tiles = ((uint64_t)g.n + 31) / 32;
  bool bad = false;
  for (uint64_t t = warp; t < tiles; t += nwarps) {
    const uint64_t v = t * 32 + lane;
    VHdr h;
    if (v < g.n) {
      h = header<MODE>(g, (uint32_t)v);
    } else {
      h.d = 0;
      h.P = 0;
      h.v = 0;
      h.bn = h.bl = h.om = h.fp = 0;
      h.a = h.b = 0;
    }
    // exclusive prefix of degrees across the tile
    uint32_t incl = h.d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t excl = incl - h.d;
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    const uint64_t out0 = rowptr[t * 32];
    uint32_t carry = 0;
    for (uint32_t r = 0; r < total; r += 32) {
      const uint32_t gi = r + lane;
      const bool active = gi < total;
      // largest k with excl[k] <= gi (a non-empty list when gi < total)
      int k = 0;
#pragma unroll
      for (int step = 16; step > 0; step >>= 1) {
        uint32_t e = __shfl_sync(FULL, excl, k + step);
        if (e <= gi) k += step;
      }
      const VHdr hk = shfl_hdr(h, k);
      const uint32_t i = gi - __shfl_sync(FULL, excl, k);
      uint32_t val = 0;
      if (MODE == 1) {
        if (active) val = le_neighbor(g, hk, i);
      } else {
        // field of neighbor i: the block head (id == 0) or a gap
        bool head = true;
        uint32_t x = 0;
        if (active) {
          const uint32_t split = (hk.bl + 1) * hk.om;
          const bool flag = i < split;
          const uint32_t j = flag ? i : i - split;
          const uint32_t len = hk.bl + (flag ? 1u : 0u);
          uint32_t blk = j / len;
          const uint32_t id = j - blk * len;
          if (!flag) blk += hk.om;
          const uint64_t bpos = hk.P + (uint64_t)blk * (uint64_t)(hk.a + (hk.bl - 1) * hk.b) +
                                (uint64_t)min(blk, hk.om) * (uint64_t)hk.b;
          if (id == 0) {
            const uint32_t hv = read_field(g.words, bpos, hk.a);
            x = (blk >= hk.fp) ? hk.v + hv + 1u : hk.v - hv - 1u;
          } else {
            head = false;
            x = read_field(g.words, bpos + hk.a + (uint64_t)(id - 1) * hk.b, hk.b) + 1u;
          }
        }
        if (lane == 0 && !head) {
          x += carry;
          head = true;
        }
        // segmented inclusive scan (segments start at heads)
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          uint32_t y = __shfl_up_sync(FULL, x, o);
          int f = __shfl_up_sync(FULL, (int)head, o);
          if (lane >= o && !head) {
            x += y;
            head = f;
          }
        }
        carry = __shfl_sync(FULL, x, 31);
        val = x;
      }
      if (active) {
        if (val >= g.n) bad = true;
        cols[out0 + gi] = val;
      }
    }
  }
  if (bad && err) atomicOr(err, 1u);
}

}  // namespace

void launch_decode_all(const DevGraph &g, const uint64_t *rowptr, uint32_t *cols,
                       unsigned int *err, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t tiles = ((uint64_t)g.n + 31) / 32;
  const uint64_t blocks_needed = (tiles + 7) / 8;
  const unsigned grid = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>(blocks_needed, (uint64_t)sm_count(dev) * 8));
  if (g.mode == GRASS_MODE_GT) decode_all_kernel<0><<<grid, 256, 0, s>>>(g, rowptr, cols, err);
  else decode_all_kernel<1><<<grid, 256, 0, s>>>(g, rowptr, cols, err);
  count_launch();
}

}  // namespace grass
