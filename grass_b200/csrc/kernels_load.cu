// kernels_load.cu -- device side of graph loading.
//
// Replaces copyPartitionToGPU (GT/src/utils.hpp:360-386): the reference
// expands the packed .offset lengths with decode_offset (GT/src/bcg.cuh:
// 368-412, one thread per vertex, grid min(8192, n/256) -- zero blocks when
// n < 256) and then runs cub::DeviceScan::ExclusiveSum.  Here the unpack is
// fused into a reduce-then-scan over 4096-vertex tiles, and a validation pass
// checks every header against its length field once, so sampling kernels can
// trust headers without per-draw bounds checks.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "graph.h"

namespace grass {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kTile = kScanThreads * kScanItems;

__global__ void bswap_kernel(uint32_t *w, uint64_t n_words) {
  uint64_t n4 = n_words / 4;
  uint4 *w4 = reinterpret_cast<uint4 *>(w);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n4;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint4 x = w4[i];
    x.x = __byte_perm(x.x, 0, 0x0123);
    x.y = __byte_perm(x.y, 0, 0x0123);
    x.z = __byte_perm(x.z, 0, 0x0123);
    x.w = __byte_perm(x.w, 0, 0x0123);
    w4[i] = x;
  }
  uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (t < n_words - n4 * 4) w[n4 * 4 + t] = __byte_perm(w[n4 * 4 + t], 0, 0x0123);
}

struct FieldLoader {  // n ubl-bit big-endian fields, ubl in [1, 64]
  const uint32_t *payload;
  uint32_t ubl;
  __device__ __forceinline__ uint64_t operator()(uint64_t u) const {
    const uint64_t bit = u * ubl;
    if (ubl <= 32) return read_field(payload, bit, (int)ubl);
    uint64_t hi = read_field(payload, bit, (int)ubl - 32);
    return (hi << 32) | read_field(payload, bit + ubl - 32, 32);
  }
};

struct CountLoader {
  const uint32_t *counts;
  __device__ __forceinline__ uint64_t operator()(uint64_t u) const { return counts[u]; }
};

// Reads u64 values that tile_scan may overwrite in place: every CTA reads its
// whole tile before its block scan and writes only after it.
struct U64Loader {
  const uint64_t *vals;
  __device__ __forceinline__ uint64_t operator()(uint64_t u) const { return vals[u]; }
};

template <class Loader>
__global__ void __launch_bounds__(kScanThreads) tile_reduce(Loader ld, uint64_t n,
                                                              uint64_t *tile_sums) {
  using BR = cub::BlockReduce<uint64_t, kScanThreads>;
  __shared__ typename BR::TempStorage tmp;
  const uint64_t base = (uint64_t)blockIdx.x * kTile;
  uint64_t sum = 0;
#pragma unroll 4
  for (int k = 0; k < kScanItems; k++) {
    uint64_t u = base + (uint64_t)k * kScanThreads + threadIdx.x;
    if (u < n) sum += ld(u);
  }
  uint64_t tot = BR(tmp).Sum(sum);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = tot;
}

// Exclusive scan of T tile sums in place by one CTA; tile_sums[T] = total.
__global__ void __launch_bounds__(1024) scan_tile_sums(uint64_t *ts, uint64_t T) {
  using BS = cub::BlockScan<uint64_t, 1024>;
  __shared__ typename BS::TempStorage tmp;
  const uint64_t per = (T + 1023) / 1024;
  const uint64_t b = threadIdx.x * per, e = min(T, b + per);
  uint64_t local = 0;
  for (uint64_t i = b; i < e; i++) local += ts[i];
  uint64_t excl, total;
  BS(tmp).ExclusiveSum(local, excl, total);
  for (uint64_t i = b; i < e; i++) {
    uint64_t x = ts[i];
    ts[i] = excl;
    excl += x;
  }
  if (threadIdx.x == 0) ts[T] = total;
}

template <class Loader>
__global__ void __launch_bounds__(kScanThreads) tile_scan(Loader ld, uint64_t n,
                                                            const uint64_t *tile_sums,
                                                            uint64_t *out) {
  using BS = cub::BlockScan<uint64_t, kScanThreads>;
  __shared__ typename BS::TempStorage tmp;
  const uint64_t base = (uint64_t)blockIdx.x * kTile + (uint64_t)threadIdx.x * kScanItems;
  uint64_t vals[kScanItems];
  uint64_t sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint64_t u = base + k;
    vals[k] = u < n ? ld(u) : 0;
    sum += vals[k];
  }
  uint64_t excl;
  BS(tmp).ExclusiveSum(sum, excl);
  excl += tile_sums[blockIdx.x];
#pragma unroll
  for (int k = 0; k < kScanItems; k++) {
    uint64_t u = base + k;
    if (u < n) out[u] = excl;
    excl += vals[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
    const uint64_t T = gridDim.x;
    out[n] = tile_sums[T];
  }
}

template <class Loader>
void scan_impl(Loader ld, uint64_t n, uint64_t *out, uint64_t *tmp, cudaStream_t s) {
  const uint64_t T = (n + kTile - 1) / kTile;
  if (T == 0) {
    cudaMemsetAsync(out, 0, sizeof(uint64_t), s);
    return;
  }
  tile_reduce<<<(unsigned)T, kScanThreads, 0, s>>>(ld, n, tmp);
  scan_tile_sums<<<1, 1024, 0, s>>>(tmp, T);
  tile_scan<<<(unsigned)T, kScanThreads, 0, s>>>(ld, n, tmp, out);
  count_launch(3);
}

template <int MODE>
__global__ void validate_kernel(DevGraph g, uint32_t *deg, unsigned long long *stats) {
  using BR = cub::BlockReduce<unsigned long long, 256>;
  __shared__ typename BR::TempStorage tmp;
  unsigned long long sum = 0, mx = 0, bad = ~0ull;
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < g.n;
       v += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t o0 = g.offsets[v], o1 = g.offsets[v + 1];
    BitCur c;
    c.init(g.words, o0);
    uint32_t d = c.gamma();
    bool ok = true;
    uint64_t end = 0;
    if (MODE == 0) {
      uint32_t hb = c.gamma(), bb = c.gamma(), fp = c.gamma();
      VHdr h = gt_header(g, (uint32_t)v);
      ok = hb >= (d ? 1u : 0u) && hb <= 32 && bb <= 32 && fp <= h.bn + 1 && d < 0x7FFFFFFFu;
      end = ok ? payload_end<0>(g, h) : 0;
    } else {
      if (d == 0) {
        end = c.pos(g.words);
      } else if (d == 1) {
        uint32_t nb = c.gamma();
        ok = nb < g.n;
        end = c.pos(g.words);
      } else {
        uint32_t rb = c.gamma(), sb = c.gamma(), fp = c.gamma();
        VHdr h = le_header(g, (uint32_t)v);
        ok = rb >= 1 && rb <= 32 && sb <= 32 && fp <= h.bn + 2 && d < 0x7FFFFFFFu;
        end = ok ? payload_end<1>(g, h) : 0;
      }
    }
    ok = ok && end == o1;
    if (!ok) bad = min(bad, (unsigned long long)v);
    if (deg) deg[v] = ok ? d : 0;
    if (ok) {
      sum += d;
      mx = max(mx, (unsigned long long)d);
    }
  }
  unsigned long long s = BR(tmp).Sum(sum);
  __syncthreads();
  unsigned long long m = BR(tmp).Reduce(mx, cub::Max());
  __syncthreads();
  unsigned long long b = BR(tmp).Reduce(bad, cub::Min());
  if (threadIdx.x == 0) {
    atomicAdd(&stats[0], s);
    atomicMax(&stats[1], m);
    if (b != ~0ull) atomicMin(&stats[2], b);
  }
}

template <int MODE, class T>
__global__ void degrees_kernel(DevGraph g, T *deg) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < g.n;
       v += (uint64_t)gridDim.x * blockDim.x)
    deg[v] = (T)record_degree(g, (uint32_t)v);
}

// One record per vertex from its stream header (run once, after validation).
template <int MODE>
__global__ void build_records_kernel(DevGraph g, uint4 *recs) {
  for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < g.n;
       v += (uint64_t)gridDim.x * blockDim.x)
    recs[v] = pack_record(stream_header<MODE>(g, (uint32_t)v));
}

// The w (1..33) stream bits at bit `off`, right-aligned (reads two words past
// the field at most: inside the zero guard).
__device__ __forceinline__ uint64_t bits_at(const uint32_t *w, uint64_t off, int width) {
  const uint32_t *q = w + (off >> 5);
  const uint32_t s = (uint32_t)off & 31u;
  const uint32_t x0 = ldw(q), x1 = ldw(q + 1), x2 = ldw(q + 2);
  const uint64_t win = ((uint64_t)__funnelshift_l(x1, x0, s) << 32) | __funnelshift_l(x2, x1, s);
  return win >> (64 - width);
}

// ORs the w (1..33) bits of `val` into the stream at bit `off` (two words at
// most; the caller has cleared them).
__device__ __forceinline__ void or_bits(uint32_t *w, uint64_t off, uint64_t val, int width) {
  const uint32_t s = (uint32_t)off & 31u;  // s + width <= 64
  const uint64_t x = val << (64 - s - width);
  const uint32_t hi = (uint32_t)(x >> 32), lo = (uint32_t)x;
  if (hi) atomicOr(w + (off >> 5), hi);
  if (lo) atomicOr(w + (off >> 5) + 1, lo);
}

// LE payloads in neighbor order (le_chunked, device_common.cuh): one warp per
// vertex.  dst starts as a copy of src; the lanes clear the vertex's payload
// bits [P, end) in dst, then move every field from its on-disk position
// (rock c at P + c a; sea k at P + (chunk_num + 1) a + k (sea_bit + 1),
// LE/src/bcg.cuh:211, 237) to its neighbor-order position.  Words shared with
// another vertex's header or payload are changed with atomicAnd / atomicOr on
// this vertex's bits only; the warp's clears are ordered before its writes by
// __syncwarp.
__global__ void __launch_bounds__(256) le_reorder_kernel(const uint32_t *__restrict__ src,
                                                         uint32_t *dst,
                                                         const uint4 *__restrict__ recs,
                                                         uint32_t n) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const VHdr h = record_header<1>(recs[v], (uint32_t)v);
    if (!le_chunked(h)) continue;  // warp-uniform
    const uint32_t sw = (uint32_t)h.b + 1u;
    const uint64_t end = payload_end<1>(DevGraph{}, h);
    const uint64_t w0 = h.P >> 5, w1 = (end - 1) >> 5;
    for (uint64_t k = w0 + lane; k <= w1; k += 32) {
      uint32_t m = 0xFFFFFFFFu;  // bits of word k inside [P, end), MSB first
      if (k == w0) m &= 0xFFFFFFFFu >> ((uint32_t)h.P & 31u);
      if (k == w1) m &= 0xFFFFFFFFu << (31u - ((uint32_t)(end - 1) & 31u));
      if (m == 0xFFFFFFFFu) dst[k] = 0u;
      else atomicAnd(dst + k, ~m);
    }
    __syncwarp();
    const uint64_t sea0 = h.P + (uint64_t)(h.bn + 1) * (uint64_t)h.a;
    for (uint32_t i = lane; i < h.d; i += 32) {
      uint32_t c, id, tl;
      le_locate(h, i, c, id, tl);
      const uint64_t X = le_chunk_pos(h, c);
      if (id == 0) {
        or_bits(dst, X, bits_at(src, h.P + (uint64_t)c * h.a, h.a), h.a);
      } else {
        const uint64_t k = (uint64_t)(h.bl - 1) * c + min(h.om, c) + id - 1;
        or_bits(dst, X + h.a + (uint64_t)(id - 1) * sw, bits_at(src, sea0 + k * sw, (int)sw),
                (int)sw);
      }
    }
  }
}

// ---- GT stream with skip fields (gt_block_pos, device_common.cuh) ----
// Both kernels take one warp per vertex and one lane per block, reading the
// on-disk stream through each block's cursor: head (a bits), then len - 1
// raw gaps (b bits), GT/chunk_compress/compressor.hpp:297-349.

__device__ __forceinline__ uint32_t bit_len(uint32_t x) { return x ? 32u - __clz(x) : 1u; }

// Pass 1: per vertex the skip-field extra width cx (bits of the largest
// running gap sum at a skip position, beyond b) and the rebuilt payload's
// length in bits.
__global__ void __launch_bounds__(256) gt_skip_measure_kernel(const uint32_t *__restrict__ src,
                                                              const uint4 *__restrict__ recs,
                                                              uint32_t n,
                                                              unsigned char *__restrict__ cx,
                                                              uint64_t *__restrict__ len) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const VHdr h = record_header<0>(recs[v], (uint32_t)v);  // on-disk layout (cx = 0)
    if (h.d == 0) {
      if (lane == 0) cx[v] = 0, len[v] = 0;
      continue;
    }
    const uint32_t longest = h.bl + (h.om ? 1u : 0u);
    uint32_t mx = 0;  // bits of the largest gap sum at a skip position
    if (longest - 1 >= kGtSkip) {
      for (uint32_t blk = lane; blk < h.bn; blk += 32) {
        const uint32_t L = blk < h.om ? h.bl + 1 : h.bl;
        BitCur c;
        c.init(src, gt_block_pos(h, blk) + h.a);
        uint32_t sum = 0;
        for (uint32_t t = 1; t < L; t++) {
          sum += h.b ? c.get(h.b) : 0u;
          if (t % kGtSkip == 0) mx = max(mx, bit_len(sum));
        }
      }
      mx = __reduce_max_sync(0xFFFFFFFFu, mx);
    }
    if (lane == 0) {
      const uint32_t x = mx > (uint32_t)h.b ? mx - (uint32_t)h.b : 0u;
      VHdr hn = h;
      hn.cx = (int)x;
      cx[v] = (unsigned char)x;
      len[v] = payload_end<0>(DevGraph{}, hn) - h.P;
    }
  }
}

// Pass 2: the rebuilt payload of every vertex at its new offset newP[v] in
// dst (zeroed), and its record updated in place (P, and cx above first_pos).
__global__ void __launch_bounds__(256) gt_skip_write_kernel(const uint32_t *__restrict__ src,
                                                            uint32_t *dst, uint4 *recs,
                                                            uint32_t n,
                                                            const unsigned char *__restrict__ cx,
                                                            const uint64_t *__restrict__ newP) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const VHdr h = record_header<0>(recs[v], (uint32_t)v);
    VHdr hn = h;
    hn.P = newP[v];
    hn.cx = cx[v];
    const int sk = hn.b + hn.cx;
    for (uint32_t blk = lane; blk < h.bn; blk += 32) {
      const uint32_t L = blk < h.om ? h.bl + 1 : h.bl;
      BitCur c;
      c.init(src, gt_block_pos(h, blk));
      uint64_t at = gt_block_pos(hn, blk);
      or_bits(dst, at, c.get(h.a), h.a);
      at += h.a;
      uint32_t sum = 0;
      for (uint32_t t = 1; t < L; t++) {
        const uint32_t gap = h.b ? c.get(h.b) : 0u;
        sum += gap;
        if (t % kGtSkip == 0) {
          if (sk) or_bits(dst, at, sum, sk);
          at += sk;
        } else {
          if (h.b) or_bits(dst, at, gap, h.b);
          at += h.b;
        }
      }
    }
    __syncwarp();  // every lane has read the old record
    if (lane == 0) recs[v] = pack_record(hn);
  }
}

unsigned grid_for(uint64_t items, int threads, int device) {
  uint64_t blocks = (items + threads - 1) / threads;
  uint64_t cap = (uint64_t)sm_count(device) * 16;
  return (unsigned)std::max<uint64_t>(1, std::min(blocks, cap));
}

}  // namespace

void launch_bswap(uint32_t *w, uint64_t n_words, cudaStream_t s) {
  if (!n_words) return;
  int dev = 0;
  cudaGetDevice(&dev);
  bswap_kernel<<<grid_for(n_words / 4 + 1, 256, dev), 256, 0, s>>>(w, n_words);
  count_launch();
}

uint64_t scan_tmp_words(uint64_t n) { return (n + kTile - 1) / kTile + 1; }

void launch_unpack_scan(const uint32_t *payload, uint64_t n, uint32_t ubl, uint64_t *out,
                        uint64_t *tmp, cudaStream_t s) {
  scan_impl(FieldLoader{payload, ubl}, n, out, tmp, s);
}

void launch_scan_u32(const uint32_t *counts, uint64_t n, uint64_t *out, uint64_t *tmp,
                     cudaStream_t s) {
  scan_impl(CountLoader{counts}, n, out, tmp, s);
}

void launch_validate(const DevGraph &g, uint32_t *deg, unsigned long long *stats,
                     cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  unsigned grid = grid_for(g.n, 256, dev);
  if (g.mode == GRASS_MODE_GT) validate_kernel<0><<<grid, 256, 0, s>>>(g, deg, stats);
  else validate_kernel<1><<<grid, 256, 0, s>>>(g, deg, stats);
  count_launch();
}

void launch_build_records(const DevGraph &g, uint4 *recs, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  unsigned grid = grid_for(g.n, 256, dev);
  if (g.mode == GRASS_MODE_GT) build_records_kernel<0><<<grid, 256, 0, s>>>(g, recs);
  else build_records_kernel<1><<<grid, 256, 0, s>>>(g, recs);
  count_launch();
}

void launch_le_reorder(const uint32_t *src, uint32_t *dst, const uint4 *recs, uint32_t n,
                       cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  le_reorder_kernel<<<(unsigned)sm_count(dev) * 8, 256, 0, s>>>(src, dst, recs, n);
  count_launch();
}

void launch_gt_skip_measure(const uint32_t *src, const uint4 *recs, uint32_t n,
                            unsigned char *cx, uint64_t *len, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  gt_skip_measure_kernel<<<(unsigned)sm_count(dev) * 8, 256, 0, s>>>(src, recs, n, cx, len);
  count_launch();
}

void launch_gt_skip_write(const uint32_t *src, uint32_t *dst, uint4 *recs, uint32_t n,
                          const unsigned char *cx, const uint64_t *newP, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  gt_skip_write_kernel<<<(unsigned)sm_count(dev) * 8, 256, 0, s>>>(src, dst, recs, n, cx, newP);
  count_launch();
}

void launch_degrees(const DevGraph &g, uint32_t *deg, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  unsigned grid = grid_for(g.n, 256, dev);
  if (g.mode == GRASS_MODE_GT) degrees_kernel<0, uint32_t><<<grid, 256, 0, s>>>(g, deg);
  else degrees_kernel<1, uint32_t><<<grid, 256, 0, s>>>(g, deg);
  count_launch();
}

void launch_degrees64(const DevGraph &g, uint64_t *deg, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  unsigned grid = grid_for(g.n, 256, dev);
  if (g.mode == GRASS_MODE_GT) degrees_kernel<0, uint64_t><<<grid, 256, 0, s>>>(g, deg);
  else degrees_kernel<1, uint64_t><<<grid, 256, 0, s>>>(g, deg);
  count_launch();
}

void launch_scan_u64_inplace(uint64_t *vals, uint64_t n, uint64_t *tmp, cudaStream_t s) {
  scan_impl(U64Loader{vals}, n, vals, tmp, s);
}

}  // namespace grass
