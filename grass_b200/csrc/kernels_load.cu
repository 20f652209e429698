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

// ---- LE device layout (sector slots, device_common.cuh) ----

// Neighbor i of an LE vertex in the on-disk layout: rocks at P + c a, seas at
// P + (chunk_num + 1) a + k (sea_bit + 1) (LE/src/bcg.cuh:195-261).
__device__ __forceinline__ uint32_t le_disk_neighbor(const uint32_t *words, const VHdr &h,
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
  const uint64_t rpos = h.P + (uint64_t)c * (uint64_t)h.a;
  const uint32_t r1m = (uint32_t)bits_at(words, rpos, h.a);
  const uint32_t r1 = c < h.fp ? h.v - r1m : h.v + r1m;
  if (id == 0) return r1;
  const uint32_t r2m = (uint32_t)bits_at(words, rpos + h.a, h.a);
  const uint32_t r2 = c + 1 < h.fp ? h.v - r2m : h.v + r2m;
  const uint64_t k = (uint64_t)(h.bl - 1) * c + min(h.om, c) + id - 1;
  const uint64_t raw =
      bits_at(words, h.P + (uint64_t)(h.bn + 1) * (uint64_t)h.a + k * (uint64_t)(h.b + 1), h.b + 1);
  const uint32_t mag = (uint32_t)(raw >> 1);
  return ((r2 - r1) / tl) * id + r1 + ((raw & 1u) ? 0u - mag : mag);
}

// Pass 0: every LE neighbor list, decoded from the on-disk stream into a
// temporary CSR (one warp per vertex).
__global__ void __launch_bounds__(256) le_disk_decode_kernel(const uint32_t *__restrict__ words,
                                                             const uint4 *__restrict__ recs,
                                                             uint32_t n,
                                                             const uint64_t *__restrict__ rowptr,
                                                             uint32_t *__restrict__ cols) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const VHdr h = le_disk_record_header(recs[v], (uint32_t)v);
    uint32_t *out = cols + rowptr[v];
    for (uint32_t i = lane; i < h.d; i += 32) out[i] = le_disk_neighbor(words, h, i);
  }
}

__device__ __forceinline__ uint32_t bit_len64(uint64_t x) { return x ? 64u - __clzll(x) : 1u; }

// Chunk lengths tried per vertex; slots must fit a sector (cb <= 256).
__constant__ uint8_t kChunkLens[] = {1, 2, 3, 4, 5, 6, 7, 8, 10, 12, 14, 16, 20, 24, 28, 32};
constexpr int kNumChunkLens = sizeof(kChunkLens);
constexpr uint32_t kMaxSlots = 63;  // K is stored in 6 bits

// Pass 1: per vertex of degree >= 2, the chunk length T with the fewest
// bits (a vertex of one sector: C cb; larger: whole sectors), its sea_bit
// (largest residual magnitude's bit count, as get_bit_num), K, rock width a
// (bits of max(|n_0 - v|, |n_{d-1} - v|), LE/chunk_compress/compressor.hpp:69)
// and first_pos (rocks below v).  meta[v] = T | sea_bit << 8 | K << 16 | a << 24.
__global__ void __launch_bounds__(256) le_choose_kernel(const uint64_t *__restrict__ rowptr,
                                                        const uint32_t *__restrict__ cols,
                                                        uint32_t n, uint32_t *__restrict__ meta,
                                                        uint32_t *__restrict__ fpos) {
  const int lane = threadIdx.x & 31;
  const unsigned FULLM = 0xFFFFFFFFu;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const uint64_t base = rowptr[v];
    const uint32_t d = (uint32_t)(rowptr[v + 1] - base);
    if (d < 2) {
      if (lane == 0) meta[v] = 0, fpos[v] = 0;
      continue;
    }
    const uint32_t *nb = cols + base;
    const int64_t vv = (int64_t)v;
    const uint32_t a = bit_len64((uint64_t)max(llabs((int64_t)nb[0] - vv),
                                               llabs((int64_t)nb[d - 1] - vv)));
    const uint32_t last = d - 1;
    uint64_t best = ~0ull;
    uint32_t bT = 1, bsb = 0, bK = 1;
    for (int t = 0; t < kNumChunkLens; t++) {
      const uint32_t T = kChunkLens[t];
      if (T > 1 && T >= d) break;  // one chunk already holds every neighbor
      uint32_t sb = 0;
      for (uint32_t i = lane; i < last; i += 32) {
        const uint32_t c = i / T, id = i - c * T;
        if (!id) continue;
        const uint32_t L = min(T, last - c * T);
        const uint32_t r1 = nb[c * T], r2 = nb[c * T + L];
        const int64_t res = (int64_t)nb[i] - ((int64_t)r1 + (int64_t)id * ((r2 - r1) / L));
        sb = max(sb, bit_len64((uint64_t)llabs(res)));
      }
      sb = __reduce_max_sync(FULLM, sb);
      const uint32_t cb = 2 * a + (T - 1) * (sb + 1);
      if (cb > 256) continue;
      const uint32_t K = min(256u / cb, kMaxSlots);
      const uint32_t C = (last - 1) / T + 1;
      const uint64_t cost = C <= K ? (uint64_t)C * cb : (uint64_t)((C + K - 1) / K) * 256u;
      if (cost < best) best = cost, bT = T, bsb = sb, bK = K;
    }
    // first_pos: the rocks (n[cT] for c < C, and n[d-1]) below v
    const uint32_t C = (last - 1) / bT + 1;
    uint32_t below = 0;
    for (uint32_t c = lane; c <= C; c += 32) below += (c < C ? nb[c * bT] : nb[last]) < v;
    below = __reduce_add_sync(FULLM, below);
    if (lane == 0) {
      meta[v] = bT | bsb << 8 | bK << 16 | a << 24;
      fpos[v] = below;
    }
  }
}

// Pass 2: every vertex's slots at its offset P[v] in dst (zeroed), and its
// record rewritten in place in the device format.
__global__ void __launch_bounds__(256) le_write_kernel(const uint64_t *__restrict__ rowptr,
                                                       const uint32_t *__restrict__ cols,
                                                       uint32_t n,
                                                       const uint32_t *__restrict__ meta,
                                                       const uint32_t *__restrict__ fpos,
                                                       const uint64_t *__restrict__ P,
                                                       uint32_t *dst, uint4 *recs) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const uint64_t base = rowptr[v];
    const uint32_t d = (uint32_t)(rowptr[v + 1] - base);
    if (d < 2) {
      if (lane == 0) recs[v] = d ? pack_slot_record(0, 0, 0, 0, 0, 1, cols[base]) : make_uint4(0, 0, 0, 0);
      continue;
    }
    const uint32_t *nb = cols + base;
    const uint32_t m = meta[v];
    const uint32_t T = m & 0xFFu, sb = (m >> 8) & 0xFFu, K = (m >> 16) & 0xFFu, a = m >> 24;
    const uint32_t sw = sb + 1, cb = 2 * a + (T - 1) * sw, last = d - 1, C = (last - 1) / T + 1;
    for (uint32_t c = lane; c < C; c += 32) {
      const uint32_t q = c / K;
      const uint64_t at = P[v] + (uint64_t)q * 256u + (uint64_t)(c - q * K) * cb;
      const uint32_t L = min(T, last - c * T);
      const uint32_t r1 = nb[c * T], r2 = nb[c * T + L];
      or_bits(dst, at, (uint64_t)llabs((int64_t)r1 - (int64_t)v), a);
      const uint32_t step = (r2 - r1) / L;
      for (uint32_t id = 1; id < L; id++) {
        const int64_t res = (int64_t)nb[c * T + id] - ((int64_t)r1 + (int64_t)id * step);
        const uint64_t f = ((uint64_t)llabs(res) << 1) | (res < 0 ? 1u : 0u);
        if (f) or_bits(dst, at + a + (uint64_t)(id - 1) * sw, f, sw);
      }
      or_bits(dst, at + a + (uint64_t)(T - 1) * sw, (uint64_t)llabs((int64_t)r2 - (int64_t)v), a);
    }
    if (lane == 0) recs[v] = pack_slot_record(P[v], a, sb, T, K, d, fpos[v]);
  }
}

// ---- GT device layout (sector slots, device_common.cuh) ----

// Pass 0: every GT neighbor list, decoded from the on-disk stream into a
// temporary CSR: one warp per vertex, one lane per block, each block's head
// and gaps read in order (GT/src/bcg.cuh:153-168).
__global__ void __launch_bounds__(256) gt_disk_decode_kernel(const uint32_t *__restrict__ words,
                                                             const uint4 *__restrict__ recs,
                                                             uint32_t n,
                                                             const uint64_t *__restrict__ rowptr,
                                                             uint32_t *__restrict__ cols) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const VHdr h = gt_disk_record_header(recs[v], (uint32_t)v);
    uint32_t *out = cols + rowptr[v];
    for (uint32_t blk = lane; blk < h.bn; blk += 32) {
      const uint32_t L = blk < h.om ? h.bl + 1 : h.bl;
      const uint32_t i0 = blk * h.bl + min(blk, h.om);
      BitCur c;
      c.init(words, gt_disk_block_pos(h, blk));
      const uint32_t hv = c.get(h.a) + 1u;
      uint32_t x = blk >= h.fp ? h.v + hv : h.v - hv;
      out[i0] = x;
      for (uint32_t t = 1; t < L; t++) {
        x += (h.b ? c.get(h.b) : 0u) + 1u;
        out[i0 + t] = x;
      }
    }
  }
}

// Pass 1: per vertex of degree >= 1, the chunk length T with the fewest bits
// (as for LE), the head width a (bits of the largest |n_cT - v| - 1), the gap
// width b (bits of the largest n_i - n_{i-1} - 1 inside a chunk; 0 without
// gaps), K, and first_pos (chunks whose head lies below v).
// meta[v] = T | b << 8 | K << 16 | a << 24.
__global__ void __launch_bounds__(256) gt_choose_kernel(const uint64_t *__restrict__ rowptr,
                                                        const uint32_t *__restrict__ cols,
                                                        uint32_t n, uint32_t *__restrict__ meta,
                                                        uint32_t *__restrict__ fpos) {
  const int lane = threadIdx.x & 31;
  const unsigned FULLM = 0xFFFFFFFFu;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const uint64_t base = rowptr[v];
    const uint32_t d = (uint32_t)(rowptr[v + 1] - base);
    if (d == 0) {
      if (lane == 0) meta[v] = 0, fpos[v] = 0;
      continue;
    }
    const uint32_t *nb = cols + base;
    const int64_t vv = (int64_t)v;
    uint64_t best = ~0ull;
    uint32_t bT = 1, bb = 0, bK = 1, ba = 1;
    for (int t = 0; t < kNumChunkLens; t++) {
      const uint32_t T = kChunkLens[t];
      if (T > 1 && T > d) break;  // one chunk already holds every neighbor
      uint32_t a = 1, b = 0;
      for (uint32_t i = lane; i < d; i += 32) {
        if (i % T == 0) {
          a = max(a, bit_len64((uint64_t)(llabs((int64_t)nb[i] - vv) - 1)));
        } else {
          b = max(b, bit_len64((uint64_t)(nb[i] - nb[i - 1] - 1)));
        }
      }
      a = __reduce_max_sync(FULLM, a);
      b = __reduce_max_sync(FULLM, b);
      const uint32_t cb = a + (T - 1) * b;
      if (cb > 256) continue;
      const uint32_t K = min(256u / cb, kMaxSlots);
      const uint32_t C = (d - 1) / T + 1;
      const uint64_t cost = C <= K ? (uint64_t)C * cb : (uint64_t)((C + K - 1) / K) * 256u;
      if (cost < best) best = cost, bT = T, bb = b, bK = K, ba = a;
    }
    const uint32_t C = (d - 1) / bT + 1;
    uint32_t below = 0;
    for (uint32_t c = lane; c < C; c += 32) below += nb[c * bT] < v;
    below = __reduce_add_sync(FULLM, below);
    if (lane == 0) {
      meta[v] = bT | bb << 8 | bK << 16 | ba << 24;
      fpos[v] = below;
    }
  }
}

// Pass 2: every vertex's slots at its offset P[v] in dst (zeroed), and its
// record rewritten in place in the device format.
__global__ void __launch_bounds__(256) gt_write_kernel(const uint64_t *__restrict__ rowptr,
                                                       const uint32_t *__restrict__ cols,
                                                       uint32_t n,
                                                       const uint32_t *__restrict__ meta,
                                                       const uint32_t *__restrict__ fpos,
                                                       const uint64_t *__restrict__ P,
                                                       uint32_t *dst, uint4 *recs) {
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  for (uint64_t v = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; v < n; v += nwarps) {
    const uint64_t base = rowptr[v];
    const uint32_t d = (uint32_t)(rowptr[v + 1] - base);
    if (d == 0) {
      if (lane == 0) recs[v] = make_uint4(0, 0, 0, 0);
      continue;
    }
    const uint32_t *nb = cols + base;
    const uint32_t m = meta[v];
    const uint32_t T = m & 0xFFu, b = (m >> 8) & 0xFFu, K = (m >> 16) & 0xFFu, a = m >> 24;
    const uint32_t cb = a + (T - 1) * b, C = (d - 1) / T + 1;
    for (uint32_t c = lane; c < C; c += 32) {
      const uint32_t q = c / K;
      uint64_t at = P[v] + (uint64_t)q * 256u + (uint64_t)(c - q * K) * cb;
      const uint32_t i0 = c * T, L = min(T, d - i0);
      const uint64_t head = (uint64_t)(llabs((int64_t)nb[i0] - (int64_t)v) - 1);
      if (head) or_bits(dst, at, head, a);
      at += a;
      for (uint32_t t = 1; t < L; t++, at += b) {
        const uint32_t gap = nb[i0 + t] - nb[i0 + t - 1] - 1;
        if (gap) or_bits(dst, at, gap, b);
      }
    }
    if (lane == 0) recs[v] = pack_slot_record(P[v], a, b, T, K, d, fpos[v]);
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

void launch_disk_decode(int mode, const uint32_t *words, const uint4 *recs, uint32_t n,
                        const uint64_t *rowptr, uint32_t *cols, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned grid = (unsigned)sm_count(dev) * 8;
  if (mode == GRASS_MODE_GT) gt_disk_decode_kernel<<<grid, 256, 0, s>>>(words, recs, n, rowptr, cols);
  else le_disk_decode_kernel<<<grid, 256, 0, s>>>(words, recs, n, rowptr, cols);
  count_launch();
}

void launch_slot_choose(int mode, const uint64_t *rowptr, const uint32_t *cols, uint32_t n,
                        uint32_t *meta, uint32_t *fpos, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned grid = (unsigned)sm_count(dev) * 8;
  if (mode == GRASS_MODE_GT) gt_choose_kernel<<<grid, 256, 0, s>>>(rowptr, cols, n, meta, fpos);
  else le_choose_kernel<<<grid, 256, 0, s>>>(rowptr, cols, n, meta, fpos);
  count_launch();
}

void launch_slot_write(int mode, const uint64_t *rowptr, const uint32_t *cols, uint32_t n,
                       const uint32_t *meta, const uint32_t *fpos, const uint64_t *P,
                       uint32_t *dst, uint4 *recs, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  const unsigned grid = (unsigned)sm_count(dev) * 8;
  if (mode == GRASS_MODE_GT)
    gt_write_kernel<<<grid, 256, 0, s>>>(rowptr, cols, n, meta, fpos, P, dst, recs);
  else
    le_write_kernel<<<grid, 256, 0, s>>>(rowptr, cols, n, meta, fpos, P, dst, recs);
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
