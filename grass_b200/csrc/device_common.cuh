// device_common.cuh -- device-side view of a compressed graph and the GT/LE
// decoders used by every kernel.
//
// Stream words: the .graph file's bytes in big-endian order per 32-bit word
// (GT/src/grass.cu:1147-1159), stored byte-swapped in HBM so that a word read
// is the next 32 stream bits MSB-first.  Two zero guard words follow the last
// word, so a 64-bit window read never leaves the allocation.
#pragma once
#include <stdint.h>

#include "rng.h"

namespace grass {

constexpr uint32_t INVALID_VERTEX = 0xFFFFFFFFu;

struct DevGraph {
  const uint32_t *__restrict__ words;
  const uint64_t *__restrict__ offsets;  // n + 1 bit offsets
  uint32_t n;
  int32_t mode;
};

struct DevCsr {
  const uint64_t *__restrict__ rowptr;
  const uint32_t *__restrict__ cols;
  uint32_t n;
};

__device__ __forceinline__ uint32_t ldw(const uint32_t *p) { return __ldg(p); }

// A field of width w in [1, 32] at bit offset off
// (the reference's get_32b(off) >> (32 - w), GT/src/bcg.cuh:64-70, 90-95).
__device__ __forceinline__ uint32_t read_field(const uint32_t *w, uint64_t off, int width) {
  const uint32_t *q = w + (off >> 5);
  uint32_t win = __funnelshift_l(ldw(q + 1), ldw(q), (uint32_t)off & 31u);
  return width ? win >> (32 - width) : 0u;
}

// Sequential MSB-first reader: the top `nb` bits of `buf` are unread stream
// bits, the rest are zero; one 32-bit word is pulled when nb <= 32.
struct BitCur {
  const uint32_t *p;
  uint64_t buf;
  int nb;
  __device__ __forceinline__ void init(const uint32_t *w, uint64_t off) {
    const uint32_t *q = w + (off >> 5);
    uint32_t s = (uint32_t)off & 31u;
    buf = (((uint64_t)ldw(q) << 32) | ldw(q + 1)) << s;
    nb = 64 - (int)s;
    p = q + 2;
  }
  __device__ __forceinline__ void fill() {
    if (nb <= 32) {
      buf |= (uint64_t)ldw(p) << (32 - nb);
      p++;
      nb += 32;
    }
  }
  // width in [1, 32]
  __device__ __forceinline__ uint32_t get(int width) {
    fill();
    uint32_t v = (uint32_t)(buf >> (64 - width));
    buf <<= width;
    nb -= width;
    return v;
  }
  // Elias-gamma of x+1, returns x (GT/src/bcg.cuh:82-107): zeros z, then
  // z+1 bits.  z is clamped to 31 as the reference's 32-bit window implies;
  // headers are validated once at load, so sampling kernels see z <= 31.
  __device__ __forceinline__ uint32_t gamma() {
    fill();
    int z = min(__clzll(buf), 31);
    buf <<= z;
    nb -= z;
    fill();
    uint32_t v = (uint32_t)(buf >> (63 - z));
    buf <<= (z + 1);
    nb -= z + 1;
    return v - 1u;
  }
  __device__ __forceinline__ uint64_t pos(const uint32_t *w) const {
    return (uint64_t)(p - w) * 32u - (uint64_t)nb;
  }
};

__device__ __forceinline__ uint32_t isqrt_u32(uint32_t x) {
  uint32_t r = (uint32_t)__fsqrt_rn((float)x);
  if ((uint64_t)r * r > x) r--;
  if ((uint64_t)(r + 1) * (r + 1) <= x) r++;
  return r;
}

// Decoded vertex header.  a = GT head_bit / LE rock_bit, b = GT body_bit /
// LE sea_bit; bn/bl/om = GT block_num/block_len/om_num or LE
// chunk_num/chunk_len/om_num (decoder convention, LE/src/bcg.cuh:141-146);
// fp = first_pos, or for LE degree 1 the single neighbor.
struct VHdr {
  uint64_t P;  // bit offset of the payload
  uint32_t v, d, bn, bl, om, fp;
  int a, b;
};

// GT header: BCGVertex ctor, GT/src/bcg.cuh:109-136 (isqrt instead of
// sqrt((float)d); equal for every degree the compressor can emit below 2^24).
__device__ __forceinline__ VHdr gt_header(const DevGraph &g, uint32_t v) {
  VHdr h;
  BitCur c;
  c.init(g.words, g.offsets[v]);
  h.v = v;
  h.d = c.gamma();
  h.a = (int)c.gamma();
  h.b = (int)c.gamma();
  h.fp = c.gamma();
  h.P = c.pos(g.words);
  uint32_t s = isqrt_u32(h.d);
  if (s * s == h.d) {
    h.bn = h.bl = s;
    h.om = 0;
  } else {
    h.bn = s + 1;
    h.bl = h.d / h.bn;
    h.om = h.d - h.bn * h.bl;
  }
  return h;
}

// GT get_vertex, GT/src/bcg.cuh:153-168: locate (block, id), read the head,
// then add id gaps.
__device__ __forceinline__ uint32_t gt_neighbor(const DevGraph &g, const VHdr &h, uint32_t i) {
  const uint32_t split = (h.bl + 1) * h.om;
  const bool flag = i < split;
  const uint32_t j = flag ? i : i - split;
  const uint32_t len = h.bl + (flag ? 1u : 0u);
  uint32_t blk = j / len;
  uint32_t id = j - blk * len;
  if (!flag) blk += h.om;
  const uint64_t pos = h.P + (uint64_t)blk * (uint64_t)(h.a + (h.bl - 1) * h.b) +
                       (uint64_t)min(blk, h.om) * (uint64_t)h.b;
  BitCur c;
  c.init(g.words, pos);
  uint32_t head = c.get(h.a);
  uint32_t cur = (blk >= h.fp) ? h.v + head + 1u : h.v - head - 1u;
  for (uint32_t k = 0; k < id; k++) cur += c.get(h.b) + 1u;
  return cur;
}

// LE header: BCGVertex ctor, LE/src/bcg.cuh:130-152.
__device__ __forceinline__ VHdr le_header(const DevGraph &g, uint32_t v) {
  VHdr h;
  BitCur c;
  c.init(g.words, g.offsets[v]);
  h.v = v;
  h.d = c.gamma();
  h.a = h.b = 0;
  h.bn = h.bl = h.om = h.fp = 0;
  if (h.d == 0) {
    h.P = 0;
    return h;
  }
  uint32_t r = c.gamma();
  if (h.d == 1) {
    h.fp = r;  // degree 1: the field holds the neighbor itself
    h.P = 0;
    return h;
  }
  h.a = (int)r;
  h.b = (int)c.gamma();
  h.fp = c.gamma();
  h.P = c.pos(g.words);
  const uint32_t D = h.d - 1;
  const uint32_t s = isqrt_u32(D);
  const uint32_t om = D - s * s;
  h.bn = s + (om > s ? 1u : 0u);
  h.bl = D / h.bn;
  h.om = D - h.bn * h.bl;
  return h;
}

// LE get_vertex, LE/src/bcg.cuh:195-261: two rocks and one signed sea.
__device__ __forceinline__ uint32_t le_neighbor(const DevGraph &g, const VHdr &h, uint32_t i) {
  if (h.d == 1) return h.fp;
  uint32_t tl = h.bl + 1;
  const uint32_t split = h.om * tl;
  const bool flag = i >= split;
  const uint32_t j = flag ? i - split : i;
  if (flag) tl -= 1;
  uint32_t c = j / tl;
  const uint32_t id = j - c * tl;
  if (flag) c += h.om;
  // The sea's position depends only on the header, so its load is issued
  // together with the rocks' (for id == 0 it re-reads the first sea, which
  // is in bounds and unused).
  const uint64_t spos =
      h.P + (uint64_t)(h.bn + 1) * (uint64_t)h.a +
      ((uint64_t)(h.bl - 1) * c + min(h.om, c) + (id ? id - 1 : 0)) * (uint64_t)(h.b + 1);
  const uint64_t rpos = h.P + (uint64_t)c * (uint64_t)h.a;
  const uint32_t *rq = g.words + (rpos >> 5);
  const uint32_t *sq = g.words + (spos >> 5);
  const uint32_t rw0 = ldw(rq), rw1 = ldw(rq + 1), rw2 = ldw(rq + 2);
  const uint32_t sw0 = ldw(sq), sw1 = ldw(sq + 1);
  // rocks c and c+1: 2*a <= 64 bits starting at bit (rpos & 31) of rw0
  const uint32_t rs = (uint32_t)rpos & 31u;
  const uint64_t rwin = ((((uint64_t)rw0 << 32) | rw1) << rs) | (rs ? ((uint64_t)rw2 << rs) >> 32 : 0);
  const uint32_t r1m = (uint32_t)(rwin >> (64 - h.a));
  const uint32_t r1 = (c < h.fp) ? h.v - r1m : h.v + r1m;
  if (id == 0) return r1;
  const uint32_t r2m = (uint32_t)((rwin << h.a) >> (64 - h.a));
  const uint32_t r2 = (c + 1 < h.fp) ? h.v - r2m : h.v + r2m;
  const uint32_t swin = __funnelshift_l(sw1, sw0, (uint32_t)spos & 31u);
  const uint32_t raw = swin >> (31 - h.b);
  const uint32_t mag = raw >> 1;
  // (r2 - r1) >= 0 for sorted rows: unsigned division is the compressor's.
  return ((r2 - r1) / tl) * id + r1 + ((raw & 1u) ? 0u - mag : mag);
}

template <int MODE>
__device__ __forceinline__ VHdr header(const DevGraph &g, uint32_t v) {
  if constexpr (MODE == 0) return gt_header(g, v);
  else return le_header(g, v);
}

template <int MODE>
__device__ __forceinline__ uint32_t neighbor(const DevGraph &g, const VHdr &h, uint32_t i) {
  if constexpr (MODE == 0) return gt_neighbor(g, h, i);
  else return le_neighbor(g, h, i);
}

// Number of bits a well-formed vertex occupies given its decoded header;
// equals offsets[v+1] - offsets[v] for files written by the reference
// compressor (GT/chunk_compress/compressor.hpp:297-349,
// LE/chunk_compress/compressor.hpp:329-390).
template <int MODE>
__device__ __forceinline__ uint64_t payload_end(const DevGraph &g, const VHdr &h) {
  if constexpr (MODE == 0) {
    return h.P + (uint64_t)h.bn * h.a + (uint64_t)(h.d - h.bn) * h.b;
  } else {
    if (h.d <= 1) return 0;  // caller checks via the header cursor instead
    return h.P + (uint64_t)(h.bn + 1) * h.a + (uint64_t)(h.d - h.bn - 1) * (h.b + 1);
  }
}

// Warp-aggregated add of a per-thread counter into a device u64.
__device__ __forceinline__ void warp_add_u64(unsigned long long *dst, uint64_t v) {
  if (!dst) return;
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, (unsigned long long)v);
}

}  // namespace grass
