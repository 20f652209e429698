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

// Vertex record: the decoded gamma header of one vertex, 16 bytes, built once
// at load from the .offset lengths and the stream headers.  Samplers read
// one aligned record (one 32-byte sector, L2-resident for graphs of tens of
// millions of vertices) instead of an 8-byte bit offset followed by a
// dependent header read from the stream.
//   x = payload bit offset P, low 32 bits
//   y = P bits 32..47 | a << 16 (6 bits) | b << 22 (6 bits)
//   z = degree d
//   w = first_pos, or for LE degree 1 the single neighbor
// A graph as the samplers see it: compressed (mode 0 GT, 1 LE: words and
// records) or an uncompressed CSR (mode 2, GRASS_MODE_CSR_INTERNAL: rowptr and
// cols), so that one sampler template serves both sides of a comparison.
struct DevGraph {
  const uint32_t *__restrict__ words;
  const uint4 *__restrict__ recs;        // n vertex records (sampling, decode)
  const uint64_t *__restrict__ offsets;  // n + 1 bit offsets (load time only)
  uint32_t n;
  int32_t mode;
  const uint64_t *__restrict__ rowptr;   // mode 2
  const uint32_t *__restrict__ cols;     // mode 2
};
constexpr int GRASS_MODE_CSR_INTERNAL = 2;

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

// One 32-byte sector of the stream as four 64-bit words in stream order (the
// first word holds stream bits 0..63 of the sector, MSB first).  A single
// 256-bit load is one L2 request; separate 32-bit loads of the same sector
// issued back to back each miss L1 and become separate L2 requests.
struct Sec {
  uint64_t q0, q1, q2, q3;
};

__device__ __forceinline__ uint64_t swap_halves(uint64_t x) { return (x << 32) | (x >> 32); }

// L2 eviction priorities.  Every draw reads one entry of a small hot table
// (vertex records, or the CSR's row pointers: tens of MB, i.e. L2-sized)
// and one or two random sectors of a large cold array (the stream, or CSR
// columns: far larger than L2).  Without hints the cold reads evict the hot
// table between its uses and every draw pays a DRAM access for it.
//   hot table  -> evict_last
//   cold reads -> GRASS_COLD_POLICY (0: normal, 1: evict_first)
//   path/frontier stores -> GRASS_ST_POLICY (0: normal, 1: evict_first)
#ifndef GRASS_HOT_POLICY
#define GRASS_HOT_POLICY 1
#endif
#ifndef GRASS_COLD_POLICY
#define GRASS_COLD_POLICY 0
#endif
#ifndef GRASS_ST_POLICY
#define GRASS_ST_POLICY 1
#endif

__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// The loads below are inline PTX, marked volatile: a non-volatile asm
// statement counts as a pure function of its inputs, so the compiler may
// execute it speculatively -- hoisted above the branch that guards its
// address (a record load for an invalid vertex id, say) -- and fault.
__device__ __forceinline__ uint4 load_record(const uint4 *p) {
  uint4 r;
#if GRASS_HOT_POLICY
  asm volatile("ld.global.nc.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p), "l"(policy_evict_last()));
#else
  asm volatile("ld.global.nc.v4.u32 {%0,%1,%2,%3}, [%4];"
      : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
      : "l"(p));
#endif
  return r;
}

// A 4-byte cold read (CSR column).
__device__ __forceinline__ uint32_t load_cold_u32(const uint32_t *p) {
#if GRASS_COLD_POLICY
  uint32_t v;
  asm volatile("ld.global.nc.L2::cache_hint.u32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(policy_evict_first()));
  return v;
#else
  return __ldg(p);
#endif
}

// Store of an output entry that is not read again by the kernel.
__device__ __forceinline__ void store_out_u32(uint32_t *p, uint32_t v) {
#if GRASS_ST_POLICY
  asm volatile("st.global.L2::cache_hint.u32 [%0], %1, %2;" ::"l"(p), "r"(v),
               "l"(policy_evict_first())
               : "memory");
#else
  *p = v;
#endif
}

__device__ __forceinline__ Sec load_sector(const uint32_t *words, uint64_t sector) {
  const uint64_t *p = reinterpret_cast<const uint64_t *>(words) + sector * 4;
  uint64_t a0, a1, a2, a3;
#if GRASS_COLD_POLICY
  asm volatile("ld.global.nc.L2::evict_first.v4.b64 {%0,%1,%2,%3}, [%4];"
      : "=l"(a0), "=l"(a1), "=l"(a2), "=l"(a3)
      : "l"(p));
#else
  asm volatile("ld.global.nc.v4.b64 {%0,%1,%2,%3}, [%4];"
      : "=l"(a0), "=l"(a1), "=l"(a2), "=l"(a3)
      : "l"(p));
#endif
  // little-endian u64 = (word 2i+1 << 32) | word 2i; stream order wants word 2i high
  return Sec{swap_halves(a0), swap_halves(a1), swap_halves(a2), swap_halves(a3)};
}

__device__ __forceinline__ uint64_t sec_word(const Sec &s, uint32_t k) {
  return k == 0 ? s.q0 : k == 1 ? s.q1 : k == 2 ? s.q2 : s.q3;
}

// The 64 stream bits starting at bit `off` (0..255) of sector a, continuing
// into sector b when they cross its end.
__device__ __forceinline__ uint64_t sec_window(const Sec &a, const Sec &b, uint32_t off) {
  const uint32_t k = off >> 6, s = off & 63u;
  const uint64_t x = sec_word(a, k);
  const uint64_t y = k == 3 ? b.q0 : sec_word(a, k + 1);
  return s ? (x << s) | (y >> (64 - s)) : x;
}

// Word k (0..7) of the 512 stream bits held by sectors A and B; 0 beyond.
__device__ __forceinline__ uint64_t sec2_word(const Sec &A, const Sec &B, uint32_t k) {
  const uint32_t q = k & 3u;
  const uint64_t x = k < 4 ? sec_word(A, q) : sec_word(B, q);
  return k < 8 ? x : 0ull;
}

// The w (1..33) stream bits at bit `off` (< 512) of sectors A:B, right-aligned.
__device__ __forceinline__ uint64_t sec2_field(const Sec &A, const Sec &B, uint32_t off, int w) {
  const uint32_t k = off >> 6, s = off & 63u;
  const uint64_t x = sec2_word(A, B, k);
  const uint64_t win = s ? (x << s) | (sec2_word(A, B, k + 1) >> (64 - s)) : x;
  return win >> (64 - w);
}

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
  int cx;      // GT: extra width of a skip field over a gap field (device layout)
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
  h.cx = 0;
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

// ---- sector slots: the device layout of both formats ----
// On disk a vertex is ~sqrt(d) blocks (GT) or chunks (LE) of ~sqrt(d)
// neighbors, so a random draw in a hub touches several 32-byte sectors: GT
// adds up to sqrt(d) gaps (GT/src/bcg.cuh:153-168), LE reads its rock pair
// and its sea from two places (LE/src/bcg.cuh:195-261).  At load every
// vertex is re-chunked for the device with its format's own method but a
// chunk length T (1..32) of its own, each chunk in a self-contained slot that
// never crosses a sector:
//   slot c of cb bits starts at P + (c / K) 256 + (c % K) cb, K <= 63 slots
//   per sector; a vertex whose slots fit in one sector is packed without
//   alignment (and lies inside one sector), a larger one starts on a sector.
// A draw reads its record and one sector.  T is chosen per vertex for the
// fewest bits.  Decoded neighbors are the file's, bit for bit.
//
// Record (16 B): x = P low 32 bits; y = P bits 32..39 | a << 8 | b << 14 |
// T << 20 | K << 26; z = degree; w = first_pos (LE degree 1: the neighbor).
// In VHdr: bl = T, om = K, bn = C (number of slots), cx = cb.

__device__ __forceinline__ uint4 pack_slot_record(uint64_t P, uint32_t a, uint32_t b, uint32_t T,
                                                  uint32_t K, uint32_t d, uint32_t fp) {
  return make_uint4((uint32_t)P,
                    ((uint32_t)(P >> 32) & 0xFFu) | (a & 63u) << 8 | (b & 63u) << 14 |
                        (T & 63u) << 20 | (K & 63u) << 26,
                    d, fp);
}

// Exact x / d for x < 2^32 and 2 <= d < 2^32 by one 64-bit multiply-high.
// M = floor((2^64 - 1) / d) + 1 = 2^64 / d + e with 0 <= e < 1, so
// x M / 2^64 = x / d + x e / 2^64, and x e / 2^64 < 2^-32 < 1 / d never
// carries the quotient past the next integer.  d = 1 passes x through.
__host__ __device__ __forceinline__ uint64_t div_magic(uint32_t d) {
  return d >= 2 ? ~0ull / d + 1 : 0ull;
}
__device__ __forceinline__ uint32_t div_by(uint32_t x, uint32_t d, uint64_t M) {
  return d >= 2 ? (uint32_t)__umul64hi((uint64_t)x, M) : x;
}

// div_magic(d) for the small divisors of the slot layout (chunk length T,
// slots per sector K, chunk length L: all below 64), read through L1.
struct DivMagic64 {
  uint64_t m[64];
};
__host__ __device__ constexpr DivMagic64 make_div_magic64() {
  DivMagic64 t{};
  for (uint32_t d = 2; d < 64; d++) t.m[d] = ~0ull / d + 1;
  return t;
}
__device__ const DivMagic64 kDivMagic64 = make_div_magic64();
__device__ __forceinline__ uint32_t div_small(uint32_t x, uint32_t d) {  // d in [1, 63]
  return div_by(x, d, __ldg(&kDivMagic64.m[d & 63u]));
}

// Bit offset of slot c.
__device__ __forceinline__ uint64_t slot_pos(const VHdr &h, uint32_t c) {
  const uint32_t q = div_small(c, h.om);
  return h.P + (uint64_t)q * 256u + (uint64_t)(c - q * h.om) * (uint32_t)h.cx;
}

// The w (1..33) bits at bit off of one sector, the field inside it.
__device__ __forceinline__ uint64_t sec1_field(const Sec &A, uint32_t off, int w) {
  const uint32_t k = off >> 6, s = off & 63u;
  const uint64_t x = sec_word(A, k);
  const uint64_t y = k < 3 ? sec_word(A, k + 1) : 0ull;
  const uint64_t win = s ? (x << s) | (y >> (64 - s)) : x;
  return win >> (64 - w);
}

// Sum of n w-bit fields from bit off of one sector (off + n w <= 256): a
// 128-bit shift window pulls the next word when needed.
__device__ __forceinline__ uint32_t sec1_sum(const Sec &A, uint32_t off, uint32_t n, int w) {
  if (!n || !w) return 0;
  uint32_t k = off >> 6;
  const uint32_t sh = off & 63u;
  uint64_t buf = sec_word(A, k) << sh;
  int nb = 64 - (int)sh;
  uint64_t nxt = k < 3 ? sec_word(A, ++k) : 0ull;
  uint32_t s = 0;
  for (uint32_t j = 0; j < n; j++) {
    uint32_t v;
    if (nb >= w) {
      v = (uint32_t)(buf >> (64 - w));
      buf <<= w;
      nb -= w;
    } else {
      const int r = w - nb;  // bits taken from nxt, 1..32
      v = (uint32_t)(((nb ? buf >> (64 - nb) : 0ull) << r) | (nxt >> (64 - r)));
      buf = nxt << r;
      nb = 64 - r;
      nxt = k < 3 ? sec_word(A, ++k) : 0ull;
    }
    s += v;
  }
  return s;
}

// ---- GT ----
// Slot c: the head |n_cT - v| - 1 (a bits), then the gaps n_i - n_{i-1} - 1
// (b bits) of neighbors cT+1 .. cT+L-1, L = min(T, d - cT); the head counts
// up from v when c >= first_pos (the reference's encoding per block,
// GT/chunk_compress/compressor.hpp:245-282, on chunks of T).

// On-disk block geometry, load time only: block blk starts at
// P + blk (a + (bl - 1) b) + min(blk, om) b (GT/src/bcg.cuh:153-163).
__device__ __forceinline__ uint64_t gt_disk_block_pos(const VHdr &h, uint32_t blk) {
  return h.P + (uint64_t)blk * ((uint64_t)h.a + (uint64_t)(h.bl - 1) * h.b) +
         (uint64_t)min(blk, h.om) * h.b;
}

// GT get_vertex on the device layout: one sector; neighbor id of slot c is
// the head value + id + the sum of its id gaps.
__device__ __forceinline__ uint32_t gt_neighbor(const DevGraph &g, const VHdr &h, uint32_t i) {
  const uint32_t c = div_small(i, h.bl), id = i - c * h.bl;
  const uint64_t pos = slot_pos(h, c);
  const Sec A = load_sector(g.words, pos >> 8);
  const uint32_t off = (uint32_t)pos & 255u;
  const uint32_t hv = (uint32_t)sec1_field(A, off, h.a) + 1u;
  return (c >= h.fp ? h.v + hv : h.v - hv) + id + sec1_sum(A, off + (uint32_t)h.a, id, h.b);
}

// Every neighbor of slot c (at bit off of sector A) into o[0..L-1].
__device__ __forceinline__ void gt_slot_decode(const Sec &A, uint32_t off, const VHdr &h,
                                               uint32_t c, uint32_t L, uint32_t *o) {
  const uint32_t hv = (uint32_t)sec1_field(A, off, h.a) + 1u;
  uint32_t x = c >= h.fp ? h.v + hv : h.v - hv;
  o[0] = x;
  uint32_t p = off + (uint32_t)h.a;
  for (uint32_t t = 1; t < L; t++, p += (uint32_t)h.b) {
    x += (h.b ? (uint32_t)sec1_field(A, p, h.b) : 0u) + 1u;
    o[t] = x;
  }
}

// On-disk geometry of an LE vertex of degree d >= 2: chunk_num, chunk_len, om
// (decoder convention, LE/src/bcg.cuh:141-146).
__device__ __forceinline__ void le_disk_geometry(uint32_t d, uint32_t &bn, uint32_t &bl,
                                                 uint32_t &om) {
  const uint32_t D = d - 1;
  const uint32_t s = isqrt_u32(D);
  const uint32_t o = D - s * s;
  bn = s + (o > s ? 1u : 0u);
  bl = D / bn;
  om = D - bn * bl;
}

// LE header: BCGVertex ctor, LE/src/bcg.cuh:130-152.
__device__ __forceinline__ VHdr le_header(const DevGraph &g, uint32_t v) {
  VHdr h;
  BitCur c;
  c.init(g.words, g.offsets[v]);
  h.v = v;
  h.d = c.gamma();
  h.a = h.b = h.cx = 0;
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
  le_disk_geometry(h.d, h.bn, h.bl, h.om);
  return h;
}

// ---- LE ----
// Slot c (the sector slots above): [rock c (a bits)][seas id = 1..T-1 (sea_bit
// + 1 bits each)][rock c+1 (a bits)]; chunk c holds neighbors cT .. cT+L-1, L
// = min(T, d - 1 - cT), and the last neighbor d - 1 is the right rock of slot
// C - 1, C = ceil((d-1)/T).  A chunk is the reference's: a left rock |n - v|,
// signed seas n - (r1 + id ((r2 - r1) / L)), a right rock, rocks signed by
// first_pos (LE/chunk_compress/compressor.hpp:288-359), on chunks of T; the
// rocks of inner chunk boundaries are stored twice.  In VHdr b = sea_bit.

// Chunk c and index id of neighbor i (id == L: the last neighbor, chunk C-1's
// right rock), and the chunk's length L.
__device__ __forceinline__ void le_locate(const VHdr &h, uint32_t i, uint32_t &c, uint32_t &id,
                                          uint32_t &L) {
  const uint32_t last = h.d - 1;
  c = i < last ? div_small(i, h.bl) : h.bn - 1;
  id = i - c * h.bl;
  L = min(h.bl, last - c * h.bl);
}

// Neighbor id of a chunk slot held in sector A at bit offset off: the left
// rock (id 0), the right rock (id == L), or r1 + ((r2 - r1) / L) id +/- sea
// (LE/src/bcg.cuh:195-261; with sea_bit = 32 the 33-bit field keeps its
// whole magnitude, as LE/src/bcg.cuh:245-252 reads it).
__device__ __forceinline__ uint32_t le_slot_value(const Sec &A, uint32_t off, const VHdr &h,
                                                  uint32_t c, uint32_t id, uint32_t L) {
  const int sw = h.b + 1;
  const uint32_t r1m = (uint32_t)sec1_field(A, off, h.a);
  const uint32_t r1 = c < h.fp ? h.v - r1m : h.v + r1m;
  if (id == 0) return r1;
  const uint32_t r2m = (uint32_t)sec1_field(A, off + (uint32_t)h.a + (h.bl - 1) * (uint32_t)sw, h.a);
  const uint32_t r2 = c + 1 < h.fp ? h.v - r2m : h.v + r2m;
  if (id == L) return r2;
  const uint64_t raw = sec1_field(A, off + (uint32_t)h.a + (id - 1) * (uint32_t)sw, sw);
  const uint32_t mag = (uint32_t)(raw >> 1);
  // (r2 - r1) >= 0 for sorted rows: unsigned division is the compressor's.
  return div_small(r2 - r1, L) * id + r1 + ((raw & 1u) ? 0u - mag : mag);
}

// Every neighbor of chunk c, its slot at bit off of sector A, into o[0..L-1]
// (and o[L], the right rock, for the last chunk): the rocks and the step once,
// then the seas in order.
__device__ __forceinline__ void le_slot_decode(const Sec &A, uint32_t off, const VHdr &h,
                                               uint32_t c, uint32_t L, bool with_right,
                                               uint32_t *o) {
  const int sw = h.b + 1;
  const uint32_t r1m = (uint32_t)sec1_field(A, off, h.a);
  const uint32_t r1 = c < h.fp ? h.v - r1m : h.v + r1m;
  const uint32_t s0 = off + (uint32_t)h.a;
  const uint32_t r2m = (uint32_t)sec1_field(A, s0 + (h.bl - 1) * (uint32_t)sw, h.a);
  const uint32_t r2 = c + 1 < h.fp ? h.v - r2m : h.v + r2m;
  const uint32_t step = div_small(r2 - r1, L);
  o[0] = r1;
  for (uint32_t id = 1; id < L; id++) {
    const uint64_t raw = sec1_field(A, s0 + (id - 1) * (uint32_t)sw, sw);
    const uint32_t mag = (uint32_t)(raw >> 1);
    o[id] = step * id + r1 + ((raw & 1u) ? 0u - mag : mag);
  }
  if (with_right) o[L] = r2;
}

// ---- slot decoders on 32-bit words (shared or global memory) ----
// w points at the slot's sector as stream words (each the next 32 bits MSB
// first), with one more readable word after it; off is the bit offset of the
// slot in it.  One funnel shift per field of up to 32 bits.
__device__ __forceinline__ uint32_t word_field(const uint32_t *w, uint32_t off, int width) {
  const uint32_t q = off >> 5, s = off & 31u;
  const uint32_t x = __funnelshift_l(w[q + 1], w[q], s);
  return width ? x >> (32 - width) : 0u;
}

// An LE sea (width sw = sea_bit + 1 <= 33) added to its interpolated base.
__device__ __forceinline__ uint32_t word_sea(const uint32_t *w, uint32_t off, int sw,
                                             uint32_t base) {
  uint32_t mag, neg;
  if (sw > 32) {  // sea_bit 32: the magnitude is the field's top 32 bits
    mag = word_field(w, off, 32);
    neg = word_field(w, off + 32, 1);
  } else {
    const uint32_t raw = word_field(w, off, sw);
    mag = raw >> 1;
    neg = raw & 1u;
  }
  return base + (neg ? 0u - mag : mag);
}

// le_slot_decode / gt_slot_decode on words.
// Fields of up to 32 bits read in order from words: a two-word window, one
// funnel shift per field, the next word loaded one ahead.  Reads up to three
// words past the last field's word.
struct WordStream {
  const uint32_t *w;
  uint32_t q, pos, lo, hi, nx;
  __device__ __forceinline__ void init(const uint32_t *words, uint32_t at) {
    w = words;
    q = at >> 5;
    pos = at & 31u;
    lo = w[q];
    hi = w[q + 1];
    nx = w[q + 2];
  }
  __device__ __forceinline__ uint32_t get(int width) {  // width 0..32
    const uint32_t x = __funnelshift_l(hi, lo, pos);
    pos += (uint32_t)width;
    if (pos >= 32) {
      pos -= 32;
      lo = hi;
      hi = nx;
      nx = w[q + 3];
      q++;
    }
    return width ? x >> (32 - width) : 0u;
  }
};

__device__ __forceinline__ void le_slot_decode_w(const uint32_t *w, uint32_t off, const VHdr &h,
                                                 uint32_t c, uint32_t L, bool with_right,
                                                 uint32_t *o) {
  const int sw = h.b + 1;
  const uint32_t s0 = off + (uint32_t)h.a;
  const uint32_t r2m = word_field(w, s0 + (h.bl - 1) * (uint32_t)sw, h.a);
  const uint32_t r2 = c + 1 < h.fp ? h.v - r2m : h.v + r2m;
  WordStream S;
  S.init(w, off);
  const uint32_t r1m = S.get(h.a);
  const uint32_t r1 = c < h.fp ? h.v - r1m : h.v + r1m;
  const uint32_t step = div_small(r2 - r1, L);
  o[0] = r1;
  uint32_t base = r1;
  for (uint32_t id = 1; id < L; id++) {
    base += step;
    uint32_t mag, neg;
    if (sw > 32) {  // sea_bit 32: the magnitude is the field's top 32 bits
      mag = S.get(32);
      neg = S.get(1);
    } else {
      const uint32_t raw = S.get(sw);
      mag = raw >> 1;
      neg = raw & 1u;
    }
    o[id] = base + (neg ? 0u - mag : mag);
  }
  if (with_right) o[L] = r2;
}

__device__ __forceinline__ void gt_slot_decode_w(const uint32_t *w, uint32_t off, const VHdr &h,
                                                 uint32_t c, uint32_t L, uint32_t *o) {
  WordStream S;
  S.init(w, off);
  const uint32_t hv = S.get(h.a) + 1u;
  uint32_t x = c >= h.fp ? h.v + hv : h.v - hv;
  o[0] = x;
  for (uint32_t t = 1; t < L; t++) {
    x += S.get(h.b) + 1u;
    o[t] = x;
  }
}

// LE get_vertex: one sector load.
__device__ __forceinline__ uint32_t le_neighbor(const DevGraph &g, const VHdr &h, uint32_t i) {
  if (h.d == 1) return h.fp;
  uint32_t c, id, L;
  le_locate(h, i, c, id, L);
  const uint64_t pos = slot_pos(h, c);
  const Sec A = load_sector(g.words, pos >> 8);
  return le_slot_value(A, (uint32_t)pos & 255u, h, c, id, L);
}

// Stream headers (gamma decode at offsets[v]); used at load time only.
template <int MODE>
__device__ __forceinline__ VHdr stream_header(const DevGraph &g, uint32_t v) {
  if constexpr (MODE == 0) return gt_header(g, v);
  else return le_header(g, v);
}

__device__ __forceinline__ uint4 pack_record(const VHdr &h) {
  uint4 r;
  r.x = (uint32_t)h.P;
  r.y = ((uint32_t)(h.P >> 32) & 0xFFFFu) | ((uint32_t)h.a & 63u) << 16 |
        ((uint32_t)h.b & 63u) << 22;
  r.z = h.d;
  r.w = h.fp;
  return r;
}

// Header from a vertex record: the same fields gt_header/le_header decode,
// with the block/chunk geometry recomputed from the degree.
template <int MODE>
__device__ __forceinline__ VHdr record_header(const uint4 r, uint32_t v) {
  VHdr h;
  h.v = v;
  h.P = (uint64_t)r.x | ((uint64_t)(r.y & 0xFFFFu) << 32);
  h.a = (int)((r.y >> 16) & 63u);
  h.b = (int)((r.y >> 22) & 63u);
  h.d = r.z;
  h.fp = r.w;
  h.cx = 0;
  h.bn = h.bl = h.om = 0;  // (CSR, mode 2: no chunk geometry)
  if constexpr (MODE == 0 || MODE == 1) {  // the device layouts (slot_pos)
    h.P = (uint64_t)r.x | ((uint64_t)(r.y & 0xFFu) << 32);
    h.a = (int)((r.y >> 8) & 63u);
    h.b = (int)((r.y >> 14) & 63u);
    h.bl = (r.y >> 20) & 63u;  // T
    h.om = (r.y >> 26) & 63u;  // K
    if constexpr (MODE == 0) {
      if (h.d) {
        h.bn = div_small(h.d - 1, h.bl) + 1;  // C = ceil(d / T)
        h.cx = h.a + (int)(h.bl - 1) * h.b;
      }
    } else if (h.d > 1) {
      h.bn = div_small(h.d - 2, h.bl) + 1;  // C = ceil((d - 1) / T)
      h.cx = 2 * h.a + (int)(h.bl - 1) * (h.b + 1);
    }
  }
  return h;
}

// Header of a GT vertex from its load-time record (pack_record of the stream
// header: on-disk block geometry), before the device layout is built.
__device__ __forceinline__ VHdr gt_disk_record_header(const uint4 r, uint32_t v) {
  VHdr h;
  h.v = v;
  h.P = (uint64_t)r.x | ((uint64_t)(r.y & 0xFFFFu) << 32);
  h.a = (int)((r.y >> 16) & 63u);
  h.b = (int)((r.y >> 22) & 63u);
  h.d = r.z;
  h.fp = r.w;
  h.cx = 0;
  const uint32_t s = isqrt_u32(h.d);
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

// Header of an LE vertex from its load-time record (pack_record of the stream
// header: on-disk geometry), before the device layout is built.
__device__ __forceinline__ VHdr le_disk_record_header(const uint4 r, uint32_t v) {
  VHdr h;
  h.v = v;
  h.P = (uint64_t)r.x | ((uint64_t)(r.y & 0xFFFFu) << 32);
  h.a = (int)((r.y >> 16) & 63u);
  h.b = (int)((r.y >> 22) & 63u);
  h.d = r.z;
  h.fp = r.w;
  h.cx = 0;
  h.bn = h.bl = h.om = 0;
  if (h.d > 1) le_disk_geometry(h.d, h.bn, h.bl, h.om);
  return h;
}

// [rowptr[v], rowptr[v+1]) of a CSR with one 32-byte load (two when the pair
// straddles a sector, v % 4 == 3).  rowptr must be allocated in whole
// sectors with one spare sector (see grass_csr allocation).
__device__ __forceinline__ void csr_row(const uint64_t *rowptr, uint32_t v, uint64_t &b,
                                        uint64_t &e) {
  const uint64_t *p = rowptr + (v & ~3u);
  uint64_t a0, a1, a2, a3;
#if GRASS_HOT_POLICY
  asm volatile("ld.global.nc.L2::evict_last.v4.b64 {%0,%1,%2,%3}, [%4];"
      : "=l"(a0), "=l"(a1), "=l"(a2), "=l"(a3)
      : "l"(p));
#else
  asm volatile("ld.global.nc.v4.b64 {%0,%1,%2,%3}, [%4];"
      : "=l"(a0), "=l"(a1), "=l"(a2), "=l"(a3)
      : "l"(p));
#endif
  const uint32_t k = v & 3u;
  b = k == 0 ? a0 : k == 1 ? a1 : k == 2 ? a2 : a3;
  e = k == 0 ? a1 : k == 1 ? a2 : k == 2 ? a3 : __ldg(p + 4);
}

// The 16-byte record of vertex v; for a CSR (mode 2) one is made from its
// row pointers: {start low 32 bits, start bits 32..47, degree, 0}.
template <int MODE>
__device__ __forceinline__ uint4 graph_record(const DevGraph &g, uint32_t v) {
  if constexpr (MODE == 2) {
    uint64_t b, e;
    csr_row(g.rowptr, v, b, e);
    return make_uint4((uint32_t)b, (uint32_t)(b >> 32) & 0xFFFFu, (uint32_t)(e - b), 0u);
  } else {
    return load_record(g.recs + v);
  }
}

template <int MODE>
__device__ __forceinline__ VHdr header(const DevGraph &g, uint32_t v) {
  return record_header<MODE>(graph_record<MODE>(g, v), v);
}

__device__ __forceinline__ uint32_t record_degree(const DevGraph &g, uint32_t v) {
  return __ldg(&g.recs[v].z);
}

// Length of gamma(x): 2 floor(log2(x+1)) + 1.
__device__ __forceinline__ uint32_t gamma_len(uint32_t x) {
  return 2u * (31u - __clz(x + 1u)) + 1u;
}

template <int MODE>
__device__ __forceinline__ uint32_t neighbor(const DevGraph &g, const VHdr &h, uint32_t i) {
  if constexpr (MODE == 0) return gt_neighbor(g, h, i);
  else if constexpr (MODE == 1) return le_neighbor(g, h, i);
  else return load_cold_u32(g.cols + h.P + i);
}

// A compressed draw (GT or LE) in two halves, so that a lane can have the
// sector loads of several draws in flight before it decodes any: where its
// slot is (draw_at), then its value from the loaded sector (draw_value).
struct DrawAt {
  uint64_t pos;       // bit offset of the slot
  uint32_t c, id, L;  // slot, index in it, slot length (LE)
};

template <int MODE>
__device__ __forceinline__ DrawAt draw_at(const VHdr &h, uint32_t i) {
  DrawAt at;
  if constexpr (MODE == 0) {
    at.c = div_small(i, h.bl);
    at.id = i - at.c * h.bl;
    at.L = 0;
  } else {
    le_locate(h, i, at.c, at.id, at.L);
  }
  at.pos = slot_pos(h, at.c);
  return at;
}

template <int MODE>
__device__ __forceinline__ uint32_t draw_value(const Sec &A, const DrawAt &at, const VHdr &h) {
  const uint32_t off = (uint32_t)at.pos & 255u;
  if constexpr (MODE == 0) {
    const uint32_t hv = (uint32_t)sec1_field(A, off, h.a) + 1u;
    return (at.c >= h.fp ? h.v + hv : h.v - hv) + at.id +
           sec1_sum(A, off + (uint32_t)h.a, at.id, h.b);
  } else {
    return le_slot_value(A, off, h, at.c, at.id, at.L);
  }
}

// End bit of a vertex's on-disk payload given its stream header (load-time
// validation).  For the files the reference compressor writes this is offsets[v+1]
// (GT/chunk_compress/compressor.hpp:297-349, LE/chunk_compress/compressor.hpp:329-390).
template <int MODE>
__device__ __forceinline__ uint64_t payload_end(const DevGraph &g, const VHdr &h) {
  if constexpr (MODE == 0) {
    return gt_disk_block_pos(h, h.bn);
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
