// rng.h -- counter-based Philox4x32-10 shared by host and device code.
//
// Replaces the reference's per-thread cuRAND XORWOW states
// (GT/src/grass.cu:1119-1124, GT/src/rand_num_gen.cuh:117-122).  Philox is
// implemented from the published description (Salmon, Moraes, Dror, Shaw,
// "Parallel Random Numbers: As Easy as 1, 2, 3", SC'11).  Being stateless,
// each draw is a pure function of (seed, counter), so a walk is identical
// whichever kernel, batch or launch order produces it.
//
// Stream layout (key = seed; counter = {c0, id_lo, id_hi, tag}):
//   random walk     c0 = step >> 2,  id = walker,  tag = TAG_RW,          word step & 3
//   k-hop           c0 = slot >> 2,  id = sample,  tag = TAG_KHOP | hop,  word slot & 3
//                   (slot = parent_index * fanout + k within the hop)
//   multi-RW        c0 = step,       id = sample,  tag = TAG_MRW,
//                   word 0 (+ word 2 as high half) picks the walker, word 1 the neighbor
//   uniform starts  c0 = i >> 2,     id = 0,       tag = TAG_START,       word i & 3
//   multi-RW roots  c0 = i >> 2,     id = 0,       tag = TAG_MRW_ROOT,    word i & 3
//   node2vec        c0 = step,       id = walker,  tag = TAG_N2V | try,
//                   word 0 picks the candidate, word 1 is the acceptance draw
//   multi-RW, continuous time (select 2): counter {k, sample, walker, TAG_MRW_CT}
//                   for event k of a walker: words 0-1 its holding time, word 2
//                   its neighbor
// Index map: idx = (r * d) >> 32 (replaces min((int)(curand_uniform * d), d - 1)).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define GRASS_HD __host__ __device__ __forceinline__
#else
#define GRASS_HD inline
#endif

namespace grass {

constexpr uint32_t TAG_RW = 0x52570001u;
constexpr uint32_t TAG_KHOP = 0x4b480000u;
constexpr uint32_t TAG_MRW = 0x4d520001u;
constexpr uint32_t TAG_START = 0x53540001u;
constexpr uint32_t TAG_MRW_ROOT = 0x4d520002u;
constexpr uint32_t TAG_GEN = 0x47454e01u;
constexpr uint32_t TAG_MRW_CT = 0x4d520003u;
constexpr uint32_t TAG_N2V = 0x4e320000u;  // | try (16 bits)

struct u32x4 {
  uint32_t x, y, z, w;
};

GRASS_HD uint32_t mulhi_u32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
  return __umulhi(a, b);
#else
  return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

GRASS_HD uint64_t mulhi_u64(uint64_t a, uint64_t b) {
#if defined(__CUDA_ARCH__)
  return __umul64hi(a, b);
#else
  return (uint64_t)(((unsigned __int128)a * b) >> 64);
#endif
}

GRASS_HD u32x4 philox4x32_10(uint64_t seed, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  uint32_t x0 = c0, x1 = c1, x2 = c2, x3 = c3;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
  for (int r = 0; r < 10; r++) {
    const uint32_t m0 = 0xD2511F53u, m1 = 0xCD9E8D57u;
    uint32_t hi0 = mulhi_u32(m0, x0), lo0 = m0 * x0;
    uint32_t hi1 = mulhi_u32(m1, x2), lo1 = m1 * x2;
    uint32_t y0 = hi1 ^ x1 ^ k0;
    uint32_t y2 = hi0 ^ x3 ^ k1;
    x0 = y0;
    x1 = lo1;
    x2 = y2;
    x3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return u32x4{x0, x1, x2, x3};
}

GRASS_HD uint32_t pick(const u32x4& v, int i) {
  return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// ---------------------------------------------------------------------------
// Deterministic exponential variates for the continuous-time multi-RW.
//
// The host oracle and the device must produce bit-identical event times, so
// the logarithm uses only correctly rounded double +, *, / in a fixed order
// (device: __dadd_rn / __dmul_rn / __ddiv_rn, which the compiler never fuses
// into FMAs; host: plain operators without FP contraction):
//   u = m 2^e with m in [sqrt(1/2), sqrt(2)),  s = (m - 1) / (m + 1),  z = s^2,
//   ln u = e ln2 + 2 s (1 + z/3 + z^2/5 + ... + z^10/21)   (atanh series;
//   |s| <= 0.1716 so the truncation error is below 1e-17 relative).
#if defined(__CUDA_ARCH__)
#define GRASS_DADD(a, b) __dadd_rn(a, b)
#define GRASS_DMUL(a, b) __dmul_rn(a, b)
#define GRASS_DDIV(a, b) __ddiv_rn(a, b)
GRASS_HD double bits_f64(uint64_t b) { return __longlong_as_double((long long)b); }
GRASS_HD uint64_t f64_bits(double d) { return (uint64_t)__double_as_longlong(d); }
#else
#define GRASS_DADD(a, b) ((a) + (b))
#define GRASS_DMUL(a, b) ((a) * (b))
#define GRASS_DDIV(a, b) ((a) / (b))
GRASS_HD double bits_f64(uint64_t b) {
  double d;
  __builtin_memcpy(&d, &b, 8);
  return d;
}
GRASS_HD uint64_t f64_bits(double d) {
  uint64_t b;
  __builtin_memcpy(&b, &d, 8);
  return b;
}
#endif

GRASS_HD double det_log(double u) {
  const uint64_t b = f64_bits(u);
  int e = (int)((b >> 52) & 0x7FF) - 1023;
  double m = bits_f64((b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull);
  if (m > 0x1.6a09e667f3bcdp+0) {
    m = GRASS_DMUL(m, 0.5);
    e += 1;
  }
  const double s = GRASS_DDIV(GRASS_DADD(m, -1.0), GRASS_DADD(m, 1.0));
  const double z = GRASS_DMUL(s, s);
  double p = 0x1.8618618618618p-5;               // 1/21
  p = GRASS_DADD(0x1.af286bca1af28p-5, GRASS_DMUL(z, p));  // 1/19
  p = GRASS_DADD(0x1.e1e1e1e1e1e1ep-5, GRASS_DMUL(z, p));  // 1/17
  p = GRASS_DADD(0x1.1111111111111p-4, GRASS_DMUL(z, p));  // 1/15
  p = GRASS_DADD(0x1.3b13b13b13b14p-4, GRASS_DMUL(z, p));  // 1/13
  p = GRASS_DADD(0x1.745d1745d1746p-4, GRASS_DMUL(z, p));  // 1/11
  p = GRASS_DADD(0x1.c71c71c71c71cp-4, GRASS_DMUL(z, p));  // 1/9
  p = GRASS_DADD(0x1.2492492492492p-3, GRASS_DMUL(z, p));  // 1/7
  p = GRASS_DADD(0x1.999999999999ap-3, GRASS_DMUL(z, p));  // 1/5
  p = GRASS_DADD(0x1.5555555555555p-2, GRASS_DMUL(z, p));  // 1/3
  const double t = GRASS_DADD(s, GRASS_DMUL(s, GRASS_DMUL(z, p)));
  return GRASS_DADD(GRASS_DMUL((double)e, 0x1.62e42fefa39efp-1), GRASS_DMUL(2.0, t));
}

// Exp(1) variate from words 0-1 of a Philox block: u = (u52 + 1/2) 2^-52 in
// (0, 1), exactly representable, then -ln u > 0.
GRASS_HD double exp_variate(uint32_t w0, uint32_t w1) {
  const uint64_t u52 = ((uint64_t)w0 << 20) | (w1 >> 12);
  const double u = GRASS_DMUL(GRASS_DADD((double)u52, 0.5), 0x1p-52);
  return -det_log(u);
}

// Next event time t + E / d of a walker at degree d > 0; strictly after t.
GRASS_HD double next_event_time(double t, double E, uint32_t d) {
  const double nt = GRASS_DADD(t, GRASS_DDIV(E, (double)d));
  return nt > t ? nt : bits_f64(f64_bits(t) + 1);
}

}  // namespace grass
