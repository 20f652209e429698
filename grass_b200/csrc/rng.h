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

}  // namespace grass
