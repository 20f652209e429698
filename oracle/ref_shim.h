/*
 * ref_shim.h -- host definitions for the CUDA names that the reference's
 * decoder header (GT/src/bcg.cuh, LE/src/bcg.cuh) uses, so that header can be
 * compiled unmodified with g++ and run on the CPU as a parity pin for the
 * oracle.  TEST INFRASTRUCTURE ONLY: built into oracle/_ref/, never shipped.
 *
 * Each definition follows the documented semantics of the CUDA intrinsic:
 *   __clz(x)                 number of leading zero bits of a 32-bit int (32 for 0)
 *   __funnelshift_l(lo,hi,s) upper 32 bits of (hi:lo) << (s & 31)
 */
#ifndef GRASS_REF_SHIM_H
#define GRASS_REF_SHIM_H

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <vector>
#include <bitset>

#define __device__
#define __host__
#define __global__
#define __forceinline__ inline

static inline int __clz(uint32_t x) { return x == 0 ? 32 : __builtin_clz(x); }

static inline uint32_t __funnelshift_l(uint32_t lo, uint32_t hi, uint32_t shift) {
  uint64_t v = ((uint64_t)hi << 32) | (uint64_t)lo;
  return (uint32_t)((v << (shift & 31u)) >> 32);
}

template <class A, class B>
static inline auto min(A a, B b) -> decltype(a + b) { return a < b ? a : b; }
template <class A, class B>
static inline auto max(A a, B b) -> decltype(a + b) { return a > b ? a : b; }

struct shim_dim3 { unsigned x, y, z; };
/* The decode_offset kernel body reads these; the harness sets them before
 * calling it once per emulated thread. */
static shim_dim3 threadIdx, blockIdx, blockDim, gridDim;

#endif
