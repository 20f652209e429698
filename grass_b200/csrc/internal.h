// internal.h -- shared host-side helpers of the grass_b200 library.
#pragma once
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>

#include <nvtx3/nvToolsExt.h>

#include <atomic>
#include <string>

#include "../../include/grass.h"

namespace grass {

// NVTX range over a scope (header-only NVTX3: a no-op unless a profiler such
// as Nsight Systems is attached), so a timeline shows each entry point and
// the phases of a graph load; the reference times its phases with host
// timers instead (GT/src/grass.cu:1564-1569, 2002-2003).
struct Nvtx {
  explicit Nvtx(const char *name) { nvtxRangePushA(name); }
  ~Nvtx() { nvtxRangePop(); }
  Nvtx(const Nvtx &) = delete;
  Nvtx &operator=(const Nvtx &) = delete;
};

// Records a message for grass_last_error() on this thread and returns code.
int set_error(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
void clear_error();

// Incremented once per kernel launch issued by this library.
extern std::atomic<uint64_t> g_launches;
inline void count_launch(uint64_t k = 1) { g_launches.fetch_add(k, std::memory_order_relaxed); }

// bits(x): number of significant bits of |x|, with bits(0) == 1
// (get_bit_num, GT/chunk_compress/compressor.hpp:15-21).
inline int bit_count(uint64_t x) { return x == 0 ? 1 : 64 - __builtin_clzll(x); }

inline uint64_t isqrt_floor(uint64_t x) {
  // floor(sqrt(x)); equals the compressor's (int64)sqrt((double)x) for x < 2^52.
  uint64_t r = (uint64_t)__builtin_sqrt((double)x);
  while (r * r > x) r--;
  while ((r + 1) * (r + 1) <= x) r++;
  return r;
}

}  // namespace grass
