// Visit-count instrumentation for the reference's own GPU random-walk app.
//
// Force-included (nvcc -include) into an otherwise unmodified build of the
// reference's randomwalk app (GT|LE/src/apps/randomwalk/main.cu) to make the
// _visits binaries; the timed binaries are built without it.  The reference
// never materialises its samples (GT/src/grass.cu:1348).  After each step it
// inverts the sample -> transit map with cub::DeviceRadixSort::SortPairs
// (GT/src/grass.cu:1967, LE/src/grass.cu:1850), whose keys_in are the
// samples' transit vertices for the next step (written at
// GT/src/grass.cu:182-184).  This header includes CUB first, then wraps the
// name SortPairs so that every later call also hands its arguments to
// grass_visit::after_sort, which copies keys_in to the host and writes the
// transits of the listed positions:
//
//   GRASS_VISIT_DUMP=<prefix>   GRASS_VISIT_STEPS=1,10,79
//   -> <prefix>.<position>.i32  (num_items int32 transits; the reference's
//      INVALID_VERTEX = n_nodes marks a walk that ended)
//
// Position p is the vertex after step p (the p-th sort of a run; the sizing
// query with a null temp pointer is not counted).  Run with -n 1.  Host-only
// translation units of the same build (AnyOption) see nothing of it.
#pragma once
#ifdef __CUDACC__
#include <cub/cub.cuh>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace grass_visit {

inline bool listed(int pos) {
  const char *s = std::getenv("GRASS_VISIT_STEPS");
  if (!s) return false;
  while (*s) {
    char *end = nullptr;
    const long v = std::strtol(s, &end, 10);
    if (end == s) return false;
    if (v == pos) return true;
    s = *end ? end + 1 : end;
  }
  return false;
}

template <typename K, typename KO, typename VI, typename VO, typename N, typename... Rest>
inline void after_sort(void *temp, size_t, K *keys_in, KO, VI, VO, N num_items, Rest...) {
  static int position = 0;
  const char *prefix = std::getenv("GRASS_VISIT_DUMP");
  if (temp == nullptr || prefix == nullptr) return;  // sizing query, or not asked
  ++position;
  if (!listed(position)) return;
  std::vector<K> h((size_t)num_items);
  if (cudaMemcpy(h.data(), keys_in, h.size() * sizeof(K), cudaMemcpyDeviceToHost) != cudaSuccess) {
    std::fprintf(stderr, "visit_hook: copy of position %d failed\n", position);
    std::exit(3);
  }
  char path[4096];
  std::snprintf(path, sizeof path, "%s.%d.i32", prefix, position);
  FILE *f = std::fopen(path, "wb");
  if (!f || std::fwrite(h.data(), sizeof(K), h.size(), f) != h.size()) {
    std::fprintf(stderr, "visit_hook: cannot write %s\n", path);
    std::exit(3);
  }
  std::fclose(f);
}

}  // namespace grass_visit

#define SortPairs(...) SortPairs(__VA_ARGS__); ::grass_visit::after_sort(__VA_ARGS__)
#endif  // __CUDACC__
