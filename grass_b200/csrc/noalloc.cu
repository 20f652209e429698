// noalloc.cu -- a decode-only sweep that allocates no device memory.
//
// grass_decode_all needs a little scratch for its row-pointer scan (one
// 64-bit partial sum per 4096-vertex tile) and takes it from the
// stream-ordered allocator.  Some callers cannot allocate at that point:
// applications that reserve the whole device up front for their own memory
// pool (where cudaMallocAsync fails for lack of memory), and latency-bound
// loops that must not pay for allocator calls or the device-wide
// synchronisation that cudaFree implies.  grass_decode_all_noalloc takes the
// same inputs and outputs but draws its scratch from the fixed array below,
// which every GPU that loads this library holds until the process exits.
#include <mutex>

#include "graph.h"

namespace {

// Tile partial sums for graphs of up to 65,536 tiles x 4096 vertices
// (268,435,456 vertices); 512 KiB plus two entries.
constexpr uint64_t kNoAllocMaxTiles = 65536;
constexpr uint64_t kNoAllocMaxVertices = kNoAllocMaxTiles * 4096;

static __device__ __align__(256) uint64_t g_decode_scratch[kNoAllocMaxTiles + 2];

// The symbol's device address, looked up once per device.  In host code
// g_decode_scratch names a host-side stand-in, not device memory, so it is
// never passed to a kernel directly.
std::mutex g_scratch_mu;
uint64_t *g_scratch_ptr[64] = {nullptr};

int scratch_for_device(int device, uint64_t **out) {
  if (device < 0 || device >= 64) return grass::set_error(GRASS_E_ARG, "device %d out of range", device);
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[device]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_decode_scratch);  // device is current
    if (e != cudaSuccess) return grass::cuda_fail(e, "cudaGetSymbolAddress(g_decode_scratch)");
    g_scratch_ptr[device] = static_cast<uint64_t *>(p);
  }
  *out = g_scratch_ptr[device];
  return GRASS_OK;
}

}  // namespace

extern "C" int grass_decode_all_noalloc(const grass_graph *g, uint64_t *d_rowptr,
                                        uint32_t *d_cols, void *stream) {
  grass::Nvtx nvtx_("grass_decode_all_noalloc");
  using namespace grass;
  clear_error();
  if (!g) return set_error(GRASS_E_ARG, "null graph");
  if (!d_rowptr || (!d_cols && g->info.num_edges)) return set_error(GRASS_E_ARG, "null output");
  const uint64_t n = g->info.n;
  if (n > kNoAllocMaxVertices)
    return set_error(GRASS_E_ARG,
                     "graph has %llu vertices; the allocation-free decode handles at most %llu "
                     "(use grass_decode_all)",
                     (unsigned long long)n, (unsigned long long)kNoAllocMaxVertices);
  DeviceGuard dg(g->device);
  uint64_t *scratch = nullptr;
  if (int rc = scratch_for_device(g->device, &scratch)) return rc;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  // Nothing in the scratch has to start at zero: the scan writes every tile
  // sum it later reads.  All calls share the array, so calls that overlap on
  // the GPU (other streams, other threads) race on it.
  launch_degrees64(g->view(), d_rowptr, st);
  launch_scan_u64_inplace(d_rowptr, n, scratch, st);
  // The planned sweep once an earlier grass_decode_all has built the graph's
  // plan (launching it allocates nothing); until then the unplanned sweep,
  // which needs no plan and is about 3x slower.
  if (!launch_decode_if_planned(g, d_rowptr, d_cols, g->d_err, st))
    launch_decode_all(g->view(), d_rowptr, d_cols, g->info.num_edges, g->d_err, st);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GRASS_OK : cuda_fail(e, "kernel launch");
}
