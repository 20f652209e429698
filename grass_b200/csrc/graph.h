// graph.h -- host-side handle types and kernel launchers (internal).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "device_common.cuh"
#include "internal.h"

namespace grass {
// Workspace of the host-buffer walk (grass_rw_host): two streams and two
// chunk-sized buffer sets, kept across calls so that steady-state calls
// allocate nothing; chunk i+1 is copied in and walked while chunk i is copied
// out.
struct HostPipe {
  std::mutex mu;
  cudaStream_t st[2] = {nullptr, nullptr};
  cudaEvent_t ev = nullptr;
  uint32_t *d_starts[2] = {nullptr, nullptr};
  uint32_t *d_paths[2] = {nullptr, nullptr};
  size_t cap_starts = 0, cap_paths = 0;  // elements per slot
  unsigned long long *d_edges = nullptr;
  ~HostPipe() {
    for (int i = 0; i < 2; i++) {
      cudaFree(d_starts[i]);
      cudaFree(d_paths[i]);
      if (st[i]) cudaStreamDestroy(st[i]);
    }
    cudaFree(d_edges);
    if (ev) cudaEventDestroy(ev);
  }
};

// Per-launch L2 access-policy window (cudaLaunchAttributeAccessPolicyWindow):
// marks the hot per-vertex table persisting so the random payload reads do
// not evict it between uses.
struct L2Window {
  const void *base = nullptr;
  size_t bytes = 0;
  float hit_ratio = 0.f;
  bool on() const { return base && bytes && hit_ratio > 0.f; }
};
}  // namespace grass

struct grass_graph {
  grass::L2Window l2win;
  grass::HostPipe *pipe = nullptr;  // created by the first grass_rw_host call
  int device = 0;
  int mode = 0;
  uint32_t *d_words = nullptr;     // n_words + guard words
  uint64_t n_words = 0;            // stream words (excluding guard words)
  uint64_t *d_offsets = nullptr;   // n + 1 bit offsets; freed once records exist
  uint4 *d_recs = nullptr;         // n vertex records
  unsigned int *d_err = nullptr;   // device error word (GRASS_E_DATA on bad ids)
  grass_graph_info info{};
  grass_tuning tuning{};
  // Decode plan, built by the first grass_decode_all and kept: the neighbor
  // ranges (v, i0, i1, 0) of vertices with degree >= 32, at most 2048
  // neighbors each, and the vertices of degree 1..31 grouped by
  // floor(log2(degree)).
  mutable std::mutex plan_mu;
  mutable uint4 *d_plan_big = nullptr;
  mutable uint32_t *d_plan_small = nullptr;
  mutable uint64_t plan_nbig = 0, plan_nsmall = 0;
  mutable bool plan_ok = false;
  // The flat plan of the default (unstaged) sweep: runs of consecutive
  // vertices (v0, v1, 0, 0) and hub neighbor ranges (v, v + 1, i0, i1).
  mutable uint4 *d_plan_flat = nullptr;
  mutable uint64_t plan_nflat = 0;
  mutable bool plan_flat_ok = false;
  grass::DevGraph view() const {
    grass::DevGraph g;
    g.words = d_words;
    g.recs = d_recs;
    g.offsets = d_offsets;
    g.n = (uint32_t)info.n;
    g.mode = mode;
    g.rowptr = nullptr;
    g.cols = nullptr;
    return g;
  }
};

struct grass_csr {
  grass::L2Window l2win;
  int device = 0;
  grass_tuning tuning{};
  uint64_t n = 0, nnz = 0;
  uint64_t *d_rowptr = nullptr;
  uint32_t *d_cols = nullptr;
  grass::DevCsr view() const {
    grass::DevCsr c;
    c.rowptr = d_rowptr;
    c.cols = d_cols;
    c.n = (uint32_t)n;
    return c;
  }
  // The same CSR as a sampler graph (mode 2) for the batched kernel.
  grass::DevGraph graph_view() const {
    grass::DevGraph g{};
    g.n = (uint32_t)n;
    g.mode = grass::GRASS_MODE_CSR_INTERNAL;
    g.rowptr = d_rowptr;
    g.cols = d_cols;
    return g;
  }
};

namespace grass {

// Zero words after the stream.  A header read starts at most at the last
// stream bit and decodes four gamma codes of at most 63 bits through a
// cursor that reads two words ahead, so reads stay within 10 words past the
// stream even for a corrupt header; validation runs before any sampling.
constexpr int kGuardWords = 16;

// RAII device switch.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

int cuda_fail(cudaError_t e, const char *what);
#define GRASS_CUDA(call)                                   \
  do {                                                     \
    cudaError_t _e = (call);                               \
    if (_e != cudaSuccess) return grass::cuda_fail(_e, #call); \
  } while (0)

// Streaming SM count of the current device (cached per device).
int sm_count(int device);
// Stream-ordered scratch on the current device from the library's own pool
// (freed memory stays mapped for reuse).
cudaError_t scratch_alloc(void **p, size_t bytes, cudaStream_t s);
void scratch_free(void *p, cudaStream_t s);

// ---- load path (kernels_load.cu) ----
// In-place byte swap of n_words words.
void launch_bswap(uint32_t *w, uint64_t n_words, cudaStream_t s);
// lens of n ubl-bit fields (payload words already native) -> exclusive scan
// into out[0..n]; tmp must hold scan_tmp_words(n) u64.
uint64_t scan_tmp_words(uint64_t n);
void launch_unpack_scan(const uint32_t *payload, uint64_t n, uint32_t ubl, uint64_t *out,
                        uint64_t *tmp, cudaStream_t s);
// u32 counts -> u64 exclusive scan into out[0..n]
void launch_scan_u32(const uint32_t *counts, uint64_t n, uint64_t *out, uint64_t *tmp,
                     cudaStream_t s);
// Header validation: stats[0] = sum of degrees, stats[1] = max degree,
// stats[2] = first bad vertex + 1 (0 if none). deg may be null.
void launch_validate(const DevGraph &g, uint32_t *deg, unsigned long long *stats,
                     cudaStream_t s);
void launch_build_records(const DevGraph &g, uint4 *recs, cudaStream_t s);
// Device layout (sector slots, device_common.cuh) of mode GT or LE: pass 0
// decodes the on-disk stream into a CSR (rowptr = scanned degrees); pass 1
// picks each vertex's chunk length, field widths and slots per sector (meta)
// and first_pos (fpos); the host places the vertices (P, bit offsets); pass 2
// writes the slots into dst (zeroed) and rewrites the records in place.
void launch_disk_decode(int mode, const uint32_t *words, const uint4 *recs, uint32_t n,
                        const uint64_t *rowptr, uint32_t *cols, cudaStream_t s);
void launch_slot_choose(int mode, const uint64_t *rowptr, const uint32_t *cols, uint32_t n,
                        uint32_t *meta, uint32_t *fpos, cudaStream_t s);
void launch_slot_write(int mode, const uint64_t *rowptr, const uint32_t *cols, uint32_t n,
                       const uint32_t *meta, const uint32_t *fpos, const uint64_t *P,
                       uint32_t *dst, uint4 *recs, cudaStream_t s);
void launch_degrees(const DevGraph &g, uint32_t *deg, cudaStream_t s);
void launch_degrees64(const DevGraph &g, uint64_t *deg, cudaStream_t s);
// In-place exclusive scan of vals[0..n) into vals[0..n]; tmp as above.
void launch_scan_u64_inplace(uint64_t *vals, uint64_t n, uint64_t *tmp, cudaStream_t s);

// ---- decode (kernels_decode.cu) ----
// E = rowptr[n] (the number of edges, known from load-time validation).
// Decode sweep through the graph's decode plan (built on first use; the
// build allocates and synchronises once).  rowptr must hold the scanned
// degrees.
int launch_decode_planned(const grass_graph *g, const uint64_t *rowptr, uint32_t *cols,
                          unsigned int *err, cudaStream_t s);
// The planned sweep if the graph's plan is already built (it then allocates
// nothing); false, with nothing launched, if it is not.
bool launch_decode_if_planned(const grass_graph *g, const uint64_t *rowptr, uint32_t *cols,
                              unsigned int *err, cudaStream_t s);
// Decode sweep without a plan: warps over fixed 2048-neighbor tasks of the
// CSR being written (no allocation, no set-up; about 2.4x slower).
void launch_decode_all(const DevGraph &g, const uint64_t *rowptr, uint32_t *cols, uint64_t E,
                       unsigned int *err, cudaStream_t s);

// ---- samplers (kernels_sample.cu) ----
void launch_uniform_starts(uint64_t n, uint64_t count, uint64_t seed, uint32_t *out,
                           cudaStream_t s, bool mrw_roots = false);
// w0: walker id of starts[0] (a chunk of a larger batch draws as walkers w0 + w).
void launch_rw(const DevGraph &g, const grass_rw_params &p, const uint32_t *starts, uint64_t W,
               uint32_t *paths, unsigned long long *edges, unsigned int *err, cudaStream_t s,
               const grass_tuning &t, const L2Window &win = L2Window(), uint64_t w0 = 0);
// Applies the process-wide parts of a tuning block (L2 fetch granularity,
// persisting-L2 carve-out) on `device` and computes the access window for a
// hot table of `bytes` at `base`.
int apply_tuning(int device, const grass_tuning &t, const void *base, size_t bytes,
                 L2Window &win);
// Random-read probe: about `reads` independent random 4-byte reads from
// buf[0, n_words) (n_words a power of two); returns the exact count issued.
uint64_t launch_random_read(const uint32_t *buf, uint64_t n_words, uint64_t reads, uint64_t seed,
                            unsigned long long *sink, cudaStream_t s);
void launch_rw_account(const DevGraph &g, const grass_rw_params &p, const uint32_t *starts,
                       uint64_t W, unsigned long long *out, cudaStream_t s);
void launch_rw_csr(const DevCsr &c, const grass_rw_params &p, const uint32_t *starts,
                   uint64_t W, uint32_t *paths, unsigned long long *edges, cudaStream_t s,
                   const grass_tuning &t, const L2Window &win = L2Window(), uint64_t w0 = 0);
// Fills unset (zero) fields of a tuning block with the defaults.
// kind: GRASS_MODE_GT, GRASS_MODE_LE or 2 (uncompressed CSR).
grass_tuning resolve_tuning(const grass_tuning &t, int kind);
void launch_khop(const DevGraph &g, const grass_khop_params &p, const uint32_t *seeds,
                 uint64_t S, uint32_t *const *hop_out, unsigned long long *edges,
                 unsigned int *err, cudaStream_t s);
// Second-order walk (MODE of g: GT, LE, or 2 for a CSR view); t: the
// acceptance thresholds {return, in, out} in [0, 2^32].
void launch_node2vec(const DevGraph &g, const grass_node2vec_params &p, const uint64_t t[3],
                     const uint32_t *starts, uint64_t W, uint32_t *paths,
                     unsigned long long *edges, unsigned int *err, cudaStream_t s,
                     uint64_t w0 = 0);
void launch_khop_csr(const DevCsr &c, const grass_khop_params &p, const uint32_t *seeds,
                     uint64_t S, uint32_t *const *hop_out, unsigned long long *edges,
                     cudaStream_t s);
int launch_mrw(const DevGraph &g, const grass_mrw_params &p, uint32_t *roots, uint64_t S,
               uint32_t *src, uint32_t *dst, unsigned long long *edges, unsigned int *err,
               cudaStream_t s);

// ---- output compaction (kernels_compact.cu) ----
constexpr uint32_t kCompactMaxSegs = GRASS_MAX_HOPS;
constexpr uint32_t kCompactFan = 0;   // edge e: parent[e / div] -> child[e]
constexpr uint32_t kCompactPath = 1;  // walk-major paths, div = L: edge (q, r) is
                                      // child[q(L+1) + r] -> child[q(L+1) + r + 1]
struct CompactSeg {
  const uint32_t *parent;  // kCompactPath: the path array, as child
  const uint32_t *child;
  uint64_t n;              // edge slots
  uint64_t tile0;          // set by launch_compact
  uint32_t div;
  uint32_t kind;
};
// Writes the valid edges of the segments, in segment then slot order, to
// src/dst[0, cap) and their total number to *count (a device word).  An edge
// is valid when its child is not GRASS_INVALID_VERTEX.
int launch_compact(const CompactSeg *segs, uint32_t nseg, uint32_t *src, uint32_t *dst,
                   uint64_t cap, unsigned long long *count, cudaStream_t s);

}  // namespace grass
