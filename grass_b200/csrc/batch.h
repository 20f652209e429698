// batch.h -- work items of the batched persistent kernel (internal).
#pragma once
#include <vector>

#include "graph.h"
#include "mrw_cta.cuh"
#include "sample_warp.cuh"

namespace grass {

// Device-side job descriptor.
struct BatchJob {
  uint32_t type, count;
  uint64_t seed;
  const uint32_t *in;
  uint32_t *roots, *out0, *out1;
  unsigned char *mscr;  // multi-RW scratch: mstride bytes per sample
  uint64_t mstride;
  unsigned long long *edges;
  uint32_t length, layout, walkers, steps, select;
  uint32_t gen_roots;  // multi-RW: draw the start vertices first (as grass_mrw_roots)
  KhopArgs khop;
};

// One work item: items [begin, end) of job `job` (walkers, seeds or samples).
struct BatchTask {
  uint32_t job, pad;
  uint64_t begin, end;
};

// Zero fields of a config take the defaults for this decode mode.
grass_batch_config resolve_batch_config(const grass_batch_config &c, int mode);

// Walk jobs of at most this many walkers are split into one-pass work items.
// Measured in the serving loop (R-MAT s24 ef16, results in device memory):
// p50 at 2 k req/s 0.73 ms against 1.01 ms, p99 at 80 % of peak 3.3 ms
// against 3.65 ms, peak 75 k against 76 k req/s; the 256-job batch within 1 %.
#ifndef GRASS_BATCH_SMALL_RW
#define GRASS_BATCH_SMALL_RW 2048
#endif

// Walkers per work item of a walk job of `count` walkers (resolved config):
// a small job takes one pass per item (32 x depth walkers), so that its
// walkers run side by side instead of in sequential passes of one warp.
inline uint64_t rw_tile(uint64_t count, const grass_batch_config &c) {
  const uint64_t pass = 32ull * c.depth;
  return count <= GRASS_BATCH_SMALL_RW && c.walker_tile > pass ? pass : c.walker_tile;
}

// Multi-RW scratch bytes of a job (count samples of mrw_sample_scratch).
inline uint64_t mrw_job_scratch(const grass_job &j) {
  return j.type == GRASS_JOB_MRW ? (uint64_t)j.count * mrw_sample_scratch(j.walkers, j.steps, j.select)
                                 : 0;
}

// Fills a device job descriptor from a job (mscr: mrw_job_scratch(j) bytes
// for a multi-RW job, else null).
BatchJob make_batch_job(const grass_job &j, unsigned char *mscr);

// Appends the work items of job index `ji`, split per config, to the queues:
// block-level items (multi-RW samples whose walkers move in parallel,
// selections 0 and 2), then warp-level items (sequential multi-RW samples,
// k-hop seed groups, walker tiles).
void split_job(const grass_job &j, uint32_t ji, const grass_batch_config &c,
               std::vector<BatchTask> &cta, std::vector<BatchTask> &mrw,
               std::vector<BatchTask> &khop, std::vector<BatchTask> &rw);

// Launches the persistent kernel on graph `dg` (compressed or CSR) of device
// `device` over ntasks work items, the first ncta of them block-level.
// d_queue: two zeroed counters.  Corrupt payloads set bit 0 of *d_err.
int launch_batch(const DevGraph &dg, int device, const BatchJob *d_jobs, const BatchTask *d_tasks,
                 uint32_t ncta, uint32_t ntasks, unsigned int *d_queue,
                 unsigned long long *d_total, unsigned int *d_err, cudaStream_t s,
                 const grass_batch_config &c);

}  // namespace grass
