// batch.h -- work items of the batched persistent kernel (internal).
#pragma once
#include <vector>

#include "graph.h"
#include "sample_warp.cuh"

namespace grass {

// Device-side job descriptor.
struct BatchJob {
  uint32_t type, count;
  uint64_t seed;
  const uint32_t *in;
  uint32_t *roots, *out0, *out1;
  uint4 *wrec;  // multi-RW: count * walkers vertex records (scratch)
  unsigned long long *edges;
  uint32_t length, layout, walkers, steps, select, pad;
  KhopArgs khop;
};

// One work item: items [begin, end) of job `job` (walkers, seeds or samples).
struct BatchTask {
  uint32_t job, pad;
  uint64_t begin, end;
};

// Zero fields of a config take the defaults for this decode mode.
grass_batch_config resolve_batch_config(const grass_batch_config &c, int mode);

// Fills a device job descriptor from a job (wrec: multi-RW scratch of count *
// walkers records, or null for other types).
BatchJob make_batch_job(const grass_job &j, uint4 *wrec);

// Appends the work items of job index `ji`, split per config, to the three
// queues (multi-RW samples, k-hop seed groups, walker tiles).
void split_job(const grass_job &j, uint32_t ji, const grass_batch_config &c,
               std::vector<BatchTask> &mrw, std::vector<BatchTask> &khop,
               std::vector<BatchTask> &rw);

// Launches the persistent kernel over ntasks work items (queue must be zero).
// Corrupt payloads set bit 0 of *d_err.
int launch_batch(const grass_graph *g, const BatchJob *d_jobs, const BatchTask *d_tasks,
                 uint32_t ntasks, unsigned int *d_queue, unsigned long long *d_total,
                 unsigned int *d_err, cudaStream_t s, const grass_batch_config &c);

}  // namespace grass
