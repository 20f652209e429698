// kernels_batch.cu -- many uneven sampling jobs in one persistent launch.
//
// The reference runs one app over all vertices per process, one kernel
// pipeline per step (GT/src/grass.cu:1417-2037).  Here a batch holds any mix
// of RW, k-hop and multi-RW jobs with their own sizes, parameters and seeds.
// The host splits them into work items -- one multi-RW sample, a few k-hop
// seeds, or a tile of walkers -- ordered longest first (multi-RW chains are
// sequential by definition), and a persistent kernel's warps pull items from
// a device counter until the queue is empty.  The queue reset, the restore of
// the multi-RW start vertices and the kernel are captured once into a CUDA
// graph and replayed by every run.
#include <algorithm>
#include <map>
#include <mutex>
#include <vector>

#include "batch.h"

// Resident blocks per SM the compiler must allow for, per graph mode (the
// register budget).  The batched-jobs workload waits on memory, so more
// resident warps pay until spills cost more: measured on the 256-job mix,
// LE is best at 3 (80 registers; 2x over 1), GT and CSR at 4 (64 registers).
#ifndef GRASS_BATCH_MIN_BLOCKS_LE
#define GRASS_BATCH_MIN_BLOCKS_LE 3
#endif
#ifndef GRASS_BATCH_MIN_BLOCKS_OTHER
#define GRASS_BATCH_MIN_BLOCKS_OTHER 4
#endif

namespace grass {
namespace {

template <int MODE, int DEPTH>
__global__ void __launch_bounds__(256, MODE == 1 ? GRASS_BATCH_MIN_BLOCKS_LE
                                               : GRASS_BATCH_MIN_BLOCKS_OTHER) batch_kernel(DevGraph g, const BatchJob *__restrict__ jobs,
                                                    const BatchTask *__restrict__ tasks,
                                                    uint32_t ncta, uint32_t ntasks,
                                                    unsigned int *queue,
                                                    unsigned long long *total,
                                                    unsigned int *err) {
  __shared__ SmemHdr sh[8];
  __shared__ CtaSmem<8> csm;
  __shared__ __align__(16) uint32_t dbuf[8][32 * kDrawBufWords];  // k-hop draw staging
  SmemHdr &my = sh[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  uint64_t all = 0;
  bool bad = false;
  // Block-level items first: multi-RW samples whose walkers move in parallel.
  while (ncta) {
    if (threadIdx.x == 0) csm.task = atomicAdd(queue + 1, 1u);
    __syncthreads();
    const uint32_t c = csm.task;
    __syncthreads();
    if (c >= ncta) break;
    const BatchTask tk = tasks[c];
    const BatchJob &jb = jobs[tk.job];
    const uint64_t s = tk.begin;
    uint64_t cnt = 0;
    if (jb.gen_roots) {
      for (uint32_t w = threadIdx.x; w < jb.walkers; w += blockDim.x)
        jb.roots[s * jb.walkers + w] = mrw_root(g.n, jb.seed, s * jb.walkers + w);
      __syncthreads();
    }
    mrw_cta_sample<MODE, 8>(g, jb.roots + s * jb.walkers, jb.out0 + s * jb.steps,
                            jb.out1 + s * jb.steps, jb.walkers, jb.steps, jb.select, jb.seed, s,
                            jb.mscr + s * jb.mstride, csm, cnt, bad);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(kFull, cnt, o);
    if (lane == 0 && cnt) {
      if (jb.edges) atomicAdd(jb.edges, (unsigned long long)cnt);
      all += cnt;
    }
  }
  for (;;) {
    uint32_t t = 0;
    if (lane == 0) t = ncta + atomicAdd(queue, 1u);
    t = __shfl_sync(kFull, t, 0);
    if (t >= ntasks) break;
    const BatchTask tk = tasks[t];
    const BatchJob &jb = jobs[tk.job];
    uint64_t cnt = 0;
    if (jb.type == GRASS_JOB_RW) {
      rw_warp<MODE, DEPTH>(g, jb.in, jb.count, jb.length, jb.seed, 0, (int)jb.layout, jb.out0,
                           tk.begin, tk.end, cnt, bad);
    } else if (jb.type == GRASS_JOB_KHOP) {
      const uint32_t parts = max(1u, tk.pad >> 8), part = tk.pad & 0xFFu;
      for (uint64_t s = tk.begin; s < tk.end; s++)
        khop_seed_warp<MODE>(g, jb.in, jb.khop, s, my, dbuf[threadIdx.x >> 5], cnt, bad, part,
                             parts);
    } else {
      for (uint64_t s = tk.begin; s < tk.end; s++) {
        if (jb.gen_roots) {
          for (uint32_t w = lane; w < jb.walkers; w += 32)
            jb.roots[s * jb.walkers + w] = mrw_root(g.n, jb.seed, s * jb.walkers + w);
          __syncwarp();
        }
        mrw_warp<MODE>(g, jb.roots + s * jb.walkers,
                       reinterpret_cast<uint4 *>(jb.mscr + s * jb.mstride), jb.walkers,
                       jb.steps, (int)jb.select, jb.seed, s, jb.out0, jb.out1, cnt, bad);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_down_sync(kFull, cnt, o);
    if (lane == 0 && cnt) {
      if (jb.edges) atomicAdd(jb.edges, (unsigned long long)cnt);
      all += cnt;
    }
  }
  if (lane == 0 && total && all) atomicAdd(total, (unsigned long long)all);
  if (bad && err) atomicOr(err, 1u);
}

using BatchKernel = void (*)(DevGraph, const BatchJob *, const BatchTask *, uint32_t, uint32_t,
                             unsigned int *, unsigned long long *, unsigned int *);

BatchKernel pick_kernel(int mode, uint32_t depth) {
  if (mode == GRASS_MODE_GT)
    return depth == 4 ? batch_kernel<0, 4> : depth == 2 ? batch_kernel<0, 2> : batch_kernel<0, 1>;
  if (mode == GRASS_MODE_CSR_INTERNAL)
    return depth == 4 ? batch_kernel<2, 4> : depth == 2 ? batch_kernel<2, 2> : batch_kernel<2, 1>;
  return depth == 4 ? batch_kernel<1, 4> : depth == 2 ? batch_kernel<1, 2> : batch_kernel<1, 1>;
}

grass_batch_config resolve(const grass_batch_config &c, int mode) {
  return resolve_batch_config(c, mode);
}

bool same_shape(const grass_batch_config &a, const grass_batch_config &b) {
  return a.walker_tile == b.walker_tile && a.depth == b.depth &&
         a.warps_per_block == b.warps_per_block && a.khop_seeds == b.khop_seeds &&
         a.warps_per_vertex == b.warps_per_vertex;
}

}  // namespace

// Defaults: the autotuner's choice on the 256-job mix for LE, GT and CSR
// alike, and in the serving loop (R-MAT s24 ef16, results in device memory)
// 82 k req/s peak and p99 3.5 ms at 80 % of it, against 78 k and 3.8 ms with
// 128-walker tiles of four interleaved walkers per lane.
grass_batch_config resolve_batch_config(const grass_batch_config &c, int mode) {
  (void)mode;
  grass_batch_config r = c;
  if (!r.walker_tile) r.walker_tile = 64;
  if (!r.depth) r.depth = 1;
  if (!r.warps_per_block) r.warps_per_block = 8;
  if (!r.khop_seeds) r.khop_seeds = 1;
  if (!r.use_graph) r.use_graph = 1;
  if (!r.warps_per_vertex) r.warps_per_vertex = 1;
  return r;
}

BatchJob make_batch_job(const grass_job &j, unsigned char *mscr) {
  BatchJob bj{};
  bj.type = j.type;
  bj.count = j.count;
  bj.seed = j.seed;
  bj.in = j.d_input;
  bj.roots = j.d_roots;
  bj.mscr = mscr;
  bj.mstride = j.type == GRASS_JOB_MRW ? mrw_sample_scratch(j.walkers, j.steps, j.select) : 0;
  bj.out0 = j.d_out0;
  bj.out1 = j.d_out1;
  bj.edges = j.d_edges;
  bj.length = j.length;
  bj.layout = j.layout;
  bj.walkers = j.walkers;
  bj.steps = j.steps;
  bj.select = j.select;
  if (j.type == GRASS_JOB_KHOP) {
    bj.khop.hops = j.hops;
    uint64_t w = 1;
    for (uint32_t h = 0; h < j.hops; h++) {
      bj.khop.fan[h] = j.fanouts[h];
      w *= j.fanouts[h];
      bj.khop.width[h] = w;
      bj.khop.out[h] = j.d_hops[h];
    }
    bj.khop.seed = j.seed;
  }
  return bj;
}

void split_job(const grass_job &j, uint32_t ji, const grass_batch_config &c,
               std::vector<BatchTask> &cta, std::vector<BatchTask> &mrw,
               std::vector<BatchTask> &khop, std::vector<BatchTask> &rw) {
  if (j.type == GRASS_JOB_KHOP) {
    // pad = part | parts << 8: warps_per_vertex items per seed group
    const uint32_t parts = c.warps_per_vertex;
    for (uint64_t s = 0; s < j.count; s += c.khop_seeds)
      for (uint32_t p = 0; p < parts; p++)
        khop.push_back({ji, p | parts << 8, s, std::min<uint64_t>(j.count, s + c.khop_seeds)});
  } else if (j.type == GRASS_JOB_MRW) {
    auto &q = j.select == GRASS_SELECT_DEGREE ? mrw : cta;
    for (uint64_t s = 0; s < j.count; s++) q.push_back({ji, 0, s, s + 1});
  } else {
    const uint64_t tile = rw_tile(j.count, c);
    for (uint64_t w = 0; w < j.count; w += tile)
      rw.push_back({ji, 0, w, std::min<uint64_t>(j.count, w + tile)});
  }
}

int launch_batch(const DevGraph &dg, int device, const BatchJob *d_jobs, const BatchTask *d_tasks,
                 uint32_t ncta, uint32_t ntasks, unsigned int *d_queue,
                 unsigned long long *d_total, unsigned int *d_err, cudaStream_t s,
                 const grass_batch_config &c) {
  BatchKernel k = pick_kernel(dg.mode, c.depth);
  const int threads = 32 * (int)c.warps_per_block;
  // Resident blocks per SM, once per (kernel, block size): the query costs
  // tens of microseconds and the serving loop launches thousands of batches.
  static std::mutex occ_mu;
  static std::map<std::pair<const void *, int>, int> occ;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lk(occ_mu);
    auto it = occ.find({(const void *)k, threads});
    if (it != occ.end()) {
      per_sm = it->second;
    } else {
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, 0);
      occ[{(const void *)k, threads}] = per_sm;
    }
  }
  if (per_sm < 1) per_sm = 1;
  const uint64_t need =
      std::max<uint64_t>(ncta, (ntasks - ncta + c.warps_per_block - 1) / c.warps_per_block);
  const unsigned grid = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>(need, (uint64_t)sm_count(device) * per_sm));
  k<<<grid, threads, 0, s>>>(dg, d_jobs, d_tasks, ncta, ntasks, d_queue, d_total, d_err);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GRASS_OK : cuda_fail(e, "batch kernel launch");
}

}  // namespace grass

using namespace grass;

struct grass_batch {
  // The graph sampled: a compressed graph or an uncompressed CSR (mode 2).
  DevGraph dg{};
  int device = 0;
  unsigned int *d_err = nullptr;  // the graph's error word, or own_err (CSR)
  unsigned int *own_err = nullptr;
  int mode() const { return dg.mode; }
  std::vector<grass_job> jobs;
  grass_batch_config cfg{};
  std::mutex mu;
  // device state built from jobs + cfg
  bool dirty = true;
  grass_batch_config built_cfg{};
  BatchJob *d_jobs = nullptr;
  BatchTask *d_tasks = nullptr;
  uint32_t ntasks = 0, ncta = 0;
  unsigned int *d_queue = nullptr;
  std::vector<void *> owned;                      // MRW record scratch (per build)
  std::vector<uint32_t *> snap;                   // per job: MRW start vertices as added
  std::vector<std::pair<uint32_t *, uint32_t *>> restore;  // (roots, snapshot)
  std::vector<uint64_t> restore_n;
  // captured graph
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  unsigned long long *exec_total = nullptr;

  void free_device() {
    if (exec) cudaGraphExecDestroy(exec);
    exec = nullptr;
    cudaFree(d_jobs);
    cudaFree(d_tasks);
    cudaFree(d_queue);
    d_jobs = nullptr;
    d_tasks = nullptr;
    d_queue = nullptr;
    for (void *p : owned) cudaFree(p);
    owned.clear();
    restore.clear();
    restore_n.clear();
    ntasks = ncta = 0;
  }
  void free_snapshots() {
    for (uint32_t *p : snap) cudaFree(p);
    snap.clear();
  }
  ~grass_batch() {
    free_device();
    free_snapshots();
    if (cap) cudaStreamDestroy(cap);
  }
};

namespace {

int build(grass_batch *b) {
  const grass_batch_config c = resolve(b->cfg, b->mode());
  b->free_device();
  std::vector<BatchJob> hj;
  std::vector<BatchTask> cta, mrw, khop, rw;
  for (size_t i = 0; i < b->jobs.size(); i++) {
    const grass_job &j = b->jobs[i];
    unsigned char *mscr = nullptr;
    if (j.type == GRASS_JOB_MRW) {
      const uint64_t nr = (uint64_t)j.count * j.walkers;
      GRASS_CUDA(cudaMalloc(&mscr, std::max<uint64_t>(mrw_job_scratch(j), 256)));
      b->owned.push_back(mscr);
      b->restore.push_back({j.d_roots, b->snap[i]});
      b->restore_n.push_back(nr);
    }
    hj.push_back(make_batch_job(j, mscr));
    split_job(j, (uint32_t)i, c, cta, mrw, khop, rw);
  }
  std::vector<BatchTask> tasks;  // block-level items, then the longest chains first
  tasks.insert(tasks.end(), cta.begin(), cta.end());
  tasks.insert(tasks.end(), mrw.begin(), mrw.end());
  tasks.insert(tasks.end(), khop.begin(), khop.end());
  tasks.insert(tasks.end(), rw.begin(), rw.end());
  if (tasks.size() > 0xFFFFFFF0ull) return set_error(GRASS_E_ARG, "batch: too many work items");
  b->ntasks = (uint32_t)tasks.size();
  b->ncta = (uint32_t)cta.size();
  GRASS_CUDA(cudaMalloc(&b->d_jobs, std::max<size_t>(hj.size(), 1) * sizeof(BatchJob)));
  GRASS_CUDA(cudaMalloc(&b->d_tasks, std::max<size_t>(tasks.size(), 1) * sizeof(BatchTask)));
  GRASS_CUDA(cudaMalloc(&b->d_queue, 2 * sizeof(unsigned int)));
  if (!hj.empty())
    GRASS_CUDA(cudaMemcpy(b->d_jobs, hj.data(), hj.size() * sizeof(BatchJob),
                          cudaMemcpyHostToDevice));
  if (!tasks.empty())
    GRASS_CUDA(cudaMemcpy(b->d_tasks, tasks.data(), tasks.size() * sizeof(BatchTask),
                          cudaMemcpyHostToDevice));
  b->built_cfg = c;
  b->dirty = false;
  return GRASS_OK;
}

// Queue reset, multi-RW root restore and the persistent kernel, on stream s.
int enqueue(grass_batch *b, cudaStream_t s, unsigned long long *total) {
  const grass_batch_config &c = b->built_cfg;
  for (size_t i = 0; i < b->restore.size(); i++)
    GRASS_CUDA(cudaMemcpyAsync(b->restore[i].first, b->restore[i].second, b->restore_n[i] * 4,
                               cudaMemcpyDeviceToDevice, s));
  GRASS_CUDA(cudaMemsetAsync(b->d_queue, 0, 2 * sizeof(unsigned int), s));
  if (!b->ntasks) return GRASS_OK;
  return launch_batch(b->dg, b->device, b->d_jobs, b->d_tasks, b->ncta, b->ntasks, b->d_queue,
                      total, b->d_err, s, c);
}

int check_job(const grass_job *j) {
  if (!j) return set_error(GRASS_E_ARG, "null job");
  switch (j->type) {
    case GRASS_JOB_RW:
      if (j->layout > 1 || (j->count && (!j->d_input || !j->d_out0)))
        return set_error(GRASS_E_ARG, "RW job: bad arguments");
      return GRASS_OK;
    case GRASS_JOB_KHOP: {
      if (j->hops == 0 || j->hops > GRASS_MAX_HOPS || (j->count && !j->d_input))
        return set_error(GRASS_E_ARG, "k-hop job: bad arguments");
      uint64_t w = 1;
      for (uint32_t h = 0; h < j->hops; h++) {
        if (!j->fanouts[h] || (j->count && !j->d_hops[h]))
          return set_error(GRASS_E_ARG, "k-hop job: fanout or output %u missing", h);
        w *= j->fanouts[h];
        if (w > (1ull << 32)) return set_error(GRASS_E_ARG, "k-hop job: fanout product too large");
      }
      return GRASS_OK;
    }
    case GRASS_JOB_MRW:
      if (!j->walkers || j->select > 2 || (j->count && (!j->d_roots || !j->d_out0 || !j->d_out1)))
        return set_error(GRASS_E_ARG, "multi-RW job: bad arguments");
      return GRASS_OK;
  }
  return set_error(GRASS_E_ARG, "unknown job type %u", j->type);
}

}  // namespace

extern "C" {

int grass_batch_create(const grass_graph *g, grass_batch **out) {
  clear_error();
  if (!g || !out) return set_error(GRASS_E_ARG, "null argument");
  *out = nullptr;
  auto *b = new (std::nothrow) grass_batch();
  if (!b) return set_error(GRASS_E_OOM, "host allocation failed");
  b->dg = g->view();
  b->device = g->device;
  b->d_err = g->d_err;
  *out = b;
  return GRASS_OK;
}

int grass_batch_create_csr(const grass_csr *c, grass_batch **out) {
  clear_error();
  if (!c || !out) return set_error(GRASS_E_ARG, "null argument");
  *out = nullptr;
  auto *b = new (std::nothrow) grass_batch();
  if (!b) return set_error(GRASS_E_OOM, "host allocation failed");
  b->dg = c->graph_view();
  b->device = c->device;
  DeviceGuard dg(c->device);
  cudaError_t e = cudaMalloc(&b->own_err, sizeof(unsigned int));
  if (e == cudaSuccess) e = cudaMemset(b->own_err, 0, sizeof(unsigned int));
  if (e != cudaSuccess) {
    cudaFree(b->own_err);
    delete b;
    return cuda_fail(e, "batch error word");
  }
  b->d_err = b->own_err;
  *out = b;
  return GRASS_OK;
}

int grass_batch_add(grass_batch *b, const grass_job *job) {
  clear_error();
  if (!b) return set_error(GRASS_E_ARG, "null batch");
  if (int rc = check_job(job)) return rc;
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuard dg(b->device);
  // Multi-RW start vertices are copied now: every run starts from them, even
  // though each run leaves the final positions in d_roots.
  uint32_t *snap = nullptr;
  if (job->type == GRASS_JOB_MRW) {
    const uint64_t nr = (uint64_t)job->count * job->walkers;
    GRASS_CUDA(cudaMalloc(&snap, std::max<uint64_t>(nr, 1) * 4));
    const cudaError_t e = cudaMemcpy(snap, job->d_roots, nr * 4, cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) {
      cudaFree(snap);
      return cuda_fail(e, "multi-RW root snapshot");
    }
  }
  b->jobs.push_back(*job);
  b->snap.push_back(snap);
  b->dirty = true;
  return GRASS_OK;
}

int grass_batch_clear(grass_batch *b) {
  if (!b) return set_error(GRASS_E_ARG, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuard dg(b->device);
  b->jobs.clear();
  b->free_device();
  b->free_snapshots();
  b->dirty = true;
  return GRASS_OK;
}

int grass_batch_set_config(grass_batch *b, const grass_batch_config *cfg) {
  if (!b || !cfg) return set_error(GRASS_E_ARG, "null argument");
  const uint32_t t = cfg->walker_tile, d = cfg->depth, w = cfg->warps_per_block,
                 v = cfg->warps_per_vertex;
  if ((t && (t % 32 || t > 4096)) || (d && d != 1 && d != 2 && d != 4) ||
      (w && w != 1 && w != 2 && w != 4 && w != 8) || cfg->use_graph > 2 ||
      (v && v != 1 && v != 2 && v != 4 && v != 8))
    return set_error(GRASS_E_ARG, "batch config: walker_tile multiple of 32 <= 4096, depth 1/2/4, "
                                  "warps_per_block 1/2/4/8, warps_per_vertex 1/2/4/8");
  std::lock_guard<std::mutex> lk(b->mu);
  b->cfg = *cfg;
  if (!same_shape(resolve(b->cfg, b->mode()), b->built_cfg)) b->dirty = true;
  return GRASS_OK;
}

int grass_batch_get_config(const grass_batch *b, grass_batch_config *cfg) {
  if (!b || !cfg) return set_error(GRASS_E_ARG, "null argument");
  *cfg = resolve(b->cfg, b->mode());
  return GRASS_OK;
}

int grass_batch_run(grass_batch *b, void *stream, unsigned long long *d_total_edges) {
  grass::Nvtx nvtx_("grass_batch_run");
  clear_error();
  if (!b) return set_error(GRASS_E_ARG, "null batch");
  std::lock_guard<std::mutex> lk(b->mu);
  DeviceGuard dg(b->device);
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  if (b->dirty) {
    if (int rc = build(b)) return rc;
  }
  if (resolve(b->cfg, b->mode()).use_graph == 2) {
    const int rc = enqueue(b, st, d_total_edges);
    if (!rc && b->ntasks) count_launch();
    return rc;
  }
  if (!b->exec || b->exec_total != d_total_edges) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    if (!b->cap) GRASS_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    GRASS_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue(b, b->cap, d_total_edges);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(b->cap, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    const cudaError_t e2 = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e2 != cudaSuccess) return cuda_fail(e2, "cudaGraphInstantiate");
    b->exec_total = d_total_edges;
  }
  GRASS_CUDA(cudaGraphLaunch(b->exec, st));
  count_launch();
  return GRASS_OK;
}

int grass_batch_autotune(grass_batch *b, void *stream, grass_batch_config *best,
                         float *best_ms) {
  grass::Nvtx nvtx_("grass_batch_autotune");
  clear_error();
  if (!b) return set_error(GRASS_E_ARG, "null batch");
  const grass_batch_config keep = b->cfg;
  grass_batch_config top{};
  float top_ms = 1e30f;
  cudaEvent_t e0, e1;
  {
    DeviceGuard dg(b->device);
    GRASS_CUDA(cudaEventCreate(&e0));
    GRASS_CUDA(cudaEventCreate(&e1));
  }
  const uint32_t tiles[] = {64, 128, 256}, depths[] = {1, 2, 4}, wpbs[] = {1, 2, 4, 8};
  const uint32_t wpvs[] = {1, 2, 4, 8};
  int rc = GRASS_OK;
  for (uint32_t t : tiles) {
    for (uint32_t d : depths) {
      for (uint32_t idx = 0; idx < 16 && !rc; idx++) {
        const uint32_t w = wpbs[idx & 3], v = wpvs[idx >> 2];
        grass_batch_config c = keep;
        c.walker_tile = t;
        c.depth = d;
        c.warps_per_block = w;
        c.warps_per_vertex = v;
        if ((rc = grass_batch_set_config(b, &c))) break;
        if ((rc = grass_batch_run(b, stream, nullptr))) break;  // build + warm-up
        float ms = 1e30f;
        for (int rep = 0; rep < 3 && !rc; rep++) {
          DeviceGuard dg(b->device);
          cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
          cudaEventRecord(e0, st);
          rc = grass_batch_run(b, stream, nullptr);
          cudaEventRecord(e1, st);
          cudaEventSynchronize(e1);
          float x = 0;
          cudaEventElapsedTime(&x, e0, e1);
          ms = std::min(ms, x);
        }
        if (rc) break;
        if (ms < top_ms) {
          top_ms = ms;
          top = resolve(c, b->mode());
        }
      }
      if (rc) break;
    }
    if (rc) break;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) {
    grass_batch_set_config(b, &keep);
    return rc;
  }
  grass_batch_set_config(b, &top);
  if (best) *best = top;
  if (best_ms) *best_ms = top_ms;
  return GRASS_OK;
}

int grass_batch_info(const grass_batch *b, uint64_t *jobs, uint64_t *work_items) {
  if (!b) return set_error(GRASS_E_ARG, "null batch");
  if (jobs) *jobs = b->jobs.size();
  if (work_items) *work_items = b->ntasks;
  return GRASS_OK;
}

int grass_batch_destroy(grass_batch *b) {
  if (!b) return GRASS_OK;
  DeviceGuard dg(b->device);
  cudaFree(b->own_err);
  delete b;
  return GRASS_OK;
}

}  // extern "C"
