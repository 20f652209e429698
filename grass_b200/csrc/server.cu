// server.cu -- serving loop over a resident compressed graph.
//
// The reference answers one app invocation per process (GT/src/main.cu:28-50,
// nextdoor() in GT/src/grass.cu:2066-2135) and has no request path.  Here
// client threads submit RW / k-hop / multi-RW requests; one dispatcher thread
// groups waiting requests into a batch, reserves their device scratch against
// the budget and issues, on one of up to sixteen streams:
//
//   H2D (job table, work items, inputs, zeroed counters)
//     -> persistent batch kernel (which also draws multi-RW start vertices)
//     -> D2H (counters, and the outputs unless they stay on the device)
//     -> host callback
//
// Device scratch comes from one allocation of the whole budget made at
// create and handed out first-fit when a batch is admitted (a stream-ordered
// pool allocation per batch cost ~0.4 ms of dispatcher time as the pool grew
// and fragmented); a batch's block returns when its callback runs, its
// outputs' block (results on the device) when the last of its requests is
// released.
//
// Requests come in two classes with separate queues and batches: RW / k-hop
// (short, parallel over walkers and seeds) and multi-RW (sequential chains
// of `steps` dependent draws).  A short request never waits for a chain that
// happens to share its batch, and chains hold at most half of the streams.
//
// The host callback (no CUDA calls) marks the requests done and wakes the
// dispatcher and the waiters.  Every request keeps its own Philox key and
// 0-based walker / seed / sample ids, so its output is the standalone call's.
//
// Device blocks of one batch (every part 256-byte aligned):
//   work: [multi-RW scratch] | H2D: [jobs][work items][queue][inputs]
//         | H2D+D2H: [edges u64 x jobs][error word] | D2H: [outputs]
//   outputs on the device: the [outputs] part is a block of its own.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batch.h"

namespace grass {
namespace {

using Clock = std::chrono::steady_clock;
constexpr uint64_t kAlign = 256;
constexpr uint32_t kMaxSlots = 16;
constexpr double kFallbackUs = 5000;  // staging wait with nothing in flight before the fallback

inline uint64_t align_up(uint64_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// A region handed out first-fit from address-ordered free ranges that
// coalesce on return: the pinned host staging arena (cudaHostAlloc takes
// milliseconds per 100 MB and must not sit in a request's latency) and the
// device scratch arena, both made once at create.
struct Arena {
  std::mutex mu;
  uint8_t *base = nullptr;
  uint64_t size = 0;
  std::map<uint64_t, uint64_t> free_;  // offset -> bytes

  static uint64_t round(uint64_t b) { return (std::max<uint64_t>(b, 1) + 4095) & ~4095ull; }
  void reset(void *p, uint64_t bytes) {
    base = static_cast<uint8_t *>(p);
    size = bytes & ~4095ull;
    free_.clear();
    if (size) free_.emplace(0, size);
  }
  // A block of at least `bytes`, or nullptr while the arena has no room.
  void *take(uint64_t bytes) {
    bytes = round(bytes);
    std::lock_guard<std::mutex> lk(mu);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < bytes) continue;
      const uint64_t off = it->first, len = it->second;
      free_.erase(it);
      if (len > bytes) free_.emplace(off + bytes, len - bytes);
      return base + off;
    }
    return nullptr;
  }
  void give(void *p, uint64_t bytes) {
    if (!p) return;
    bytes = round(bytes);
    std::lock_guard<std::mutex> lk(mu);
    uint64_t off = static_cast<uint8_t *>(p) - base;
    auto next = free_.lower_bound(off);
    if (next != free_.end() && off + bytes == next->first) {
      bytes += next->second;
      next = free_.erase(next);
    }
    if (next != free_.begin()) {
      auto prev = std::prev(next);
      if (prev->first + prev->second == off) {
        prev->second += bytes;
        return;
      }
    }
    free_.emplace(off, bytes);
  }
};

// Pinned buffers for batches larger than the whole arena, cached by size
// class.  cudaFreeHost synchronises the device, so buffers are only freed
// when the server ends.
struct PinnedPool {
  std::mutex mu;
  std::multimap<uint64_t, void *> free_;
  std::vector<void *> all;

  // alloc_us accumulates the time spent in cudaHostAlloc.
  void *get(uint64_t bytes, uint64_t &cap, double &alloc_us) {
    // Capacities 2^k * {4, 5, 6, 7} / 4 (at most 25% slack), 1 MiB at least.
    uint64_t p2 = 1ull << 20;
    while (p2 * 2 <= bytes) p2 <<= 1;
    cap = p2;
    for (uint64_t q = 5; cap < bytes; q++) cap = p2 * q / 4;
    {
      std::lock_guard<std::mutex> lk(mu);
      auto it = free_.lower_bound(cap);
      if (it != free_.end() && it->first <= 4 * cap) {
        void *p = it->second;
        cap = it->first;
        free_.erase(it);
        return p;
      }
    }
    void *p = nullptr;
    const auto t0 = std::chrono::steady_clock::now();
    const cudaError_t e = cudaHostAlloc(&p, cap, cudaHostAllocDefault);
    alloc_us +=
        std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count();
    if (e != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    std::lock_guard<std::mutex> lk(mu);
    all.push_back(p);
    return p;
  }
  void put(void *p, uint64_t cap) {
    if (!p) return;
    std::lock_guard<std::mutex> lk(mu);
    free_.emplace(cap, p);
  }
  ~PinnedPool() {
    for (void *p : all) cudaFreeHost(p);
  }
};

struct Batch;

struct Req {
  uint64_t ticket = 0;
  grass_request rq{};
  std::vector<uint32_t> input;
  uint32_t *pin_in = nullptr;  // input copied at submit into pinned staging, read by the
  uint64_t pin_bytes = 0;      // kernel in place (RW starts, k-hop seeds)
  bool draw_roots = false;  // MRW roots drawn on the device from the seed
  int cls = 0;              // 0: RW / k-hop, 1: multi-RW
  uint32_t nout = 0;
  uint64_t out_words[GRASS_MAX_HOPS] = {0};
  uint64_t in_words = 0, mscr_bytes = 0;
  uint64_t bytes = 0;  // device scratch without the batch's tables
  uint64_t in_bytes = 0, out_bytes = 0;  // staging (aligned inputs, aligned outputs)
  uint64_t draws = 0;  // sampled edges at most (batch sizing)
  double t_submit = 0, t_launch = 0, t_done = 0;
  int status = GRASS_OK;
  bool done = false;
  Batch *batch = nullptr;
  uint64_t out_off[GRASS_MAX_HOPS] = {0};  // byte offsets in the batch's D2H staging
  uint32_t job = 0;                        // index in the batch
  uint64_t edges = 0;
};

struct Batch {
  uint64_t seq = 0;
  uint32_t slot = 0;
  int cls = 0;
  std::vector<Req *> reqs;
  uint64_t bytes = 0;  // device block (budget charge)
  uint64_t h2d_off = 0, h2d_bytes = 0, d2h_off = 0, d2h_bytes = 0;
  void *in_host = nullptr, *out_host = nullptr;
  uint64_t in_cap = 0, out_cap = 0;  // reserved bytes
  bool oversize = false;             // staging from the fallback pool, not the arena
  uint8_t *d_work = nullptr, *d_out = nullptr;  // device blocks (d_out: results on device)
  uint64_t work_bytes = 0, out_bytes = 0;       // their sizes (budget charges)
  uint32_t refs = 0;  // requests not yet released
  grass_server *srv = nullptr;
};

}  // namespace
}  // namespace grass

using grass::Batch;
using grass::Req;

struct grass_server {
  const grass_graph *g = nullptr;
  grass_server_config cfg{};
  grass_batch_config bcfg{};
  cudaStream_t streams[grass::kMaxSlots] = {nullptr};
  bool slot_busy[grass::kMaxSlots] = {false};
  grass::Arena staging, scratch;  // pinned host, device
  grass::PinnedPool pinned;
  bool dev_out = false;  // results stay on the device

  std::mutex mu;
  std::condition_variable cv_work;  // dispatcher: new request, finished batch, stop
  std::condition_variable cv_done;  // waiters
  std::thread th;
  bool stop = false;
  std::deque<Req *> waiting[2];  // per class, FIFO
  uint64_t waiting_draws[2] = {0, 0};
  uint32_t running_cls[2] = {0, 0};
  std::unordered_map<uint64_t, Req *> reqs;
  uint64_t next_ticket = 1, next_batch = 1;
  uint32_t running = 0;
  uint64_t in_use = 0;
  grass_server_stats st{};
  double busy_since = 0;
  double staging_blocked_since = -1;  // first failed staging take with nothing in flight
  grass::Clock::time_point t0;

  double now_us() const {
    return std::chrono::duration<double, std::micro>(grass::Clock::now() - t0).count();
  }
  void loop();
  uint32_t free_slot(int cls) const;
  double window_left(int cls, double now) const;
  Batch *form(double now, int cls);
  void launch(Batch *b);
  void finish(Batch *b, int status);
  void release_in(Batch *b) {
    if (b->oversize) pinned.put(b->in_host, b->in_cap);
    else staging.give(b->in_host, b->in_cap);
    b->in_host = nullptr;
  }
  void release_out(Batch *b) {
    if (b->oversize) pinned.put(b->out_host, b->out_cap);
    else staging.give(b->out_host, b->out_cap);
    b->out_host = nullptr;
    if (b->d_out) scratch.give(b->d_out, b->out_bytes);
    b->d_out = nullptr;
  }
};

namespace grass {
namespace {

// Output sizes, device bytes and draw count of a request; GRASS_OK or an
// argument error.  Mirrors the checks of the standalone calls.
int size_request(const grass_request &r, Req &q) {
  q.nout = 0;
  const uint64_t c = r.count;
  switch (r.type) {
    case GRASS_JOB_RW:
      if (r.layout > 1 || r.length > (1u << 24) || (c && !r.input))
        return set_error(GRASS_E_ARG, "RW request: bad arguments");
      q.in_words = c;
      q.nout = 1;
      q.out_words[0] = c * (r.length + 1ull);
      q.draws = c * (uint64_t)r.length;
      break;
    case GRASS_JOB_KHOP: {
      if (r.hops == 0 || r.hops > GRASS_MAX_HOPS || (c && !r.input))
        return set_error(GRASS_E_ARG, "k-hop request: bad arguments");
      uint64_t w = 1;
      q.draws = 0;
      for (uint32_t h = 0; h < r.hops; h++) {
        if (!r.fanouts[h]) return set_error(GRASS_E_ARG, "k-hop request: fanout %u is zero", h);
        w *= r.fanouts[h];
        if (w > (1ull << 32)) return set_error(GRASS_E_ARG, "k-hop request: fanout product too large");
        q.out_words[h] = c * w;
        q.draws += c * w;
      }
      q.in_words = c;
      q.nout = r.hops;
      break;
    }
    case GRASS_JOB_MRW:
      if (!r.walkers || r.select > 2 || r.steps > (1u << 28))
        return set_error(GRASS_E_ARG, "multi-RW request: bad arguments");
      q.in_words = c * r.walkers;
      q.mscr_bytes = c * mrw_sample_scratch(r.walkers, r.steps, r.select);
      q.nout = 2;
      q.out_words[0] = q.out_words[1] = c * (uint64_t)r.steps;
      q.draws = c * (uint64_t)r.steps;
      q.draw_roots = r.input == nullptr;
      break;
    default:
      return set_error(GRASS_E_ARG, "unknown request type %u", r.type);
  }
  q.in_bytes = align_up(q.in_words * 4);
  q.out_bytes = 0;
  for (uint32_t k = 0; k < q.nout; k++) q.out_bytes += align_up(q.out_words[k] * 4);
  q.bytes = q.in_bytes + align_up(q.mscr_bytes) + q.out_bytes;
  return GRASS_OK;
}

uint64_t table_bytes(size_t njobs, size_t ntasks) {
  return align_up(njobs * sizeof(BatchJob)) + align_up(ntasks * sizeof(BatchTask)) + kAlign +
         align_up(njobs * 8 + 4);
}

// Work items of a request (an upper bound is enough for the budget).
uint64_t task_bound(const Req &q, const grass_batch_config &c) {
  const uint64_t n = q.rq.count;
  if (q.rq.type == GRASS_JOB_RW) {
    const uint64_t t = rw_tile(n, c);
    return (n + t - 1) / t;
  }
  if (q.rq.type == GRASS_JOB_KHOP) return (n + c.khop_seeds - 1) / c.khop_seeds;
  return n;
}

void CUDART_CB on_batch_done(void *arg) {
  Batch *b = static_cast<Batch *>(arg);
  b->srv->finish(b, GRASS_OK);
}

}  // namespace
}  // namespace grass

// A free stream for a batch of this class, or kMaxSlots.
uint32_t grass_server::free_slot(int cls) const {
  using namespace grass;
  if (cls == 1 && running_cls[1] >= std::max<uint32_t>(1, cfg.max_inflight / 2)) return kMaxSlots;
  for (uint32_t i = 0; i < cfg.max_inflight; i++)
    if (!slot_busy[i]) return i;
  return kMaxSlots;
}

// Microseconds until this class's batch is due (<= 0: due now).  The window
// is window_min_us while no batch of the class runs and window_max_us while
// one does; enough waiting work or requests close it at once.
double grass_server::window_left(int cls, double now) const {
  const auto &wq = waiting[cls];
  if (stop || waiting_draws[cls] >= cfg.target_draws || wq.size() >= cfg.max_batch_jobs) return 0;
  const double window = running_cls[cls] ? cfg.window_max_us : cfg.window_min_us;
  return wq.front()->t_submit + window - now;
}

// Takes waiting requests of one class (FIFO) while the device budget and
// the staging arena allow.  Called with mu held.
Batch *grass_server::form(double now, int cls) {
  using namespace grass;
  auto &wq = waiting[cls];
  if (wq.empty()) return nullptr;
  const uint32_t slot = free_slot(cls);
  if (slot == kMaxSlots || window_left(cls, now) > 0) return nullptr;
  Batch *b = new Batch();
  uint64_t data = 0, ntasks = 0, sin = 0, sout = 0;
  const uint64_t cap = staging.size / 8;  // request data per batch (one request may exceed it)
  while (!wq.empty() && b->reqs.size() < cfg.max_batch_jobs) {
    Req *q = wq.front();
    const uint64_t nt = task_bound(*q, bcfg);
    const uint64_t need = data + q->bytes + table_bytes(b->reqs.size() + 1, ntasks + nt);
    if (in_use + need > cfg.scratch_budget) break;
    if (!b->reqs.empty() && data + q->bytes > cap) break;
    data += q->bytes;
    ntasks += nt;
    sin += q->in_bytes;
    sout += q->out_bytes;
    b->reqs.push_back(q);
    wq.pop_front();
    waiting_draws[cls] -= q->draws;
  }
  if (b->reqs.empty()) {  // the oldest request waits for scratch to free up
    delete b;
    return nullptr;
  }
  // Staging: tables and inputs in, counters (and outputs) out.  Device:
  // the work block, and the outputs' own block when they stay on the device.
  b->bytes = data + table_bytes(b->reqs.size(), ntasks);
  b->out_bytes = dev_out ? sout : 0;
  b->work_bytes = b->bytes - b->out_bytes;
  b->in_cap = table_bytes(b->reqs.size(), ntasks) + sin;
  b->out_cap = align_up(b->reqs.size() * 8 + 4) + (dev_out ? 0 : sout);
  bool fallback = false;
  if (Arena::round(b->in_cap) + Arena::round(b->out_cap) > staging.size) {
    b->oversize = true;  // a single request larger than the arena
  } else {
    b->in_host = staging.take(b->in_cap);
    b->out_host = b->in_host ? staging.take(b->out_cap) : nullptr;
    if (!b->out_host) {
      staging.give(b->in_host, b->in_cap);
      b->in_host = nullptr;
      // With batches in flight their finish frees staging (and wakes this
      // loop): wait.  With none, the arena is held by results their callers
      // have not released.  Releases usually follow within microseconds, but
      // waiting for them could wait for good (a caller may hold one result
      // while it waits for the next), so after kFallbackUs with nothing in
      // flight this batch stages through the pinned fallback pool instead.
      if (running == 0) {
        if (staging_blocked_since < 0) staging_blocked_since = now;
        if (now - staging_blocked_since >= kFallbackUs) b->oversize = fallback = true;
      } else {
        staging_blocked_since = -1;
      }
    }
  }
  bool ok = b->oversize || b->out_host;
  if (ok) {
    b->d_work = static_cast<uint8_t *>(scratch.take(b->work_bytes));
    b->d_out = !b->d_work || !b->out_bytes ? nullptr : static_cast<uint8_t *>(scratch.take(b->out_bytes));
    ok = b->d_work && (b->d_out || !b->out_bytes);
  }
  if (!ok) {  // wait for a finish or releases (fragmented arenas); requests go back in order
    if (!b->oversize) {
      staging.give(b->in_host, b->in_cap);
      staging.give(b->out_host, b->out_cap);
    }
    scratch.give(b->d_work, b->work_bytes);
    scratch.give(b->d_out, b->out_bytes);
    for (auto it = b->reqs.rbegin(); it != b->reqs.rend(); ++it) {
      wq.push_front(*it);
      waiting_draws[cls] += (*it)->draws;
    }
    delete b;
    return nullptr;
  }
  if (fallback) st.staging_fallbacks++;
  staging_blocked_since = -1;
  b->slot = slot;
  b->cls = cls;
  running_cls[cls]++;
  b->seq = next_batch++;
  b->srv = this;
  b->refs = (uint32_t)b->reqs.size();
  slot_busy[slot] = true;
  in_use += b->bytes;
  st.scratch_peak = std::max(st.scratch_peak, in_use);
  if (running++ == 0) busy_since = now;
  st.batches++;
  for (Req *q : b->reqs) {
    q->batch = b;
    q->t_launch = now;
  }
  return b;
}

// Issues one batch on its slot's stream.  Called without mu.
void grass_server::launch(Batch *b) {
  using namespace grass;
  cudaStream_t s = streams[b->slot];
  const size_t nj = b->reqs.size();
  std::vector<BatchJob> jobs(nj);
  std::vector<BatchTask> cta, mrw, khop, rw;
  // Offsets inside the device block.
  uint64_t off = 0;
  std::vector<uint64_t> mscr_off(nj), in_off(nj);
  for (size_t i = 0; i < nj; i++) {
    mscr_off[i] = off;
    off += align_up(b->reqs[i]->mscr_bytes);
  }
  b->h2d_off = off;
  const uint64_t jobs_off = off;
  off += align_up(nj * sizeof(BatchJob));
  grass_job gj{};
  for (size_t i = 0; i < nj; i++) {
    const grass_request &r = b->reqs[i]->rq;
    gj.type = r.type;
    gj.count = r.count;
    gj.walkers = r.walkers;
    gj.steps = r.steps;
    gj.select = r.select;
    split_job(gj, (uint32_t)i, bcfg, cta, mrw, khop, rw);
  }
  const uint64_t ntasks = cta.size() + mrw.size() + khop.size() + rw.size();
  const uint64_t tasks_off = off;
  off += align_up(ntasks * sizeof(BatchTask));
  const uint64_t queue_off = off;
  off += kAlign;
  for (size_t i = 0; i < nj; i++) {
    in_off[i] = off;
    if (!b->reqs[i]->pin_in) off += align_up(b->reqs[i]->in_words * 4);
  }
  b->d2h_off = off;
  const uint64_t edges_off = off, err_off = off + nj * 8;
  const uint64_t hdr = align_up(nj * 8 + 4);
  off += hdr;
  b->h2d_bytes = off - b->h2d_off;
  // Outputs: after the header in the work block, or in their own block.
  uint64_t oo = 0;
  for (size_t i = 0; i < nj; i++) {
    Req *q = b->reqs[i];
    for (uint32_t k = 0; k < q->nout; k++) {
      q->out_off[k] = oo;
      oo += align_up(q->out_words[k] * 4);
    }
  }
  b->d2h_bytes = hdr + (dev_out ? 0 : oo);
  uint8_t *const d = b->d_work;
  uint8_t *const dout = dev_out ? b->d_out : d + b->d2h_off + hdr;

  int rc = GRASS_OK;
  const double t_issue = now_us();
  double t_alloc = 0;
  double ph[6] = {0, 0, 0, 0, 0, 0};
  double tp = t_issue;
  auto lap = [&](int k) {
    const double x = now_us();
    ph[k] += x - tp;
    tp = x;
  };
  {
    DeviceGuard dg(g->device);
    if (b->oversize) {
      b->in_host = pinned.get(b->h2d_bytes, b->in_cap, t_alloc);
      b->out_host = pinned.get(b->d2h_bytes, b->out_cap, t_alloc);
    }
    if (!b->in_host || !b->out_host) rc = set_error(GRASS_E_OOM, "pinned staging allocation failed");
    if (!rc && (b->h2d_bytes > b->in_cap || b->d2h_bytes > b->out_cap))
      rc = set_error(GRASS_E_ARG, "internal: staging layout exceeds its reservation");
    if (!rc && (off > b->work_bytes || (dev_out && oo > b->out_bytes)))
      rc = set_error(GRASS_E_ARG, "internal: device layout exceeds its reservation");
    cudaError_t e = cudaSuccess;
    lap(0);
    if (!rc) {
      uint8_t *h = static_cast<uint8_t *>(b->in_host) - b->h2d_off;  // h[x] mirrors d[x]
      for (size_t i = 0; i < nj; i++) {
        Req *q = b->reqs[i];
        const grass_request &r = q->rq;
        grass_job j{};
        j.type = r.type;
        j.count = r.count;
        j.seed = r.seed;
        j.d_input = q->pin_in ? q->pin_in : reinterpret_cast<const uint32_t *>(d + in_off[i]);
        j.d_roots = reinterpret_cast<uint32_t *>(d + in_off[i]);
        j.d_edges = reinterpret_cast<unsigned long long *>(d + edges_off) + i;
        j.length = r.length;
        j.layout = r.layout;
        j.hops = r.hops;
        for (uint32_t k = 0; k < GRASS_MAX_HOPS; k++) j.fanouts[k] = r.fanouts[k];
        j.walkers = r.walkers;
        j.steps = r.steps;
        j.select = r.select;
        uint32_t *outs[GRASS_MAX_HOPS] = {nullptr};
        for (uint32_t k = 0; k < q->nout; k++)
          outs[k] = reinterpret_cast<uint32_t *>(dout + q->out_off[k]);
        if (r.type == GRASS_JOB_KHOP)
          for (uint32_t k = 0; k < r.hops; k++) j.d_hops[k] = outs[k];
        else {
          j.d_out0 = outs[0];
          j.d_out1 = outs[1];
        }
        jobs[i] = make_batch_job(j, d + mscr_off[i]);
        jobs[i].gen_roots = q->draw_roots ? 1u : 0u;  // drawn by the batch kernel
        if (!q->draw_roots && !q->pin_in && q->in_words)
          memcpy(h + in_off[i], q->input.data(), q->in_words * 4);
      }
      memcpy(h + jobs_off, jobs.data(), nj * sizeof(BatchJob));
      BatchTask *ht = reinterpret_cast<BatchTask *>(h + tasks_off);
      for (const auto *v : {&cta, &mrw, &khop, &rw})
        for (const BatchTask &t : *v) *ht++ = t;
      memset(h + queue_off, 0, kAlign);
      memset(h + edges_off, 0, align_up(nj * 8 + 4));
      lap(1);
      e = cudaMemcpyAsync(d + b->h2d_off, b->in_host, b->h2d_bytes, cudaMemcpyHostToDevice, s);
      if (e != cudaSuccess) rc = cuda_fail(e, "server upload");
      lap(2);
    }
    if (!rc && ntasks)
      rc = launch_batch(g->view(), g->device, reinterpret_cast<const BatchJob *>(d + jobs_off),
                        reinterpret_cast<const BatchTask *>(d + tasks_off), (uint32_t)cta.size(),
                        (uint32_t)ntasks,
                        reinterpret_cast<unsigned int *>(d + queue_off), nullptr,
                        reinterpret_cast<unsigned int *>(d + err_off), s, bcfg);
    if (!rc && ntasks) count_launch();
    lap(3);
    if (!rc) {
      e = cudaMemcpyAsync(b->out_host, d + b->d2h_off, b->d2h_bytes, cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) rc = cuda_fail(e, "server download");
    }
    lap(4);
    if (!rc) {
      e = cudaLaunchHostFunc(s, on_batch_done, b);
      if (e != cudaSuccess) rc = cuda_fail(e, "server completion callback");
    }
    lap(5);
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    st.issue_us += now_us() - t_issue;
    st.staging_alloc_us += t_alloc;
    for (int k = 0; k < 6; k++) st.phase_us[k] += ph[k];
  }
  if (rc) {
    // Nothing will call back: wait for what was queued, then fail the batch.
    cudaStreamSynchronize(s);
    cudaGetLastError();
    finish(b, rc);
  }
}

// Marks a batch's requests done and returns its scratch.  Runs on CUDA's
// callback thread (no CUDA calls) or on the dispatcher after a failure.
void grass_server::finish(Batch *b, int status) {
  using namespace grass;
  const double now = now_us();
  unsigned int err = 0;
  const uint8_t *out = static_cast<const uint8_t *>(b->out_host);
  if (!status && out) memcpy(&err, out + b->reqs.size() * 8, 4);
  // Before any request is marked done: a release may free the batch.  The
  // batch's GPU work is over, so its work block can serve the next batch.
  release_in(b);
  scratch.give(b->d_work, b->work_bytes);
  b->d_work = nullptr;
  for (Req *q : b->reqs) {
    staging.give(q->pin_in, q->pin_bytes);
    q->pin_in = nullptr;
  }
  {
    std::lock_guard<std::mutex> lk(mu);
    for (size_t i = 0; i < b->reqs.size(); i++) {
      Req *q = b->reqs[i];
      q->t_done = now;
      q->status = status ? status : err ? GRASS_E_DATA : GRASS_OK;
      if (!q->status) {
        memcpy(&q->edges, out + i * 8, 8);
        st.edges += q->edges;
        st.completed++;
      } else {
        st.failed++;
      }
      q->done = true;
    }
    in_use -= b->work_bytes;  // the outputs' block (if any) returns at release
    if (status) {
      scratch.give(b->d_out, b->out_bytes);
      b->d_out = nullptr;
      in_use -= b->out_bytes;
      b->out_bytes = 0;
    }
    slot_busy[b->slot] = false;
    running_cls[b->cls]--;
    if (--running == 0) st.busy_us += now - busy_since;
    cv_work.notify_all();
    cv_done.notify_all();
  }
}

void grass_server::loop() {
  using namespace grass;
  cudaSetDevice(g->device);
  std::unique_lock<std::mutex> lk(mu);
  for (;;) {
    if (stop && waiting[0].empty() && waiting[1].empty() && running == 0) break;
    const double now = now_us();
    // The class with the older head request goes first.
    int first = 0;
    if (!waiting[1].empty() &&
        (waiting[0].empty() || waiting[1].front()->t_submit < waiting[0].front()->t_submit))
      first = 1;
    Batch *b = form(now, first);
    if (!b) b = form(now, 1 - first);
    if (b) {
      lk.unlock();
      launch(b);
      lk.lock();
      continue;
    }
    // Sleep until a window closes, or a submit/finish.  A batch that was due
    // but not formed waits for scratch or a stream: only a finish helps.
    double wait_us = staging_blocked_since >= 0 && running == 0 ? kFallbackUs / 4 : 50000;
    for (int c = 0; c < 2; c++) {
      if (waiting[c].empty() || free_slot(c) == kMaxSlots) continue;
      const double left = window_left(c, now);
      if (left > 0) wait_us = std::min(wait_us, left);
    }
    cv_work.wait_for(lk, std::chrono::microseconds((int64_t)wait_us + 1));
  }
}

extern "C" {

int grass_server_create(const grass_graph *g, const grass_server_config *cfg,
                        grass_server **out) {
  grass::Nvtx nvtx_("grass_server_create");
  using namespace grass;
  clear_error();
  if (!g || !out) return set_error(GRASS_E_ARG, "null argument");
  *out = nullptr;
  auto *s = new (std::nothrow) grass_server();
  if (!s) return set_error(GRASS_E_OOM, "host allocation failed");
  s->g = g;
  if (cfg) s->cfg = *cfg;
  grass_server_config &c = s->cfg;
  if (!c.scratch_budget) c.scratch_budget = 8ull << 30;
  if (!c.target_draws) c.target_draws = 1ull << 20;
  if (!c.staging_bytes) c.staging_bytes = 1ull << 30;
  if (!c.window_min_us) c.window_min_us = 200;
  if (!c.window_max_us) c.window_max_us = 1000;
  if (c.window_max_us < c.window_min_us) c.window_max_us = c.window_min_us;
  if (!c.max_inflight) c.max_inflight = 16;
  if (!c.max_batch_jobs) c.max_batch_jobs = 4096;
  if (c.max_inflight > kMaxSlots) {
    delete s;
    return set_error(GRASS_E_ARG, "max_inflight above %u", kMaxSlots);
  }
  s->bcfg = resolve_batch_config(c.batch, g->mode);
  c.batch = s->bcfg;
  s->dev_out = c.results_on_device != 0;
  DeviceGuard dg(g->device);
  auto undo = [s]() {
    for (auto st : s->streams)
      if (st) cudaStreamDestroy(st);
    if (s->scratch.base) cudaFree(s->scratch.base);
    if (s->staging.base) cudaFreeHost(s->staging.base);
    delete s;
  };
  cudaError_t e = cudaSuccess;
  for (uint32_t i = 0; e == cudaSuccess && i < c.max_inflight; i++)
    e = cudaStreamCreateWithFlags(&s->streams[i], cudaStreamNonBlocking);
  void *dp = nullptr, *hp = nullptr;
  // (slack for the 4 KiB rounding of a batch's blocks)
  const uint64_t dbytes = ((c.scratch_budget + 4095) & ~4095ull) + (64u << 10);
  if (e == cudaSuccess) e = cudaMalloc(&dp, dbytes);
  if (e == cudaSuccess) s->scratch.reset(dp, dbytes);
  if (e == cudaSuccess) e = cudaHostAlloc(&hp, Arena::round(c.staging_bytes), cudaHostAllocDefault);
  if (e == cudaSuccess) s->staging.reset(hp, Arena::round(c.staging_bytes));
  if (e != cudaSuccess) {
    const int rc = cuda_fail(e, "server setup (streams, scratch, staging)");
    undo();
    return rc;
  }
  s->t0 = Clock::now();
  try {
    s->th = std::thread([s] { s->loop(); });
  } catch (...) {
    undo();
    return set_error(GRASS_E_OOM, "cannot start the dispatcher thread");
  }
  *out = s;
  return GRASS_OK;
}

int grass_server_submit(grass_server *s, const grass_request *r, uint64_t *ticket) {
  grass::Nvtx nvtx_("grass_server_submit");
  using namespace grass;
  clear_error();
  if (!s || !r || !ticket) return set_error(GRASS_E_ARG, "null argument");
  auto *q = new (std::nothrow) Req();
  if (!q) return set_error(GRASS_E_OOM, "host allocation failed");
  q->rq = *r;
  if (int rc = size_request(*r, *q)) {
    delete q;
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.rejected++;
    return rc;
  }
  if (q->bytes + table_bytes(1, task_bound(*q, s->bcfg)) > s->cfg.scratch_budget) {
    const uint64_t need = q->bytes;
    delete q;
    std::lock_guard<std::mutex> lk(s->mu);
    s->st.rejected++;
    return set_error(GRASS_E_BUDGET, "request needs %llu scratch bytes, budget %llu",
                     (unsigned long long)need, (unsigned long long)s->cfg.scratch_budget);
  }
  if (r->type != GRASS_JOB_MRW && q->in_words) {
    // Copied here, on the caller's thread, into pinned memory that the batch
    // kernel reads in place; the dispatcher then has no input to copy.
    q->pin_bytes = q->in_words * 4;
    q->pin_in = static_cast<uint32_t *>(s->staging.take(q->pin_bytes));
    if (q->pin_in) {
      memcpy(q->pin_in, r->input, q->pin_bytes);
      q->bytes -= q->in_bytes;  // no device copy of the input
      q->in_bytes = 0;
    }
  }
  if (!q->draw_roots && !q->pin_in && q->in_words)
    q->input.assign(r->input, r->input + q->in_words);
  q->rq.input = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) {
      s->staging.give(q->pin_in, q->pin_bytes);
      delete q;
      return set_error(GRASS_E_ARG, "server is shutting down");
    }
    q->ticket = s->next_ticket++;
    q->t_submit = s->now_us();
    q->cls = r->type == GRASS_JOB_MRW ? 1 : 0;
    s->reqs.emplace(q->ticket, q);
    s->waiting[q->cls].push_back(q);
    s->waiting_draws[q->cls] += q->draws;
    s->st.submitted++;
    *ticket = q->ticket;
  }
  s->cv_work.notify_one();
  return GRASS_OK;
}

int grass_server_poll(grass_server *s, uint64_t ticket, int *done) {
  using namespace grass;
  clear_error();
  if (!s || !done) return set_error(GRASS_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return set_error(GRASS_E_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  *done = it->second->done ? 1 : 0;
  return GRASS_OK;
}

int grass_server_wait(grass_server *s, uint64_t ticket, uint32_t timeout_ms, grass_result *res) {
  using namespace grass;
  clear_error();
  if (!s) return set_error(GRASS_E_ARG, "null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return set_error(GRASS_E_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  Req *q = it->second;
  if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), [q] { return q->done; }))
    return set_error(GRASS_E_TIMEOUT, "request %llu still running after %u ms",
                     (unsigned long long)ticket, timeout_ms);
  if (res) {
    memset(res, 0, sizeof(*res));
    res->status = q->status;
    res->submit_us = q->t_submit;
    res->launch_us = q->t_launch;
    res->done_us = q->t_done;
    res->batch = q->batch ? q->batch->seq : 0;
    if (!q->status) {
      res->n_outputs = q->nout;
      res->edges = q->edges;
      res->on_device = s->dev_out ? 1u : 0u;
      const uint8_t *out =
          s->dev_out ? q->batch->d_out
                     : static_cast<const uint8_t *>(q->batch->out_host) +
                           align_up(q->batch->reqs.size() * 8 + 4);
      for (uint32_t k = 0; k < q->nout; k++) {
        res->out[k] = reinterpret_cast<const uint32_t *>(out + q->out_off[k]);
        res->out_words[k] = q->out_words[k];
      }
    }
  }
  if (q->status) return set_error(q->status, "request %llu failed", (unsigned long long)ticket);
  return GRASS_OK;
}

int grass_server_release(grass_server *s, uint64_t ticket) {
  using namespace grass;
  clear_error();
  if (!s) return set_error(GRASS_E_ARG, "null argument");
  Batch *free_b = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return set_error(GRASS_E_ARG, "unknown ticket %llu", (unsigned long long)ticket);
    Req *q = it->second;
    if (!q->done) return set_error(GRASS_E_ARG, "request %llu is still running", (unsigned long long)ticket);
    if (q->batch && --q->batch->refs == 0) {
      free_b = q->batch;
      s->in_use -= free_b->out_bytes;  // outputs kept on the device, if any
    }
    s->reqs.erase(it);
    delete q;
  }
  if (free_b) {
    s->release_out(free_b);
    delete free_b;
    s->cv_work.notify_all();  // staging freed: a waiting batch may fit now
  }
  return GRASS_OK;
}

int grass_server_stats_get(grass_server *s, grass_server_stats *out) {
  using namespace grass;
  clear_error();
  if (!s || !out) return set_error(GRASS_E_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  *out = s->st;
  out->waiting = s->waiting[0].size() + s->waiting[1].size();
  out->running = s->running;
  out->scratch_in_use = s->in_use;
  if (s->running) out->busy_us += s->now_us() - s->busy_since;
  return GRASS_OK;
}

int grass_server_destroy(grass_server *s, uint32_t timeout_ms) {
  grass::Nvtx nvtx_("grass_server_destroy");
  using namespace grass;
  clear_error();
  if (!s) return GRASS_OK;
  int rc = GRASS_OK;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    // Requests not yet launched are failed; running batches finish.
    for (auto &wq : s->waiting) {
      for (Req *q : wq) {
        q->status = GRASS_E_TIMEOUT;
        q->done = true;
        s->st.failed++;
        s->staging.give(q->pin_in, q->pin_bytes);
        q->pin_in = nullptr;
      }
      wq.clear();
    }
    s->waiting_draws[0] = s->waiting_draws[1] = 0;
    s->stop = true;
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms),
                             [s] { return s->running == 0; }))
      rc = set_error(GRASS_E_TIMEOUT, "%u batches still running after %u ms", s->running, timeout_ms);
  }
  if (rc) return rc;  // the dispatcher and callbacks still reference the server
  s->th.join();
  DeviceGuard dg(s->g->device);
  for (uint32_t i = 0; i < kMaxSlots; i++)
    if (s->streams[i]) {
      cudaStreamSynchronize(s->streams[i]);
      cudaStreamDestroy(s->streams[i]);
    }
  for (auto &kv : s->reqs) {
    Batch *b = kv.second->batch;
    if (b && --b->refs == 0) {
      s->release_out(b);
      delete b;
    }
    delete kv.second;
  }
  s->reqs.clear();
  cudaFree(s->scratch.base);
  cudaFreeHost(s->staging.base);
  delete s;
  return GRASS_OK;
}

}  // extern "C"
