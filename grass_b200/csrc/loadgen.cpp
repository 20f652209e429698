// loadgen.cpp -- open-loop Poisson load generator for the serving loop.
//
// The reference has no serving path and no load generator (its apps run once
// per process, GT/src/main.cu:28-50).  This drives the C ABI only: either a
// grass_server (mode 0) or, on the same request trace, the plain method of
// one standalone launch per request (mode 1), and reports latency
// percentiles and sampled edges per second.
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <list>
#include <thread>
#include <vector>

#include "internal.h"

namespace grass {
namespace {

using Clock = std::chrono::steady_clock;

uint64_t splitmix64(uint64_t &x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

double unit(uint64_t &x) { return ((splitmix64(x) >> 11) + 0.5) * 0x1.0p-53; }  // (0, 1)

double normal(uint64_t &x) {  // Box-Muller
  const double u = unit(x), v = unit(x);
  return std::sqrt(-2.0 * std::log(u)) * std::cos(6.283185307179586 * v);
}

struct TraceReq {
  grass_request rq{};
  std::vector<uint32_t> input;
  double arrival_us = 0;
};

std::vector<TraceReq> make_trace(const grass_loadgen_config &c, uint64_t n) {
  std::vector<TraceReq> tr(c.requests);
  uint64_t x = c.seed;
  double t = 0;
  for (uint32_t i = 0; i < c.requests; i++) {
    TraceReq &q = tr[i];
    t += -std::log(unit(x)) / c.rate * 1e6;
    q.arrival_us = t;
    grass_request &r = q.rq;
    uint64_t y = c.seed ^ (0xA5A5A5A5ull << 32) ^ i;
    r.seed = splitmix64(y);
    const uint32_t pick = (uint32_t)(unit(x) * 100);
    const double sz = std::exp(c.size_mu + c.size_sigma * normal(x));
    const uint32_t count =
        (uint32_t)std::min<double>(std::max<double>(std::llround(sz), 1.0), c.size_max);
    if (pick < c.pct_rw) {
      r.type = GRASS_JOB_RW;
      r.count = count;
      r.length = c.rw_len_min + (uint32_t)(unit(x) * (c.rw_len_max - c.rw_len_min + 1));
      r.layout = 0;
    } else if (pick < c.pct_rw + c.pct_khop) {
      r.type = GRASS_JOB_KHOP;
      r.count = count;
      const uint32_t f = std::min<uint32_t>((uint32_t)(unit(x) * c.n_fanouts), c.n_fanouts - 1);
      r.hops = 0;
      for (uint32_t h = 0; h < 4 && c.fanouts[f][h]; h++) r.fanouts[r.hops++] = c.fanouts[f][h];
    } else {
      r.type = GRASS_JOB_MRW;
      r.count = c.mrw_samples;
      r.walkers = c.mrw_walkers;
      r.steps = c.mrw_steps;
      r.select = c.mrw_select;
    }
    if (r.type != GRASS_JOB_MRW) {
      q.input.resize(r.count);
      uint64_t z = r.seed;
      for (auto &v : q.input) v = (uint32_t)(((splitmix64(z) >> 32) * n) >> 32);
      r.input = q.input.data();
    }
  }
  return tr;
}

double pct(std::vector<double> v, double p) {
  if (v.empty()) return 0;
  std::sort(v.begin(), v.end());
  size_t k = (size_t)std::ceil(p * v.size());
  return v[k ? k - 1 : 0];
}

struct Outcome {
  std::vector<double> lat[3];
  std::vector<double> all, queue, service;
  double issue_us = 0, alloc_us = 0, phase_us[6] = {0, 0, 0, 0, 0, 0};
  double edges = 0, first = 1e300, last = 0;
  uint64_t completed = 0, rejected = 0, failed = 0;
};

void finish_report(const grass_loadgen_config &c, const Outcome &o, grass_loadgen_report *r) {
  r->completed = o.completed;
  r->rejected = o.rejected;
  r->failed = o.failed;
  r->p50_us = pct(o.all, 0.50);
  r->p99_us = pct(o.all, 0.99);
  r->p999_us = pct(o.all, 0.999);
  double s = 0, m = 0;
  for (double v : o.all) {
    s += v;
    m = std::max(m, v);
  }
  r->mean_us = o.all.empty() ? 0 : s / o.all.size();
  r->max_us = m;
  for (int t = 0; t < 3; t++) {
    r->p50_type_us[t] = pct(o.lat[t], 0.50);
    r->p99_type_us[t] = pct(o.lat[t], 0.99);
  }
  r->queue_p50_us = pct(o.queue, 0.50);
  r->queue_p99_us = pct(o.queue, 0.99);
  r->service_p50_us = pct(o.service, 0.50);
  r->service_p99_us = pct(o.service, 0.99);
  r->issue_us = o.issue_us;
  r->staging_alloc_us = o.alloc_us;
  for (int k = 0; k < 6; k++) r->phase_us[k] = o.phase_us[k];
  r->wall_s = o.last > o.first ? (o.last - o.first) * 1e-6 : 0;
  r->edges = o.edges;
  r->edges_per_s = r->wall_s > 0 ? o.edges / r->wall_s : 0;
  r->offered_rate = c.rate;
  r->achieved_rate = r->wall_s > 0 ? o.completed / r->wall_s : 0;
}

// Spins (yielding) until the clock reaches t0 + us.
void wait_until(Clock::time_point t0, double us) {
  const auto due = t0 + std::chrono::nanoseconds((int64_t)(us * 1e3));
  while (Clock::now() < due) std::this_thread::yield();
}

double since_us(Clock::time_point t0) {
  return std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
}

int run_server(const grass_graph *g, const grass_loadgen_config &c, std::vector<TraceReq> &tr,
               Outcome &o, uint64_t &batches) {
  grass_server *srv = nullptr;
  if (int rc = grass_server_create(g, &c.server, &srv)) return rc;
  const size_t N = tr.size();
  std::vector<uint64_t> ticket(N, 0);
  std::vector<double> lag(N, 0), submit_at(N, 0);
  std::vector<std::atomic<int>> state(N);  // 0 pending, 1 submitted, 2 rejected
  for (auto &s : state) s.store(0);
  Clock::time_point t0;
  std::atomic<bool> started{false};
  // The collector takes results as they finish and releases each at once,
  // oldest first but not only in order: a request still queued must not keep
  // later, finished results (and the staging or scratch they hold) alive.
  std::thread collector([&] {
    while (!started.load(std::memory_order_acquire)) std::this_thread::yield();
    auto record = [&](size_t i, int rc, const grass_result &res) {
      if (rc || res.status) {
        o.failed++;
      } else {
        // Latency from the scheduled arrival: the server's own submit-to-done
        // plus how late the submit was.
        const double l = res.done_us - res.submit_us + lag[i];
        o.all.push_back(l);
        o.lat[std::min<uint32_t>(tr[i].rq.type, 2)].push_back(l);
        o.queue.push_back(res.launch_us - res.submit_us + lag[i]);
        o.service.push_back(res.done_us - res.launch_us);
        o.edges += (double)res.edges;
        o.completed++;
        o.last = std::max(o.last, submit_at[i] + (res.done_us - res.submit_us));
      }
      grass_server_release(srv, ticket[i]);
    };
    std::list<size_t> open;  // submitted, not yet collected, in ticket order
    size_t next = 0, closed = 0;
    double oldest_since = -1;  // when the collector started waiting on open.front()
    // Later requests are checked only while the oldest has been waited for a
    // while (a queued request, not merely a long one), and a bounded number
    // per pass, so that polling does not compete with the dispatcher.
    constexpr size_t kScan = 256;
    constexpr double kScanAfterUs = 10000;
    while (closed < N) {
      while (next < N) {
        const int sv = state[next].load(std::memory_order_acquire);
        if (sv == 0) break;
        if (sv == 2) closed++;
        else open.push_back(next);
        next++;
      }
      if (open.empty()) {
        std::this_thread::yield();
        continue;
      }
      const size_t i = open.front();
      if (oldest_since < 0) oldest_since = since_us(t0);
      grass_result res;
      const int rc = grass_server_wait(srv, ticket[i], 2, &res);
      if (rc != GRASS_E_TIMEOUT) {
        record(i, rc, res);
        open.pop_front();
        closed++;
        oldest_since = -1;
        continue;
      }
      size_t k = since_us(t0) - oldest_since < kScanAfterUs ? kScan : 0;
      for (auto it = std::next(open.begin()); it != open.end() && k < kScan; k++) {
        int d = 0;
        if (grass_server_poll(srv, ticket[*it], &d) == GRASS_OK && d) {
          grass_result r2;
          record(*it, grass_server_wait(srv, ticket[*it], 0, &r2), r2);
          it = open.erase(it);
          closed++;
        } else {
          ++it;
        }
      }
      if (since_us(t0) - oldest_since > 1e3 * c.timeout_ms) {  // give the oldest up
        o.failed++;
        open.pop_front();
        closed++;
        oldest_since = -1;
      }
    }
  });
  t0 = Clock::now();
  started.store(true, std::memory_order_release);
  for (size_t i = 0; i < N; i++) {
    wait_until(t0, tr[i].arrival_us);
    const double at = since_us(t0);
    lag[i] = at - tr[i].arrival_us;
    submit_at[i] = at;
    o.first = std::min(o.first, tr[i].arrival_us);
    if (grass_server_submit(srv, &tr[i].rq, &ticket[i]) == GRASS_OK) {
      state[i].store(1, std::memory_order_release);
    } else {
      o.rejected++;
      state[i].store(2, std::memory_order_release);
    }
  }
  collector.join();
  grass_server_stats st;
  grass_server_stats_get(srv, &st);
  batches = st.batches;
  o.issue_us = st.issue_us;
  o.alloc_us = st.staging_alloc_us;
  for (int k = 0; k < 6; k++) o.phase_us[k] = st.phase_us[k];
  return grass_server_destroy(srv, c.timeout_ms);
}

int run_single(const grass_graph *g, const grass_loadgen_config &c, std::vector<TraceReq> &tr,
               Outcome &o) {
  // Buffers for the largest request of the trace, reused by every request.
  uint64_t max_in = 1, max_out = 1;
  for (auto &q : tr) {
    const grass_request &r = q.rq;
    uint64_t in = r.count, out = 0;
    if (r.type == GRASS_JOB_RW) out = (uint64_t)r.count * (r.length + 1);
    if (r.type == GRASS_JOB_KHOP) {
      uint64_t w = 1;
      for (uint32_t h = 0; h < r.hops; h++) out += (uint64_t)r.count * (w *= r.fanouts[h]);
    }
    if (r.type == GRASS_JOB_MRW) {
      in = (uint64_t)r.count * r.walkers;
      out = 2ull * r.count * r.steps;
    }
    max_in = std::max(max_in, in);
    max_out = std::max(max_out, out);
  }
  int dev = 0;
  cudaGetDevice(&dev);
  cudaStream_t s = nullptr;
  uint32_t *d_in = nullptr, *d_out = nullptr, *h_in = nullptr, *h_out = nullptr;
  unsigned long long *d_e = nullptr, *h_e = nullptr;
  int rc = GRASS_OK;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&d_in, max_in * 4) != cudaSuccess || cudaMalloc(&d_out, max_out * 4) != cudaSuccess ||
      cudaMalloc(&d_e, 8) != cudaSuccess || cudaMallocHost(&h_in, max_in * 4) != cudaSuccess ||
      cudaMallocHost(&h_out, max_out * 4) != cudaSuccess || cudaMallocHost(&h_e, 8) != cudaSuccess)
    rc = set_error(GRASS_E_OOM, "one-job-per-launch buffers");
  const Clock::time_point t0 = Clock::now();
  for (size_t i = 0; !rc && i < tr.size(); i++) {
    const grass_request &r = tr[i].rq;
    wait_until(t0, tr[i].arrival_us);
    o.first = std::min(o.first, tr[i].arrival_us);
    uint64_t in = r.type == GRASS_JOB_MRW ? (uint64_t)r.count * r.walkers : r.count;
    uint64_t out_words = 0;
    int k = GRASS_OK;
    if (r.type != GRASS_JOB_MRW) {
      memcpy(h_in, r.input, in * 4);
      cudaMemcpyAsync(d_in, h_in, in * 4, cudaMemcpyHostToDevice, s);
    }
    cudaMemsetAsync(d_e, 0, 8, s);
    if (r.type == GRASS_JOB_RW) {
      grass_rw_params p{r.length, r.layout, r.seed};
      out_words = (uint64_t)r.count * (r.length + 1);
      k = grass_rw(g, &p, d_in, r.count, d_out, d_e, s);
    } else if (r.type == GRASS_JOB_KHOP) {
      grass_khop_params p{};
      p.hops = r.hops;
      for (uint32_t h = 0; h < r.hops; h++) p.fanouts[h] = r.fanouts[h];
      p.seed = r.seed;
      uint32_t *outs[GRASS_MAX_HOPS] = {nullptr};
      uint64_t w = 1;
      for (uint32_t h = 0; h < r.hops; h++) {
        outs[h] = d_out + out_words;
        out_words += (uint64_t)r.count * (w *= r.fanouts[h]);
      }
      k = grass_khop(g, &p, d_in, r.count, outs, d_e, s);
    } else {
      grass_mrw_params p{r.walkers, r.steps, r.select, 0, r.seed};
      grass_graph_info info;
      grass_get_info(g, &info);
      k = grass_mrw_roots(info.n, r.count, r.walkers, r.seed, d_in, s);
      out_words = 2ull * r.count * r.steps;
      if (!k)
        k = grass_mrw(g, &p, d_in, r.count, d_out, d_out + (uint64_t)r.count * r.steps, d_e, s);
    }
    cudaMemcpyAsync(h_out, d_out, out_words * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(h_e, d_e, 8, cudaMemcpyDeviceToHost, s);
    const cudaError_t e = cudaStreamSynchronize(s);
    const double done = since_us(t0);
    if (k || e != cudaSuccess) {
      o.failed++;
      if (e != cudaSuccess) rc = set_error(GRASS_E_CUDA, "one-job-per-launch: %s", cudaGetErrorString(e));
      continue;
    }
    const double l = done - tr[i].arrival_us;
    o.all.push_back(l);
    o.lat[std::min<uint32_t>(r.type, 2)].push_back(l);
    o.edges += (double)*h_e;
    o.completed++;
    o.last = std::max(o.last, done);
  }
  if (s) cudaStreamDestroy(s);
  cudaFree(d_in);
  cudaFree(d_out);
  cudaFree(d_e);
  cudaFreeHost(h_in);
  cudaFreeHost(h_out);
  cudaFreeHost(h_e);
  (void)dev;
  return rc;
}

}  // namespace
}  // namespace grass

extern "C" int grass_loadgen_run(const grass_graph *g, const grass_loadgen_config *c,
                                 grass_loadgen_report *r) {
  using namespace grass;
  clear_error();
  if (!g || !c || !r) return set_error(GRASS_E_ARG, "null argument");
  if (!(c->rate > 0) || c->mode > 1 || c->pct_rw + c->pct_khop > 100 ||
      (c->pct_khop && !c->n_fanouts) || c->n_fanouts > 8 || c->rw_len_max < c->rw_len_min ||
      !c->size_max || (c->pct_rw + c->pct_khop < 100 && (!c->mrw_walkers || !c->mrw_samples)))
    return set_error(GRASS_E_ARG, "loadgen: bad configuration");
  grass_graph_info info;
  if (int rc = grass_get_info(g, &info)) return rc;
  grass_loadgen_config cc = *c;
  if (!cc.timeout_ms) cc.timeout_ms = 120000;
  std::vector<TraceReq> tr = make_trace(cc, info.n);
  memset(r, 0, sizeof(*r));
  Outcome o;
  const uint64_t l0 = grass_launch_count();
  uint64_t batches = 0;
  const int rc = cc.mode == 0 ? run_server(g, cc, tr, o, batches) : run_single(g, cc, tr, o);
  finish_report(cc, o, r);
  r->batches = cc.mode == 0 ? batches : o.completed;
  r->launches = grass_launch_count() - l0;
  return rc;
}
