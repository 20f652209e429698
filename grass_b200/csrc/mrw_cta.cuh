// mrw_cta.cuh -- multi random walk with one thread block per sample, walkers
// in parallel (MultiRWApp, GT/src/apps/multiRW/multiRW.cu:3-112).
//
// The warp version (sample_warp.cuh, mrw_warp) takes the T steps one after
// another: ~2 dependent DRAM reads per step, ~19 ms for 10,000 steps.  Two
// selections allow the walkers to move in parallel instead:
//
//  * uniform (select 0): the walker of step t is a function of the Philox
//    block of step t alone, so the block first computes every step's walker,
//    groups the steps by walker (counting sort), and then each thread moves
//    its walkers through their own steps in order.  Bit-identical to the
//    sequential stream; latency ~ the longest per-walker chain.
//
//  * degree-proportional, continuous time (select 2): a walker at degree d
//    waits Exp(d) and then moves to a uniform neighbor, independently of the
//    others.  By the competing-exponentials property, the time-ordered
//    sequence of moves has the law of the sequential degree-proportional
//    process (next mover x with probability d_x / sum d).  Each walker's
//    events come from its own Philox stream (counter {k, sample, walker,
//    TAG_MRW_CT}); the block simulates all walkers up to a time horizon,
//    raising the horizon in phases until T events exist, sorts the events by
//    (time, walker) and keeps the first T.  Event times use det_log, so the
//    host oracle (an event heap) reproduces them bit for bit.
#pragma once
#include "sample_warp.cuh"

namespace grass {

struct CtEvent {
  uint64_t t;  // bits of the (positive) event time: integer order = time order
  uint32_t w, src, dst, pad;
};

struct CtWalker {
  uint32_t v, k, z, pad;  // vertex, event index, neighbor word of event k
  double t;               // time of event k (+inf when the walker cannot move)
};

// Block workspace; NW = most warps per block.
template <int NW>
struct CtaSmem {
  uint32_t hist[NW][256];
  uint32_t tot[256];
  uint64_t red[32];
  uint32_t n_events, overflow, skip, task;
};

__host__ __device__ inline uint64_t mrw_ct_cap(uint32_t T) { return 2ull * T + 4096; }

// Byte offsets in the scratch of a continuous-time sample (from a 256-byte
// aligned base): walkers (24 B), vertex records (16 B, 16-aligned), first
// event past the T-th per walker (4 B), then two event buffers of cap each.
struct CtLayout {
  uint64_t rec, first, ev, total;
  __host__ __device__ CtLayout(uint32_t R, uint32_t T) {
    rec = ((uint64_t)R * sizeof(CtWalker) + 63) & ~63ull;
    first = rec + (uint64_t)R * 16;
    ev = (first + (uint64_t)R * 4 + 63) & ~63ull;
    total = ev + 2 * mrw_ct_cap(T) * sizeof(CtEvent);
  }
};

// Device scratch of one sample, by selection (256-byte multiple).
__host__ __device__ inline uint64_t mrw_sample_scratch(uint32_t R, uint32_t T, uint32_t select) {
  uint64_t b;
  if (select == GRASS_SELECT_UNIFORM)
    b = ((uint64_t)R + 1 + T) * 4;  // step counts per walker + step lists
  else if (select == GRASS_SELECT_DEGREE_CT)
    b = CtLayout(R, T).total;
  else
    b = (uint64_t)R * 16;  // mrw_warp: one vertex record per walker
  return (b + 255) & ~255ull;
}

template <int NW>
__device__ __forceinline__ uint64_t cta_sum_u64(uint64_t v, CtaSmem<NW> &sm) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  __syncthreads();
  if (lane == 0) sm.red[wid] = v;
  __syncthreads();
  uint64_t r = 0;
  for (int i = 0; i < nw; i++) r += sm.red[i];
  __syncthreads();
  return r;
}

// In-place exclusive scan of a[0..n) (global memory) by the whole block.
template <int NW>
__device__ void cta_exclusive_scan(uint32_t *a, uint32_t n, CtaSmem<NW> &sm) {
  const uint32_t nt = blockDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const uint32_t per = (n + nt - 1) / nt;
  const uint32_t b = min(n, tid * per), e = min(n, b + per);
  uint32_t sum = 0;
  for (uint32_t i = b; i < e; i++) sum += a[i];
  uint32_t incl = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, o);
    if ((int)lane >= o) incl += y;
  }
  if (lane == 31) sm.tot[wid] = incl;
  __syncthreads();
  uint32_t run = incl - sum;
  for (uint32_t i = 0; i < wid; i++) run += sm.tot[i];
  for (uint32_t i = b; i < e; i++) {
    const uint32_t x = a[i];
    a[i] = run;
    run += x;
  }
  __syncthreads();
}

// Stable LSD radix sort of a[0..n) by time bits (8-bit digits, passes whose
// digit is the same for every event are skipped), ping-ponging with b;
// returns the sorted buffer.  Each warp owns a contiguous tile; within a
// round of 32 events, __match_any_sync ranks equal digits so the scatter
// keeps input order.  Events with equal times are then ordered by walker.
template <int NW>
__device__ CtEvent *cta_sort_events(CtEvent *a, CtEvent *b, uint32_t n, CtaSmem<NW> &sm) {
  const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t tile = ((n + nw - 1) / nw + 31) / 32 * 32;
  const uint32_t t0 = min(n, wid * tile), t1 = min(n, t0 + tile);
  for (int shift = 0; shift < 64; shift += 8) {
    for (uint32_t i = tid; i < nw * 256; i += blockDim.x) sm.hist[i >> 8][i & 255] = 0;
    __syncthreads();
    for (uint32_t i = t0 + lane; i < t1; i += 32)
      atomicAdd(&sm.hist[wid][(uint32_t)(a[i].t >> shift) & 255u], 1u);
    __syncthreads();
    for (uint32_t d = tid; d < 256; d += blockDim.x) {  // column prefix over warps
      uint32_t run = 0;
      for (uint32_t w = 0; w < nw; w++) {
        const uint32_t c = sm.hist[w][d];
        sm.hist[w][d] = run;
        run += c;
      }
      sm.tot[d] = run;
    }
    __syncthreads();
    if (wid == 0) {  // digit prefix; a digit holding every event makes the pass a no-op
      uint32_t v[8], s = 0;
      bool all = false;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        v[k] = sm.tot[lane * 8 + k];
        s += v[k];
        all |= v[k] == n;
      }
      uint32_t incl = s;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, incl, o);
        if ((int)lane >= o) incl += y;
      }
      uint32_t run = incl - s;
#pragma unroll
      for (int k = 0; k < 8; k++) {
        sm.tot[lane * 8 + k] = run;
        run += v[k];
      }
      const bool skip = __any_sync(kFull, all);
      if (lane == 0) sm.skip = skip ? 1u : 0u;
    }
    __syncthreads();
    if (sm.skip) continue;  // (read by all before warp 0 can write it again)
    for (uint32_t base = t0; base < t1; base += 32) {
      const uint32_t i = base + lane;
      const bool ok = i < t1;
      CtEvent e{};
      uint32_t dg = 256u;
      if (ok) {
        e = a[i];
        dg = (uint32_t)(e.t >> shift) & 255u;
      }
      const unsigned peers = __match_any_sync(kFull, dg);
      const unsigned below = peers & ((1u << lane) - 1u);
      if (ok) b[sm.tot[dg] + sm.hist[wid][dg] + __popc(below)] = e;
      __syncwarp();
      if (ok && below == 0) sm.hist[wid][dg] += __popc(peers);
      __syncwarp();
    }
    __syncthreads();
    CtEvent *x = a;
    a = b;
    b = x;
  }
  // Ties (equal times, necessarily different walkers) in walker order.
  for (uint32_t i = tid; i < n; i += blockDim.x) {
    if ((i == 0 || a[i - 1].t != a[i].t) && i + 1 < n && a[i + 1].t == a[i].t) {
      uint32_t j = i + 1;
      while (j < n && a[j].t == a[i].t) j++;
      for (uint32_t p = i + 1; p < j; p++) {
        const CtEvent x = a[p];
        uint32_t q = p;
        while (q > i && a[q - 1].w > x.w) {
          a[q] = a[q - 1];
          q--;
        }
        a[q] = x;
      }
    }
  }
  __syncthreads();
  return a;
}

// Uniform multi-RW of one sample by the whole block.  scr: R + 1 + T words.
// Step t: walker mulhi(word 0, R), neighbor mulhi(word 1, d) of
// Philox(seed; t, sample, .., TAG_MRW) -- the stream of mrw_warp.
template <int MODE, int NW>
__device__ void mrw_uniform_cta(const DevGraph &g, uint32_t *roots, uint32_t *src, uint32_t *dst,
                                uint32_t R, uint32_t T, uint64_t seed, uint64_t sample,
                                uint32_t *scr, CtaSmem<NW> &sm, uint64_t &cnt, bool &bad) {
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  const uint32_t s_lo = (uint32_t)sample, s_hi = (uint32_t)(sample >> 32);
  uint32_t *cur = scr, *list = scr + R + 1;
  for (uint32_t i = tid; i <= R; i += nt) cur[i] = 0;
  __syncthreads();
  for (uint32_t t = tid; t < T; t += nt)
    atomicAdd(&cur[mulhi_u32(philox4x32_10(seed, t, s_lo, s_hi, TAG_MRW).x, R)], 1u);
  __syncthreads();
  cta_exclusive_scan(cur, R + 1, sm);
  for (uint32_t t = tid; t < T; t += nt)
    list[atomicAdd(&cur[mulhi_u32(philox4x32_10(seed, t, s_lo, s_hi, TAG_MRW).x, R)], 1u)] = t;
  __syncthreads();
  // Walker w's steps are list[cur[w-1] .. cur[w]) (cur[-1] = 0); two walkers
  // per thread advance together so their DRAM reads overlap.
  constexpr int G = 2;
  for (uint32_t w0 = tid; w0 < R; w0 += G * nt) {
    uint32_t pos[G], end[G], v[G];
    uint4 rc[G];
#pragma unroll
    for (int q = 0; q < G; q++) {
      const uint32_t w = w0 + q * nt;
      pos[q] = end[q] = 0;
      v[q] = INVALID_VERTEX;
      rc[q] = make_uint4(0u, 0u, 0u, 0u);
      if (w < R) {
        pos[q] = w ? cur[w - 1] : 0u;
        end[q] = cur[w];
        for (uint32_t p = pos[q] + 1; p < end[q]; p++) {  // steps in order (a handful)
          const uint32_t x = list[p];
          uint32_t j = p;
          while (j > pos[q] && list[j - 1] > x) {
            list[j] = list[j - 1];
            j--;
          }
          list[j] = x;
        }
        v[q] = roots[w];
        if (v[q] < g.n) rc[q] = graph_record<MODE>(g, v[q]);
      }
    }
    for (;;) {
      bool any = false;
#pragma unroll
      for (int q = 0; q < G; q++) {
        if (pos[q] >= end[q]) continue;
        any = true;
        const uint32_t t = list[pos[q]++];
        src[t] = v[q];
        if (rc[q].z == 0) {
          dst[t] = INVALID_VERTEX;
          continue;
        }
        const uint32_t ry = philox4x32_10(seed, t, s_lo, s_hi, TAG_MRW).y;
        const VHdr h = record_header<MODE>(rc[q], v[q]);
        const uint32_t nv = neighbor<MODE>(g, h, mulhi_u32(ry, h.d));
        if (nv >= g.n) {
          bad = true;
          dst[t] = INVALID_VERTEX;
          continue;
        }
        dst[t] = nv;
        cnt++;
        v[q] = nv;
        rc[q] = graph_record<MODE>(g, nv);
      }
      if (!any) break;
    }
#pragma unroll
    for (int q = 0; q < G; q++)
      if (w0 + q * nt < R) roots[w0 + q * nt] = v[q];
  }
  __syncthreads();
}

__device__ __forceinline__ double ct_inf() { return __longlong_as_double(0x7FF0000000000000ll); }

// Arms event k of a walker whose vertex record is r, after time t0.
__device__ __forceinline__ void ct_arm(CtWalker &s, const uint4 &r, uint64_t seed, uint32_t s_lo,
                                       uint32_t w, double t0) {
  if (r.z == 0) {
    s.t = ct_inf();
    return;
  }
  const u32x4 b = philox4x32_10(seed, s.k, s_lo, w, TAG_MRW_CT);
  s.z = b.z;
  s.t = next_event_time(t0, exp_variate(b.x, b.y), r.z);
}

// Degree-proportional multi-RW of one sample in continuous time (select 2).
// scr: mrw_sample_scratch(R, T, 2) bytes.
template <int MODE, int NW>
__device__ void mrw_ct_cta(const DevGraph &g, uint32_t *roots, uint32_t *src, uint32_t *dst,
                           uint32_t R, uint32_t T, uint64_t seed, uint64_t sample,
                           unsigned char *scr, CtaSmem<NW> &sm, uint64_t &cnt, bool &bad) {
  const uint32_t tid = threadIdx.x, nt = blockDim.x;
  const uint32_t s_lo = (uint32_t)sample;
  const uint32_t cap = (uint32_t)mrw_ct_cap(T);
  const CtLayout lay(R, T);
  CtWalker *W = reinterpret_cast<CtWalker *>(scr);
  uint4 *rec = reinterpret_cast<uint4 *>(scr + lay.rec);
  uint32_t *first = reinterpret_cast<uint32_t *>(scr + lay.first);
  CtEvent *A = reinterpret_cast<CtEvent *>(scr + lay.ev);
  CtEvent *B = A + cap;
  uint32_t N = 0;
  bool done = false;
  double frac = 0.5, ext = 0.75;
  for (int attempt = 0; attempt < 6 && !done; attempt++) {
    uint64_t dsum = 0;
    for (uint32_t w = tid; w < R; w += nt) {
      CtWalker s{};
      s.v = roots[w];
      const uint4 r = s.v < g.n ? graph_record<MODE>(g, s.v) : make_uint4(0u, 0u, 0u, 0u);
      ct_arm(s, r, seed, s_lo, w, 0.0);
      W[w] = s;
      rec[w] = r;
      dsum += r.z;
    }
    if (tid == 0) {
      sm.n_events = 0;
      sm.overflow = 0;
    }
    dsum = cta_sum_u64(dsum, sm);
    if (dsum == 0) {
      N = 0;
      done = true;
      break;
    }
    double H = frac * (double)T / (double)dsum;
    bool overflow = false;
    for (int phase = 0; phase < 512; phase++) {
      // Every walker runs its events with time <= H; two per thread together.
      constexpr int G = 2;
      for (uint32_t w0 = tid; w0 < R; w0 += G * nt) {
        CtWalker s[G];
        uint4 r[G];
#pragma unroll
        for (int q = 0; q < G; q++) {
          const uint32_t w = w0 + q * nt;
          if (w < R) {
            s[q] = W[w];
            r[q] = rec[w];
          } else {
            s[q].t = ct_inf();
          }
        }
        for (;;) {
          bool any = false;
#pragma unroll
          for (int q = 0; q < G; q++) {
            if (!(s[q].t <= H)) continue;
            any = true;
            const uint32_t w = w0 + q * nt;
            const VHdr h = record_header<MODE>(r[q], s[q].v);
            const uint32_t nv = neighbor<MODE>(g, h, mulhi_u32(s[q].z, h.d));
            if (nv >= g.n) {  // corrupt payload: the walker stops
              bad = true;
              s[q].t = ct_inf();
              continue;
            }
            const uint32_t idx = atomicAdd(&sm.n_events, 1u);
            if (idx < cap) A[idx] = CtEvent{f64_bits(s[q].t), w, s[q].v, nv, 0u};
            r[q] = graph_record<MODE>(g, nv);
            s[q].v = nv;
            s[q].k++;
            ct_arm(s[q], r[q], seed, s_lo, w, s[q].t);
          }
          if (!any) break;
        }
#pragma unroll
        for (int q = 0; q < G; q++) {
          const uint32_t w = w0 + q * nt;
          if (w < R) {
            W[w] = s[q];
            rec[w] = r[q];
          }
        }
      }
      __syncthreads();
      N = sm.n_events;
      if (N > cap) {
        overflow = true;
        break;
      }
      if (N >= T) {
        done = true;
        break;
      }
      uint64_t rate = 0;  // total degree of the walkers that can still move
      for (uint32_t w = tid; w < R; w += nt)
        if (W[w].t < ct_inf()) rate += rec[w].z;
      rate = cta_sum_u64(rate, sm);
      if (rate == 0) {
        done = true;
        break;
      }
      const double left = (double)(T - N);
      H += (left < 64.0 ? 2.0 : ext) * left / (double)rate;
    }
    __syncthreads();
    if (!done) {  // too many events in one phase (or no convergence): smaller steps
      frac *= 0.25;
      ext *= 0.5;
      (void)overflow;
    }
  }
  if (!done) {
    bad = true;
    N = 0;
  }
  const CtEvent *E = cta_sort_events(A, B, N, sm);
  for (uint32_t r = tid; r < T; r += nt) {
    if (r < N) {
      src[r] = E[r].src;
      dst[r] = E[r].dst;
    } else {
      src[r] = INVALID_VERTEX;
      dst[r] = INVALID_VERTEX;
    }
  }
  // Final vertices: before each walker's first event past the T-th.
  for (uint32_t w = tid; w < R; w += nt) first[w] = 0xFFFFFFFFu;
  __syncthreads();
  for (uint32_t r = T + tid; r < N; r += nt) atomicMin(&first[E[r].w], r);
  __syncthreads();
  for (uint32_t w = tid; w < R; w += nt)
    roots[w] = first[w] != 0xFFFFFFFFu ? E[first[w]].src : W[w].v;
  if (tid == 0) cnt += min(N, T);
  __syncthreads();
}

// One sample of a multi-RW job with a block-level selection (0 or 2).
template <int MODE, int NW>
__device__ __forceinline__ void mrw_cta_sample(const DevGraph &g, uint32_t *roots, uint32_t *src,
                                               uint32_t *dst, uint32_t R, uint32_t T,
                                               uint32_t select, uint64_t seed, uint64_t sample,
                                               unsigned char *scr, CtaSmem<NW> &sm,
                                               uint64_t &cnt, bool &bad) {
  if (select == GRASS_SELECT_UNIFORM)
    mrw_uniform_cta<MODE, NW>(g, roots, src, dst, R, T, seed, sample,
                              reinterpret_cast<uint32_t *>(scr), sm, cnt, bad);
  else
    mrw_ct_cta<MODE, NW>(g, roots, src, dst, R, T, seed, sample, scr, sm, cnt, bad);
}

}  // namespace grass
