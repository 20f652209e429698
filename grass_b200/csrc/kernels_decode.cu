// kernels_decode.cu -- decode-only sweep: every neighbor list into CSR.
//
// Replaces the reference's two decoders for whole lists: the block-cooperative
// GlobalDecoder (GT/src/bcg.cuh:171-345, used by the grid/thread-block
// kernels at GT/src/grass.cu:529-553, 762-786) and repeated
// BCGVertex::get_vertex calls (LE/src/bcg.cuh:195-261).
//
// Work is split over the neighbor index space, not over vertices: task t
// covers neighbors [t*C, (t+1)*C) of the CSR being written, whatever
// vertices they belong to, so a hub vertex with 10^5 neighbors is spread over
// many warps instead of serialising one.  Per task a warp
//  1. finds the vertex holding the first neighbor with a 32-ary search of
//     rowptr (one coalesced probe per level);
//  2. for each round of 32 consecutive neighbors, loads the row ends and
//     records of a window of 32 vertices (coalesced), maps every lane to its
//     vertex by a shuffle binary search and takes the header by shuffle;
//  3. decodes: LE -- each neighbor is two rocks and one signed sea
//     (independent); GT -- each lane reads its own field (block head or gap)
//     and a segmented warp scan turns gaps into ids, with the running value
//     carried from round to round (and, at a task start inside a block,
//     decoded once by lane 0);
//  4. writes its 32 ids with one coalesced store.
#include <type_traits>
#include <vector>

#include "graph.h"

namespace grass {

namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr uint32_t kTaskNeighbors = 2048;  // multiple of 32

__device__ __forceinline__ VHdr shfl_hdr(const VHdr &h, int src) {
  VHdr o;
  o.P = __shfl_sync(FULL, h.P, src);
  o.v = __shfl_sync(FULL, h.v, src);
  o.d = __shfl_sync(FULL, h.d, src);
  o.bn = __shfl_sync(FULL, h.bn, src);
  o.bl = __shfl_sync(FULL, h.bl, src);
  o.om = __shfl_sync(FULL, h.om, src);
  o.fp = __shfl_sync(FULL, h.fp, src);
  o.cx = __shfl_sync(FULL, h.cx, src);
  o.a = __shfl_sync(FULL, h.a, src);
  o.b = __shfl_sync(FULL, h.b, src);
  return o;
}

// Largest v in [0, n) with rowptr[v] <= x, for x < rowptr[n].
__device__ __forceinline__ uint32_t warp_row_of(const uint64_t *rowptr, uint32_t n, uint64_t x) {
  const int lane = threadIdx.x & 31;
  uint64_t lo = 0, hi = n;  // rowptr[lo] <= x < rowptr[hi]
  while (hi - lo > 1) {
    const uint64_t step = (hi - lo + 31) / 32;
    const uint64_t p = lo + (uint64_t)(lane + 1) * step;
    const bool le = p < hi && rowptr[p] <= x;
    const uint32_t c = __popc(__ballot_sync(FULL, le));
    const uint64_t nlo = lo + (uint64_t)c * step;
    hi = min(hi, lo + (uint64_t)(c + 1) * step);
    lo = nlo;
  }
  return (uint32_t)lo;
}

// Largest v in [lo, n) with rowptr[v] <= x, one thread (rare fallback).
__device__ __forceinline__ uint32_t row_of_serial(const uint64_t *rowptr, uint32_t lo, uint32_t n,
                                                  uint64_t x) {
  uint32_t hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (rowptr[mid] <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <int MODE>
__global__ void __launch_bounds__(256) decode_all_kernel(DevGraph g, const uint64_t *rowptr,
                                                           uint32_t *cols, uint64_t E,
                                                           unsigned int *err) {
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const uint64_t tasks = (E + kTaskNeighbors - 1) / kTaskNeighbors;
  bool bad = false;
  for (uint64_t t = warp; t < tasks; t += nwarps) {
    const uint64_t g0 = t * kTaskNeighbors;
    const uint64_t g1 = min(E, g0 + kTaskNeighbors);
    uint32_t vr = warp_row_of(rowptr, g.n, g0);
    // Header of the vertex that holds the whole current round (fast path),
    // kept across rounds of the same vertex.
    uint32_t cv = 0xFFFFFFFFu;
    uint64_t cstart = 0, cend = 0;
    VHdr ch{};
    bool ch_ok = false;
    for (uint64_t r = g0; r < g1; r += 32) {  // warp-uniform
      const uint64_t gl = r + lane;
      const bool act = gl < g1;
      const uint64_t rlast = min(g1, r + 32) - 1;
      if (vr != cv) {
        cv = vr;
        cstart = rowptr[vr];
        cend = rowptr[vr + 1];
        ch_ok = false;
      }
      VHdr hk;
      uint64_t startv;
      bool far = false;
      int k = 0;
      const bool single = cstart <= r && rlast < cend;  // warp-uniform
      if (single) {
        // Fast path: the round lies inside vertex vr (most rounds of a
        // skewed graph): no window, no owner search.
        if (!ch_ok) {
          ch = header<MODE>(g, vr);
          ch_ok = true;
        }
        hk = ch;
        startv = cstart;
      } else {
        // window of vertices [vr, vr + 32): row ends and headers, one per lane
        const uint32_t wv = vr + lane;
        const uint64_t base = rowptr[vr];
        const uint64_t e = wv < g.n ? rowptr[wv + 1] : ~0ull;
        VHdr hw;
        if (wv < g.n) {
          hw = header<MODE>(g, wv);
        } else {
          hw.d = 0; hw.P = 0; hw.v = 0; hw.bn = hw.bl = hw.om = hw.fp = 0; hw.a = hw.b = hw.cx = 0;
        }
        // owner lane k: number of window rows that end at or before gl
        // (binary lifting over 31 probes gives the exact count when it is
        // below 32)
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const uint64_t ek = __shfl_sync(FULL, e, k + step - 1);
          if (ek <= gl) k += step;
        }
        // a count of 32 means gl lies beyond the window (a run of >= 32 empty
        // rows); those lanes resolve their vertex and header on their own.
        const uint64_t e31 = __shfl_sync(FULL, e, 31);
        far = act && e31 <= gl;
        const int src = far ? 0 : k;
        const uint64_t prev_e = __shfl_sync(FULL, e, src > 0 ? src - 1 : 0);
        hk = shfl_hdr(hw, src);
        startv = src == 0 ? base : prev_e;
        if (far) {
          const uint32_t v = row_of_serial(rowptr, vr + 32, g.n, gl);
          hk = header<MODE>(g, v);
          startv = rowptr[v];
        }
      }
      // each neighbor is one independent draw of one sector slot
      const uint32_t val = act ? neighbor<MODE>(g, hk, (uint32_t)(gl - startv)) : 0u;
      if (act) {
        if (val >= g.n) bad = true;
        cols[gl] = val;
      }
      // next window starts at the vertex of the round's last neighbor
      if (!single) {
        const uint32_t vlast = __shfl_sync(FULL, far ? 0xFFFFFFFFu : vr + (uint32_t)k, 31);
        if (vlast != 0xFFFFFFFFu) {
          vr = vlast;
        } else {
          const uint64_t gl31 = r + 31;
          vr = gl31 < g1 ? warp_row_of(rowptr, g.n, gl31) : vr;
        }
      }
    }
  }
  if (bad && err) atomicOr(err, 1u);
}

// ---------------------------------------------------------------------------
// Planned sweep.  The first sweep of a graph builds a plan once: vertices of
// degree >= 32 become neighbor ranges of at most 2048 (hubs are split), the
// others are grouped by floor(log2(degree)).  Then
//  * a range is decoded by one warp, one lane per chunk slot, 32 slots at a
//    time (decode_range_kernel);
//  * a small vertex is decoded by one lane, slot after slot; a warp takes 32
//    vertices of one degree class, so its lanes run for similar lengths.
constexpr uint32_t kBigDegree = 32;
#ifndef GRASS_DECODE_RANGE
#define GRASS_DECODE_RANGE 2048
#endif
constexpr uint32_t kRange = GRASS_DECODE_RANGE;  // neighbors per range item

// Sequential decoders of one vertex (one lane each), from neighbor 0.
struct LeSeq {
  const uint32_t *w;
  VHdr h;
  uint32_t c, id, L;  // chunk, index in it, its length
  uint32_t off;       // bit offset of the chunk's slot in sector A
  Sec A;

  __device__ __forceinline__ void load_chunk() {
    const uint64_t pos = slot_pos(h, c);
    A = load_sector(w, pos >> 8);
    off = (uint32_t)pos & 255u;
    L = min(h.bl, h.d - 1 - c * h.bl);
  }
  __device__ __forceinline__ void init(const uint32_t *words, const VHdr &hd) {
    w = words;
    h = hd;
    c = id = 0;
    if (h.d > 1) load_chunk();
  }
  __device__ __forceinline__ uint32_t next() {
    if (h.d == 1) return h.fp;
    const uint32_t val = le_slot_value(A, off, h, c, id, L);
    if (++id == L && c + 1 < h.bn) {  // the next chunk's left rock is this one's right rock
      c++;
      id = 0;
      load_chunk();
    }
    return val;
  }
};

struct GtSeq {
  const uint32_t *w;
  VHdr h;
  uint32_t c, id, L;  // slot, index in it, its length
  uint32_t off, x;    // bit offset of the slot in sector A; the previous value
  Sec A;

  __device__ __forceinline__ void load_chunk() {
    const uint64_t pos = slot_pos(h, c);
    A = load_sector(w, pos >> 8);
    off = (uint32_t)pos & 255u;
    L = min(h.bl, h.d - c * h.bl);
  }
  __device__ __forceinline__ void init(const uint32_t *words, const VHdr &hd) {
    w = words;
    h = hd;
    c = id = 0;
    if (h.d) load_chunk();
  }
  __device__ __forceinline__ uint32_t next() {
    if (id == 0) {
      const uint32_t hv = (uint32_t)sec1_field(A, off, h.a) + 1u;
      x = c >= h.fp ? h.v + hv : h.v - hv;
    } else {
      x += (h.b ? (uint32_t)sec1_field(A, off + (uint32_t)h.a + (id - 1) * (uint32_t)h.b, h.b)
                : 0u) + 1u;
    }
    if (++id == L && c + 1 < h.bn) {
      c++;
      id = 0;
      load_chunk();
    }
    return x;
  }
};

// Plan construction, in vertex order so that a warp of the small-vertex
// kernel takes 32 neighbouring vertices of one class (adjacent payloads).
// One warp per chunk of kPlanChunk vertices: the count pass stores, per
// chunk, the number of ranges and of vertices in each class; the host turns
// them into per-chunk cursors; the fill pass writes in order (ballot ranks).
constexpr int kCats = 6;  // ranges, then classes floor(log2(d)) = 0..4
constexpr uint32_t kPlanChunk = 1024;

__device__ __forceinline__ void plan_cat(uint32_t d, int &cat, uint32_t &w) {
  if (d >= kBigDegree) {
    cat = 0;
    w = (d + kRange - 1) / kRange;
  } else if (d) {
    cat = 1 + (31 - __clz(d));
    w = 1;
  } else {
    cat = -1;
    w = 0;
  }
}

__global__ void plan_count_kernel(const uint4 *__restrict__ recs, uint32_t n, uint32_t nchunks,
                                  uint32_t *counts) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= nchunks) return;
  uint32_t tot[kCats] = {0, 0, 0, 0, 0, 0};
  const uint32_t v0 = warp * kPlanChunk, v1 = min(n, v0 + kPlanChunk);
  for (uint32_t b = v0; b < v1; b += 32) {
    const uint32_t v = b + lane;
    int cat;
    uint32_t w;
    plan_cat(v < v1 ? recs[v].z : 0u, cat, w);
#pragma unroll
    for (int c = 0; c < kCats; c++) tot[c] += __reduce_add_sync(FULL, cat == c ? w : 0u);
  }
  if (lane < kCats) {
    uint32_t x = 0;
#pragma unroll
    for (int c = 0; c < kCats; c++)
      if (lane == c) x = tot[c];
    counts[(uint64_t)warp * kCats + lane] = x;
  }
}

__global__ void plan_fill_kernel(const uint4 *__restrict__ recs, uint32_t n, uint32_t nchunks,
                                 const unsigned long long *cursors, uint4 *big,
                                 uint32_t *small) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= nchunks) return;
  unsigned long long cur[kCats];
#pragma unroll
  for (int c = 0; c < kCats; c++) cur[c] = cursors[(uint64_t)warp * kCats + c];
  const uint32_t v0 = warp * kPlanChunk, v1 = min(n, v0 + kPlanChunk);
  const unsigned below = (1u << lane) - 1u;
  for (uint32_t b = v0; b < v1; b += 32) {
    const uint32_t v = b + lane;
    const uint32_t d = v < v1 ? recs[v].z : 0u;
    int cat;
    uint32_t w;
    plan_cat(d, cat, w);
    // ranges: exclusive scan of the range counts over the lanes
    uint32_t incl = cat == 0 ? w : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    if (cat == 0) {
      const unsigned long long p = cur[0] + incl - w;
      for (uint32_t j = 0; j < w; j++)
        big[p + j] = make_uint4(v, j * kRange, min(d, (j + 1) * kRange), 0u);
    }
    cur[0] += __shfl_sync(FULL, incl, 31);
#pragma unroll
    for (int c = 1; c < kCats; c++) {
      const unsigned m = __ballot_sync(FULL, cat == c);
      if (cat == c) small[cur[c] + __popc(m & below)] = v;
      cur[c] += __popc(m);
    }
  }
}

// ---- slot staging for the range sweep ----
// Lane 0 of a warp copies the sectors that hold each group of 32 chunk slots
// into one of the warp's D shared-memory buffers with one bulk copy
// (cp.async.bulk, completion counted on that buffer's mbarrier), D - 1 groups
// ahead of the group being decoded (D = 1: copy, then decode), and the lanes
// read their fields from shared memory, one funnel shift per field.  Every
// wait is bounded: a copy that has not landed after kStagePolls polls is
// reported (error word bit 2, GRASS_E_TIMEOUT) and the warp reads global
// memory from then on, waiting once more, bounded, for its copies in flight
// before it exits.
constexpr int kDecodeWarps = 8;          // warps per range block
constexpr uint32_t kGroupBytes = 1056;   // 32 slots lie in at most 32 sectors; + one
                                         // sector that field reads may touch
constexpr uint32_t kOutWords = 32 * 33;  // a group's neighbors (32 chunks of <= 32, + 1)
// Polls of the copy's mbarrier before the warp gives up (far beyond the
// microseconds one copy takes).
#ifndef GRASS_STAGE_POLLS
#define GRASS_STAGE_POLLS (1u << 22)
#endif
constexpr uint32_t kStagePolls = GRASS_STAGE_POLLS;
// Test hook, off in the library: with GRASS_STAGE_NEVER_COPY the barrier is
// armed for the copy's bytes but no copy is issued, so the phase never
// completes and every wait runs out -- the timeout path is exercised with
// nothing in flight.
#ifndef GRASS_STAGE_NEVER_COPY
#define GRASS_STAGE_NEVER_COPY 0
#endif

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void stage_bar_init(uint64_t *bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Copies `bytes` (a multiple of 16) from 16-byte aligned global `src` to
// shared `dst`; the barrier's current phase completes when they have landed.
__device__ __forceinline__ void stage_copy(void *dst, const void *src, uint32_t bytes,
                                           uint64_t *bar) {
  // order the lanes' earlier reads of dst before the copy's writes
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
  if (GRASS_STAGE_NEVER_COPY) return;
  asm volatile(
      "cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Waits for phase `parity` of the barrier, at most kStagePolls polls.
__device__ __forceinline__ bool stage_wait(uint64_t *bar, uint32_t parity) {
  for (uint32_t i = 0; i < kStagePolls; i++) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

// Metadata of the 32 range items a warp takes at a time (lane k loads item k's
// record and row start once; the group loop reads them back by broadcast).
struct RangeMeta {
  uint4 rec[32];
  uint64_t base[32];
  uint32_t v[32], i0[32], i1[32];
};

// Shared memory of one range warp, in a block of its own that starts on a
// 128-byte boundary: DEPTH staging buffers (each a multiple of 16 bytes, as
// cp.async.bulk requires of its destination), the group's decoded neighbors,
// the item metadata, then the buffers' mbarriers (8-byte aligned).
template <int DEPTH>  // DEPTH 0: no staging buffers, no barriers
struct WarpSmem {
  static constexpr uint32_t stage_off() { return 0; }
  static constexpr uint32_t out_off() { return DEPTH * kGroupBytes; }
  static constexpr uint32_t meta_off() { return out_off() + kOutWords * 4; }
  static constexpr uint32_t bar_off() { return meta_off() + (uint32_t)sizeof(RangeMeta); }
  static constexpr uint32_t bytes() { return (bar_off() + DEPTH * 8 + 127) / 128 * 128; }
};
static_assert(kGroupBytes % 16 == 0 && (kOutWords * 4) % 16 == 0 && sizeof(RangeMeta) % 16 == 0,
              "staging alignment");

// Range sweep on the device layout (GT or LE): one lane per chunk slot.  A
// warp takes 32 range items at a time: lane k loads item k's record and row
// start, and a scan over the lanes numbers the items' groups of 32 slots
// 0 .. total-1 in item order.  The warp then walks that sequence: each lane
// decodes its chunk's neighbors into shared memory, and the warp writes the
// group's neighbors to the CSR with coalesced stores.  DEPTH 0 (the default)
// reads the slot words from global memory through L1; DEPTH 1, 2 or 4 stages
// each group's sectors in shared memory DEPTH - 1 groups ahead (across item
// boundaries, see above).  Measured on R-MAT s22 ef32, the unstaged sweep is
// the fastest: 7 % (LE) and 23 % (GT) faster than staging at depth 1.
template <int MODE, int DEPTH>
__global__ void __launch_bounds__(256) decode_range_kernel(DevGraph g, const uint64_t *rowptr,
                                                           uint32_t *cols,
                                                           const uint4 *__restrict__ items,
                                                           uint64_t nitems, unsigned int *err) {
  extern __shared__ __align__(128) unsigned char le_smem[];
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  using WS = WarpSmem<DEPTH>;
  static_assert(WS::bytes() % 128 == 0 && WS::bar_off() % 8 == 0 && WS::meta_off() % 16 == 0,
                "warp block alignment");
  unsigned char *mine = le_smem + (threadIdx.x >> 5) * WS::bytes();
  unsigned char *stage = mine + WS::stage_off();
  uint32_t *out = reinterpret_cast<uint32_t *>(mine + WS::out_off());
  RangeMeta &m = *reinterpret_cast<RangeMeta *>(mine + WS::meta_off());
  uint64_t *bars = reinterpret_cast<uint64_t *>(mine + WS::bar_off());
  uint32_t phase = 0;    // bit b: parity of buffer b's next completion
  uint32_t pending = 0;  // bit b: buffer b has a copy issued and not yet waited for
  constexpr uint32_t D = DEPTH > 0 ? DEPTH : 1;  // ring size (DEPTH 0: unstaged)
  bool stage_ok = DEPTH > 0;
  if (lane < DEPTH) stage_bar_init(bars + lane);
  __syncwarp();
  bool bad = false;
  for (uint64_t tb = warp * 32; tb < nitems; tb += nwarps * 32) {
    // lane k: item tb + k, its slots [c0, c1] and their group count
    const uint64_t t = tb + lane;
    uint32_t c0 = 0, c1 = 0, ng = 0;
    if (t < nitems) {
      const uint4 it = items[t];
      const uint4 r = graph_record<MODE>(g, it.x);
      const VHdr h = record_header<MODE>(r, it.x);
      m.rec[lane] = r;
      m.v[lane] = it.x;
      m.base[lane] = rowptr[it.x];
      m.i0[lane] = it.y;
      m.i1[lane] = it.z;
      // slot of neighbor i: i / T (LE: the last neighbor is slot C-1's right rock)
      const uint32_t last = h.d - 1;
      c0 = MODE == 0 || it.y < last ? div_small(it.y, h.bl) : h.bn - 1;
      c1 = MODE == 0 || it.z - 1 < last ? div_small(it.z - 1, h.bl) : h.bn - 1;
      ng = (c1 - c0) / 32 + 1;
    }
    uint32_t incl = ng;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t excl = incl - ng;  // this item's first group in the sequence
    const uint32_t total = __shfl_sync(FULL, incl, 31);
    __syncwarp();
    // the item holding group s of the sequence (items with groups come first)
    auto item_of = [&](uint32_t s) -> int {
      return __popc(__ballot_sync(FULL, ng > 0 && excl <= s)) - 1;
    };
    // sectors [qa, qb] of group s
    auto group_sectors = [&](uint32_t s, uint64_t &qa, uint64_t &qb) {
      const int k = item_of(s);
      const uint32_t j = s - __shfl_sync(FULL, excl, k);
      const uint32_t kc0 = __shfl_sync(FULL, c0, k), kc1 = __shfl_sync(FULL, c1, k);
      const VHdr hk = record_header<MODE>(m.rec[k], m.v[k]);
      const uint32_t ca = kc0 + 32 * j, cz = min(kc1, ca + 31);
      qa = slot_pos(hk, ca) >> 8;
      qb = slot_pos(hk, cz) >> 8;
    };
    auto issue = [&](uint32_t s) {
      if (DEPTH == 0 || !stage_ok) return;
      const uint32_t b = s % D;
      uint64_t qa, qb;
      group_sectors(s, qa, qb);
      if (lane == 0)
        stage_copy(stage + b * kGroupBytes, g.words + qa * 8, (uint32_t)(qb - qa + 1) * 32u,
                   bars + b);
      pending |= 1u << b;
    };
    if constexpr (DEPTH > 1)
      for (uint32_t s = 0; s + 1 < (uint32_t)DEPTH && s < total; s++) issue(s);
    int kcur = -1;
    VHdr h;
    uint64_t base = 0;
    uint32_t i0 = 0, i1 = 0, kc0 = 0, kc1 = 0, kex = 0;
    for (uint32_t s = 0; s < total; s++) {  // warp-uniform
      if (DEPTH > 0 && s + DEPTH - 1 < total) issue(s + DEPTH - 1);
      const int k = item_of(s);
      if (k != kcur) {  // the next item: its header and range from the metadata
        kcur = k;
        h = record_header<MODE>(m.rec[k], m.v[k]);
        base = m.base[k];
        i0 = m.i0[k];
        i1 = m.i1[k];
        kc0 = __shfl_sync(FULL, c0, k);
        kc1 = __shfl_sync(FULL, c1, k);
        kex = __shfl_sync(FULL, excl, k);
      }
      const uint32_t T = h.bl, last = h.d - 1, j = s - kex;
      bool staged = false;
      const uint32_t b = s % D;
      if (DEPTH > 0 && stage_ok) {
        if (__all_sync(FULL, stage_wait(bars + b, (phase >> b) & 1u))) {
          phase ^= 1u << b;
          pending &= ~(1u << b);
          staged = true;
        } else {  // the copy did not land in time: report, go on from global memory
          if (lane == 0 && err) atomicOr(err, 2u);
          stage_ok = false;
        }
      }
      const uint32_t cg = kc0 + 32 * j, c = cg + lane;
      if (c <= kc1) {
        const uint64_t pos = slot_pos(h, c);
        // the slot's sector as words: from the staged group, or (after a
        // timeout) from global memory
        const uint32_t *w;
        if (staged) {
          const uint64_t qa = slot_pos(h, cg) >> 8;
          w = reinterpret_cast<const uint32_t *>(stage + b * kGroupBytes + ((pos >> 8) - qa) * 32u);
        } else {
          w = g.words + (pos >> 8) * 8;
        }
        if constexpr (MODE == 0) {
          gt_slot_decode_w(w, (uint32_t)pos & 255u, h, c, min(T, h.d - c * T), out + (c - cg) * T);
        } else {  // the last chunk also holds neighbor d-1, its right rock
          le_slot_decode_w(w, (uint32_t)pos & 255u, h, c, min(T, last - c * T), c + 1 == h.bn,
                           out + (c - cg) * T);
        }
      }
      __syncwarp();
      const uint32_t nb0 = cg * T, nhi = cg + 32 >= h.bn ? h.d : (cg + 32) * T;
      const uint32_t lo = max(i0, nb0), hi = min(i1, nhi);
      for (uint32_t q = lo + lane; q < hi; q += 32) {
        const uint32_t val = out[q - nb0];
        bad |= val >= g.n;
        cols[base + q] = val;
      }
      __syncwarp();  // the group's buffers are free for the next group
    }
    __syncwarp();  // the metadata is free for the next batch
  }
  // copies still in flight after a timeout: one more bounded wait each
  for (int b = 0; b < DEPTH; b++)
    if ((pending >> b) & 1u) stage_wait(bars + b, (phase >> b) & 1u);
  if (bad && err) atomicOr(err, 1u);
}

// ---- the flat sweep (the default) ----
// A warp takes one item of the flat plan: a run of consecutive vertices
// [v0, v1) (i1 == 0), or one vertex's neighbor range [i0, i1) (hubs, degree
// >= kRange).  The item's output is one contiguous stretch of the CSR, and
// its chunk slots, taken in vertex order, fill it in order.  So the warp
// walks the item 32 vertices at a time (lane k loads vertex k's record and
// counts its slots), numbers their slots by a warp scan, and decodes them 32
// at a time, one slot per lane, whatever vertex each belongs to: a group of
// 32 slots is a contiguous stretch of at most 32 * 33 neighbors, decoded into
// shared memory and written with coalesced stores.  A lane reads its slot's
// fields as 32-bit words from global memory through L1 (one funnel shift per
// field); measured faster than loading the sector into registers and reading
// the fields in order from there (LE 1.00 against 1.04 ms, GT 1.16 against
// 1.43 ms on R-MAT s22 ef32).  LE vertices of degree 1 count as one slot (the
// neighbor is in the record).
constexpr uint32_t kFlatHub = kRange;  // degree from which a vertex is split into ranges

// Resident 256-thread blocks per SM: 4 (64 registers, no spill; 4 x 33 KB of
// shared memory).  Unbounded, the LE kernel took 80 registers (3 blocks) and
// ran 1.08 ms against 0.94 ms at 4 (GT: 74 registers, 1.43 against 1.17 ms)
// on R-MAT s22 ef32.
#ifndef GRASS_DECODE_FLAT_MIN_BLOCKS
#define GRASS_DECODE_FLAT_MIN_BLOCKS 4
#endif

template <int MODE>
__global__ void __launch_bounds__(256, GRASS_DECODE_FLAT_MIN_BLOCKS) decode_flat_kernel(DevGraph g, const uint64_t *rowptr,
                                                          uint32_t *cols,
                                                          const uint4 *__restrict__ items,
                                                          uint64_t nitems, unsigned int *err) {
  __shared__ __align__(16) uint32_t out_all[8][kOutWords];
  uint32_t *out = out_all[threadIdx.x >> 5];
  const int lane = threadIdx.x & 31;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  bool bad = false;
  for (uint64_t t = warp; t < nitems; t += nwarps) {
    const uint4 it = items[t];
    const bool run = it.w == 0;
    const uint32_t v0 = it.x, v1 = run ? it.y : it.x + 1;
    for (uint32_t vb = v0; vb < v1; vb += 32) {
      // lane k: vertex vb + k, its slots [c0, c0 + ns) and first output position
      const uint32_t v = vb + lane;
      const bool vok = v < v1;
      uint4 r = make_uint4(0, 0, 0, 0);
      uint32_t c0 = 0, ns = 0;
      uint64_t ob = 0;  // output position of the vertex's slot c0's first neighbor
      if (vok) {
        r = graph_record<MODE>(g, v);
        const VHdr h = record_header<MODE>(r, v);
        const uint32_t i0 = run ? 0u : it.z, i1 = run ? h.d : it.w;
        if (MODE == 1 && h.d == 1) {
          ns = 1;
        } else if (h.d) {
          const uint32_t last = h.d - 1;
          c0 = MODE == 0 || i0 < last ? div_small(i0, h.bl) : h.bn - 1;
          const uint32_t c1 = MODE == 0 || i1 - 1 < last ? div_small(i1 - 1, h.bl) : h.bn - 1;
          ns = c1 - c0 + 1;
        }
        ob = rowptr[v] + (uint64_t)c0 * h.bl;
      }
      uint32_t sincl = ns;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(FULL, sincl, o);
        if (lane >= o) sincl += y;
      }
      const uint32_t sexcl = sincl - ns, stot = __shfl_sync(FULL, sincl, 31);
      // the item's stored stretch: [lo, hi) of the CSR
      const uint64_t v_lo = run ? __shfl_sync(FULL, ob, 0) : rowptr[v0] + it.z;
      const uint64_t v_hi = run ? rowptr[min(v1, vb + 32)] : rowptr[v0] + it.w;
      for (uint32_t sg = 0; sg < stot; sg += 32) {  // warp-uniform
        const uint32_t sl = sg + lane;
        // the lane's vertex: the last k with sexcl_k <= sl
        int k = 0;
#pragma unroll
        for (int step = 16; step > 0; step >>= 1) {
          const uint32_t e = __shfl_sync(FULL, sexcl, k + step);
          if (k + step < 32 && e <= sl) k += step;
        }
        const uint32_t kx = __shfl_sync(FULL, r.x, k), ky = __shfl_sync(FULL, r.y, k);
        const uint32_t kz = __shfl_sync(FULL, r.z, k), kw = __shfl_sync(FULL, r.w, k);
        const uint32_t kc0 = __shfl_sync(FULL, c0, k), kse = __shfl_sync(FULL, sexcl, k);
        const uint64_t kob = __shfl_sync(FULL, ob, k);
        const bool act = sl < stot;
        const VHdr h = record_header<MODE>(make_uint4(kx, ky, kz, kw), vb + (uint32_t)k);
        const uint32_t c = kc0 + (sl - kse);
        const uint64_t pos0 = kob + (uint64_t)(sl - kse) * h.bl;  // slot's first output position
        const uint64_t g_lo = __shfl_sync(FULL, pos0, 0);
        // the slot's neighbors: GT min(T, d - cT); LE min(T, d-1-cT) (+ the right
        // rock in the last slot); LE degree 1: the record's neighbor
        uint32_t len = 0;
        if (act) {
          if (MODE == 1 && h.d == 1) {
            len = 1;
            out[pos0 - g_lo] = h.fp;
          } else {
            const uint64_t p = slot_pos(h, c);
            const uint32_t *w = g.words + (p >> 8) * 8;
            if constexpr (MODE == 0) {
              len = min(h.bl, h.d - c * h.bl);
              gt_slot_decode_w(w, (uint32_t)p & 255u, h, c, len, out + (pos0 - g_lo));
            } else {
              const uint32_t L = min(h.bl, h.d - 1 - c * h.bl);
              const bool right = c + 1 == h.bn;
              le_slot_decode_w(w, (uint32_t)p & 255u, h, c, L, right, out + (pos0 - g_lo));
              len = L + (right ? 1u : 0u);
            }
          }
        }
        const uint64_t g_hi = __reduce_max_sync(FULL, act ? (uint32_t)(pos0 - g_lo) + len : 0u) + g_lo;
        __syncwarp();
        const uint64_t lo = max(g_lo, v_lo), hi = min(g_hi, v_hi);
        for (uint64_t q = lo + lane; q < hi; q += 32) {
          const uint32_t val = out[q - g_lo];
          bad |= val >= g.n;
          cols[q] = val;
        }
        __syncwarp();  // the group's buffer is free for the next group
      }
    }
  }
  if (bad && err) atomicOr(err, 1u);
}

// Flat plan: items in vertex order.  One warp per chunk of kPlanChunk
// vertices.  A vertex of degree >= kFlatHub becomes ceil(d / kRange) range
// items (v, v + 1, i0, i1); the others form runs, a run starting at the
// chunk's first vertex, after a hub, and wherever the chunk's running degree
// sum crosses a multiple of kRange.  Runs get (v0, 0, 0, 0) here; their end
// is the next item's first vertex (flat_plan_link_kernel).
template <bool FILL>
__global__ void flat_plan_kernel(const uint4 *__restrict__ recs, uint32_t n, uint32_t nchunks,
                                 uint32_t *counts, const unsigned long long *cursors,
                                 uint4 *items) {
  const int lane = threadIdx.x & 31;
  const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (warp >= nchunks) return;
  const uint32_t v0 = warp * kPlanChunk, v1 = min(n, v0 + kPlanChunk);
  unsigned long long cur = FILL ? cursors[warp] : 0ull;
  uint32_t tot = 0;
  uint64_t carry = 0;       // degree sum of the chunk's vertices before this sub-chunk
  bool prev_hub = true;     // (the chunk's first vertex starts a run)
  uint64_t prev_win = 0;
  for (uint32_t b = v0; b < v1; b += 32) {
    const uint32_t v = b + lane;
    const uint32_t d = v < v1 ? recs[v].z : 0u;
    const bool hub = v < v1 && d >= kFlatHub;
    uint64_t incl = d;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint64_t y = __shfl_up_sync(FULL, incl, o);
      if (lane >= o) incl += y;
    }
    const uint64_t pre = carry + incl - d;  // chunk degree sum before v
    const uint64_t win = pre / kRange;
    const uint32_t hub_up = __shfl_up_sync(FULL, (uint32_t)hub, 1);
    const bool ph = lane ? hub_up != 0u : prev_hub;
    const uint64_t pw_up = __shfl_up_sync(FULL, win, 1);
    const uint64_t pw = lane ? pw_up : prev_win;
    const bool start = v < v1 && !hub && (ph || win != pw);
    const uint32_t w_items = hub ? (d + kRange - 1) / kRange : (start ? 1u : 0u);
    uint32_t wi = w_items;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(FULL, wi, o);
      if (lane >= o) wi += y;
    }
    if (FILL && w_items) {
      const unsigned long long at = cur + wi - w_items;
      if (hub) {
        for (uint32_t j = 0; j < w_items; j++)
          items[at + j] = make_uint4(v, v + 1, j * kRange, min(d, (j + 1) * kRange));
      } else {
        items[at] = make_uint4(v, 0u, 0u, 0u);
      }
    }
    const uint32_t wsum = __shfl_sync(FULL, wi, 31);
    cur += wsum;
    tot += wsum;
    carry += __shfl_sync(FULL, incl, 31);
    prev_hub = __shfl_sync(FULL, (uint32_t)hub, 31) != 0u;
    prev_win = __shfl_sync(FULL, win, 31);
  }
  if (!FILL && lane == 0) counts[warp] = tot;
}

// A run ends where the next item starts (or at n).
__global__ void flat_plan_link_kernel(uint4 *items, uint64_t nitems, uint32_t n) {
  const uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  if (k >= nitems) return;
  if (items[k].w == 0) items[k].y = k + 1 < nitems ? items[k + 1].x : n;
}

template <int MODE>
__global__ void __launch_bounds__(256) decode_small_kernel(DevGraph g, const uint64_t *rowptr,
                                                             uint32_t *cols,
                                                             const uint32_t *__restrict__ verts,
                                                             uint64_t nv, unsigned int *err) {
  bool bad = false;
  const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q0 = (uint64_t)blockIdx.x * blockDim.x; q0 < nv; q0 += nt) {
    const uint64_t q = q0 + threadIdx.x;
    uint32_t d = 0;
    uint32_t *out = nullptr;
    std::conditional_t<MODE == 0, GtSeq, LeSeq> st;
    if (q < nv) {
      const uint32_t v = verts[q];
      const VHdr h = header<MODE>(g, v);
      d = h.d;
      out = cols + rowptr[v];
      st.init(g.words, h);
    }
    for (uint32_t k = 0; k < d; k++) {
      const uint32_t val = st.next();
      bad |= val >= g.n;
      out[k] = val;
    }
  }
  if (bad && err) atomicOr(err, 1u);
}

}  // namespace

static void launch_plan_kernels(const grass_graph *g, const uint64_t *rowptr, uint32_t *cols,
                                unsigned int *err, cudaStream_t s);

template <int MODE, int DEPTH>
static void launch_range(const DevGraph &v, const uint64_t *rowptr, uint32_t *cols,
                         const grass_graph *g, unsigned grid, unsigned int *err, cudaStream_t s) {
  const uint32_t smem = kDecodeWarps * WarpSmem<DEPTH>::bytes();
  static std::once_flag once;  // opt in to more than 48 KB of dynamic shared memory
  std::call_once(once, [&] {
    cudaFuncSetAttribute(decode_range_kernel<MODE, DEPTH>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  decode_range_kernel<MODE, DEPTH><<<grid, 32 * kDecodeWarps, smem, s>>>(
      v, rowptr, cols, g->d_plan_big, g->plan_nbig, err);
}

template <int MODE>
static void launch_range_depth(const DevGraph &v, const uint64_t *rowptr, uint32_t *cols,
                               const grass_graph *g, unsigned grid, unsigned int *err,
                               cudaStream_t s) {
  switch (g->tuning.decode_stage_depth) {
    case 1: launch_range<MODE, 1>(v, rowptr, cols, g, grid, err, s); break;
    case 2: launch_range<MODE, 2>(v, rowptr, cols, g, grid, err, s); break;
    case 4: launch_range<MODE, 4>(v, rowptr, cols, g, grid, err, s); break;
    default: launch_range<MODE, 0>(v, rowptr, cols, g, grid, err, s);  // unstaged
  }
}

// Builds the flat plan (once) on stream s.
static int build_flat_plan(const grass_graph *g, cudaStream_t s) {
  const uint32_t n = (uint32_t)g->info.n;
  const uint32_t nchunks = (n + kPlanChunk - 1) / kPlanChunk;
  const unsigned pgrid = (nchunks + 7) / 8;  // 8 warps (chunks) per block
  uint32_t *cnt = nullptr;
  unsigned long long *cur = nullptr;
  GRASS_CUDA(cudaMalloc(&cnt, (uint64_t)nchunks * sizeof(uint32_t)));
  cudaError_t e = cudaMalloc(&cur, (uint64_t)nchunks * sizeof(unsigned long long));
  std::vector<uint32_t> hc(nchunks);
  std::vector<unsigned long long> hcur(nchunks);
  uint64_t tot = 0;
  if (e == cudaSuccess) {
    flat_plan_kernel<false><<<pgrid, 256, 0, s>>>(g->d_recs, n, nchunks, cnt, nullptr, nullptr);
    count_launch();
    e = cudaMemcpyAsync(hc.data(), cnt, hc.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) {
    for (uint32_t ch = 0; ch < nchunks; ch++) {
      hcur[ch] = tot;
      tot += hc[ch];
    }
    e = cudaMalloc(&g->d_plan_flat, std::max<uint64_t>(tot, 1) * sizeof(uint4));
  }
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(cur, hcur.data(), hcur.size() * sizeof(unsigned long long),
                        cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) {
    flat_plan_kernel<true><<<pgrid, 256, 0, s>>>(g->d_recs, n, nchunks, nullptr, cur,
                                                 g->d_plan_flat);
    count_launch();
    if (tot) {
      flat_plan_link_kernel<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(g->d_plan_flat, tot, n);
      count_launch();
    }
    e = cudaStreamSynchronize(s);
  }
  cudaFree(cnt);
  cudaFree(cur);
  if (e != cudaSuccess) {
    cudaFree(g->d_plan_flat);
    g->d_plan_flat = nullptr;
    return cuda_fail(e, "flat decode plan build");
  }
  g->plan_nflat = tot;
  g->plan_flat_ok = true;
  return GRASS_OK;
}

static void launch_flat(const grass_graph *g, const uint64_t *rowptr, uint32_t *cols,
                        unsigned int *err, cudaStream_t s) {
  if (!g->plan_nflat) return;
  const DevGraph v = g->view();
  const unsigned grid = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>((g->plan_nflat + 7) / 8, (uint64_t)sm_count(g->device) * 8));
  if (g->mode == GRASS_MODE_GT)
    decode_flat_kernel<0><<<grid, 256, 0, s>>>(v, rowptr, cols, g->d_plan_flat, g->plan_nflat, err);
  else
    decode_flat_kernel<1><<<grid, 256, 0, s>>>(v, rowptr, cols, g->d_plan_flat, g->plan_nflat, err);
  count_launch();
}

int launch_decode_planned(const grass_graph *g, const uint64_t *rowptr, uint32_t *cols,
                          unsigned int *err, cudaStream_t s) {
  const uint32_t n = (uint32_t)g->info.n;
  if (!g->info.num_edges) return GRASS_OK;
  if (g->tuning.decode_stage_depth == 0) {  // the flat sweep
    {
      std::lock_guard<std::mutex> lk(g->plan_mu);
      if (!g->plan_flat_ok) {
        const int rc = build_flat_plan(g, s);
        if (rc) return rc;
      }
    }
    launch_flat(g, rowptr, cols, err, s);
    return GRASS_OK;
  }
  {
    std::lock_guard<std::mutex> lk(g->plan_mu);
    if (!g->plan_ok) {
      const uint32_t nchunks = (n + kPlanChunk - 1) / kPlanChunk;
      const unsigned pgrid = (nchunks + 7) / 8;  // 8 warps (chunks) per block
      uint32_t *cnt = nullptr;
      unsigned long long *cur = nullptr;
      GRASS_CUDA(cudaMalloc(&cnt, (uint64_t)nchunks * kCats * sizeof(uint32_t)));
      cudaError_t e = cudaMalloc(&cur, (uint64_t)nchunks * kCats * sizeof(unsigned long long));
      if (e != cudaSuccess) {
        cudaFree(cnt);
        return cuda_fail(e, "decode plan scratch");
      }
      plan_count_kernel<<<pgrid, 256>>>(g->d_recs, n, nchunks, cnt);
      count_launch();
      std::vector<uint32_t> hc((uint64_t)nchunks * kCats);
      std::vector<unsigned long long> hcur(hc.size());
      e = cudaMemcpy(hc.data(), cnt, hc.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost);
      // cursors: ranges in chunk order; the classes back to back, each in chunk order
      uint64_t tot[kCats] = {0, 0, 0, 0, 0, 0};
      for (uint64_t k = 0; k < hc.size(); k++) tot[k % kCats] += hc[k];
      uint64_t base[kCats] = {0, 0, 0, 0, 0, 0};
      for (int c = 2; c < kCats; c++) base[c] = base[c - 1] + tot[c - 1];
      for (uint32_t ch = 0; ch < nchunks; ch++)
        for (int c = 0; c < kCats; c++) {
          hcur[(uint64_t)ch * kCats + c] = base[c];
          base[c] += hc[(uint64_t)ch * kCats + c];
        }
      g->plan_nbig = tot[0];
      g->plan_nsmall = 0;
      for (int c = 1; c < kCats; c++) g->plan_nsmall += tot[c];
      if (e == cudaSuccess)
        e = cudaMalloc(&g->d_plan_big, std::max<uint64_t>(g->plan_nbig, 1) * sizeof(uint4));
      if (e == cudaSuccess)
        e = cudaMalloc(&g->d_plan_small, std::max<uint64_t>(g->plan_nsmall, 1) * sizeof(uint32_t));
      if (e == cudaSuccess)
        e = cudaMemcpy(cur, hcur.data(), hcur.size() * sizeof(unsigned long long),
                       cudaMemcpyHostToDevice);
      if (e == cudaSuccess) {
        plan_fill_kernel<<<pgrid, 256>>>(g->d_recs, n, nchunks, cur, g->d_plan_big,
                                         g->d_plan_small);
        count_launch();
        e = cudaDeviceSynchronize();
      }
      cudaFree(cnt);
      cudaFree(cur);
      if (e != cudaSuccess) {
        cudaFree(g->d_plan_big);
        cudaFree(g->d_plan_small);
        g->d_plan_big = nullptr;
        g->d_plan_small = nullptr;
        return cuda_fail(e, "decode plan build");
      }
      g->plan_ok = true;
    }
  }
  launch_plan_kernels(g, rowptr, cols, err, s);
  return GRASS_OK;
}

bool launch_decode_if_planned(const grass_graph *g, const uint64_t *rowptr, uint32_t *cols,
                              unsigned int *err, cudaStream_t s) {
  const bool flat = g->tuning.decode_stage_depth == 0;
  {
    std::lock_guard<std::mutex> lk(g->plan_mu);
    if (flat ? !g->plan_flat_ok : !g->plan_ok) return false;
  }
  if (!g->info.num_edges) return true;
  if (flat) launch_flat(g, rowptr, cols, err, s);
  else launch_plan_kernels(g, rowptr, cols, err, s);
  return true;
}

// The range and small-vertex sweeps of a built plan (launches only).
static void launch_plan_kernels(const grass_graph *g, const uint64_t *rowptr, uint32_t *cols,
                                unsigned int *err, cudaStream_t s) {
  const int dev = g->device;
  const DevGraph v = g->view();
  const int per_sm = 8;
  if (g->plan_nbig) {
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((g->plan_nbig + 7) / 8, (uint64_t)sm_count(dev) * per_sm));
    if (g->mode == GRASS_MODE_GT) launch_range_depth<0>(v, rowptr, cols, g, grid, err, s);
    else launch_range_depth<1>(v, rowptr, cols, g, grid, err, s);
    count_launch();
  }
  if (g->plan_nsmall) {
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((g->plan_nsmall + 255) / 256, (uint64_t)sm_count(dev) * per_sm));
    if (g->mode == GRASS_MODE_GT)
      decode_small_kernel<0><<<grid, 256, 0, s>>>(v, rowptr, cols, g->d_plan_small,
                                                  g->plan_nsmall, err);
    else
      decode_small_kernel<1><<<grid, 256, 0, s>>>(v, rowptr, cols, g->d_plan_small,
                                                  g->plan_nsmall, err);
    count_launch();
  }
}

void launch_decode_all(const DevGraph &g, const uint64_t *rowptr, uint32_t *cols, uint64_t E,
                       unsigned int *err, cudaStream_t s) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (!E) return;
  const uint64_t tasks = (E + kTaskNeighbors - 1) / kTaskNeighbors;
  const uint64_t blocks_needed = (tasks + 7) / 8;
  const unsigned grid = (unsigned)std::max<uint64_t>(
      1, std::min<uint64_t>(blocks_needed, (uint64_t)sm_count(dev) * 8));
  if (g.mode == GRASS_MODE_GT)
    decode_all_kernel<0><<<grid, 256, 0, s>>>(g, rowptr, cols, E, err);
  else
    decode_all_kernel<1><<<grid, 256, 0, s>>>(g, rowptr, cols, E, err);
  count_launch();
}

}  // namespace grass
