// sample_warp.cuh -- warp-level sampling routines shared by the standalone
// multi-RW kernel and the batched persistent kernel.  Each routine is run by
// all 32 lanes of one warp and needs at most the warp's own shared-memory
// slot (SmemHdr), so a persistent warp can pick up any job type from a work
// queue.
#pragma once
#include "device_common.cuh"

namespace grass {

constexpr unsigned kFull = 0xFFFFFFFFu;

__device__ __forceinline__ void path_store(uint32_t *paths, int layout, uint64_t W, uint32_t L,
                                           uint64_t w, uint32_t s, uint32_t v) {
  if (layout == GRASS_LAYOUT_WALK_MAJOR) store_out_u32(paths + w * (uint64_t)(L + 1) + s, v);
  else store_out_u32(paths + (uint64_t)s * W + w, v);
}

// Random walk of walkers [b, e) of a job of W walkers (starts[0..W)), DEPTH
// walkers per lane per pass.  Same draws as rw_kernel / rw_gt_kernel:
// walker w uses Philox(seed; step>>2, w0+w, .., TAG_RW).
template <int MODE, int DEPTH>
__device__ __forceinline__ void rw_warp(const DevGraph &g, const uint32_t *starts, uint64_t W,
                                        uint32_t L, uint64_t seed, uint64_t w0, int layout,
                                        uint32_t *paths, uint64_t b, uint64_t e, uint64_t &cnt,
                                        bool &bad) {
  const int lane = threadIdx.x & 31;
  for (uint64_t wb = b; wb < e; wb += 32 * DEPTH) {  // warp-uniform
    uint32_t v[DEPTH];
    u32x4 r[DEPTH];
#pragma unroll
    for (int k = 0; k < DEPTH; k++) {
      const uint64_t w = wb + (uint64_t)k * 32 + lane;
      v[k] = INVALID_VERTEX;
      r[k] = u32x4{0, 0, 0, 0};
      if (w < e) {
        const uint32_t s0 = starts[w];
        path_store(paths, layout, W, L, w, 0, s0);
        v[k] = s0 < g.n ? s0 : INVALID_VERTEX;
      }
    }
    for (uint32_t s = 0; s < L; s++) {
#pragma unroll
      for (int k = 0; k < DEPTH; k++) {
        const uint64_t w = wb + (uint64_t)k * 32 + lane;
        if ((s & 3) == 0) {
          const uint64_t id = w0 + w;
          r[k] = philox4x32_10(seed, s >> 2, (uint32_t)id, (uint32_t)(id >> 32), TAG_RW);
        }
        bool active = v[k] != INVALID_VERTEX;
        uint32_t nv = INVALID_VERTEX;
        if (active) {
          const VHdr h = header<MODE>(g, v[k]);
          if (h.d == 0) {
            active = false;
            v[k] = INVALID_VERTEX;
          } else {
            nv = neighbor<MODE>(g, h, mulhi_u32(pick(r[k], s & 3), h.d));
          }
        }
        if (active) {
          if (nv >= g.n) {
            bad = true;
            v[k] = INVALID_VERTEX;
          } else {
            v[k] = nv;
            cnt++;
          }
        }
        if (w < e) path_store(paths, layout, W, L, w, s + 1, v[k]);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// k-hop of one seed (KHopApp, GT/src/apps/khop/khop.cu:1-79, with runtime
// fanouts).  For each hop the frontier is taken in chunks of 32 transits:
// lane p decodes the header of transit p into the warp's shared-memory slot,
// then the chunk's f*32 draws are spread over the lanes.

struct KhopArgs {
  uint32_t hops;
  uint32_t fan[GRASS_MAX_HOPS];
  uint64_t width[GRASS_MAX_HOPS];  // prod_{j<=h} fan[j]
  uint32_t *out[GRASS_MAX_HOPS];
  uint64_t seed;
};

struct SmemHdr {
  uint64_t P[32];
  uint32_t v[32], d[32], bn[32], bl[32], om[32], fp[32];
  int a[32], b[32], cx[32];
  uint64_t ob[32];  // k-hop: first output slot of transit i (parent index * fanout)
  __device__ __forceinline__ void put(int i, const VHdr &h) {
    P[i] = h.P; v[i] = h.v; d[i] = h.d; bn[i] = h.bn; bl[i] = h.bl; om[i] = h.om; fp[i] = h.fp;
    a[i] = h.a; b[i] = h.b; cx[i] = h.cx;
  }
  __device__ __forceinline__ VHdr get(int i) const {
    VHdr h;
    h.P = P[i]; h.v = v[i]; h.d = d[i]; h.bn = bn[i]; h.bl = bl[i]; h.om = om[i]; h.fp = fp[i];
    h.a = a[i]; h.b = b[i]; h.cx = cx[i];
    return h;
  }
};

// Word k (0..3) of a Philox block held as four values.
__device__ __forceinline__ uint32_t pick4(uint32_t x, uint32_t y, uint32_t z, uint32_t w, int k) {
  return k == 0 ? x : k == 1 ? y : k == 2 ? z : w;
}

// Per-lane staging of a k-hop draw's slot sector: 32 bytes copied by two
// 16-byte cp.async (no registers held while the copy is in flight), in a
// buffer of kDrawBufWords words (the sector, and the words that field reads
// past its end may touch; a multiple of 16 bytes).
constexpr uint32_t kDrawBufWords = 12;
__device__ __forceinline__ void draw_copy(uint32_t *dst, const uint32_t *words, uint64_t sector) {
  const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
  const uint32_t *src = words + sector * 8;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d + 16), "l"(src + 4) : "memory");
}
__device__ __forceinline__ void draw_copy_wait() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

// A GT neighbor from its slot's words (slot at bit off): the head, then id gaps.
__device__ __forceinline__ uint32_t gt_draw_w(const uint32_t *w, uint32_t off, uint32_t v,
                                              uint32_t fp, int a, int b, uint32_t c,
                                              uint32_t id) {
  const uint32_t hv = word_field(w, off, a) + 1u;
  uint32_t x = (c >= fp ? v + hv : v - hv) + id;
  uint32_t at = off + (uint32_t)a;
  for (uint32_t t = 0; t < id; t++, at += (uint32_t)b) x += word_field(w, at, b);
  return x;
}

// An LE neighbor from its slot's words: the left rock (id 0), the right rock
// (id == L), or the interpolated base plus the signed sea.
__device__ __forceinline__ uint32_t le_draw_w(const uint32_t *w, uint32_t off, uint32_t v,
                                              uint32_t fp, int a, int sb, uint32_t T, uint32_t c,
                                              uint32_t id, uint32_t L) {
  const uint32_t sw = (uint32_t)sb + 1u;
  const uint32_t r1m = word_field(w, off, a);
  const uint32_t r1 = c < fp ? v - r1m : v + r1m;
  if (id == 0) return r1;
  const uint32_t s0 = off + (uint32_t)a;
  const uint32_t r2m = word_field(w, s0 + (T - 1) * sw, a);
  const uint32_t r2 = c + 1 < fp ? v - r2m : v + r2m;
  if (id == L) return r2;
  // (r2 - r1) >= 0 for sorted rows: unsigned division is the compressor's
  return word_sea(w, s0 + (id - 1) * sw, (int)sw, div_small(r2 - r1, L) * id + r1);
}

// With parts > 1, `parts` warps share the seed: warp `part` takes the subtrees
// of the first hop's children part, part + parts, ... for every later hop.
// Every part draws the first hop itself (the same values: each writes them,
// only part 0 counts them), so no warp waits for another.  Draws keep their
// Philox slot, so the output is the same for any number of parts.
//
// Draw slot k of hop h (its index in the seed's hop-h output row) uses word
// k & 3 of Philox(seed; k >> 2, s, s >> 32, TAG_KHOP | h).  The frontier is
// taken G transits at a time (G = 32, fewer only for fanouts above 2^27, so
// that a group's draw count fits 32 bits): lane p loads the header of transit
// p, then the group's G f draws are spread over the lanes.  With one part and
// G = 32 a group's slots are contiguous (pc f + j, pc a multiple of 32), so the
// lanes compute the group's Philox blocks once per 128 draws, lane l block l of
// the window, and hand the words out by shuffles; otherwise each draw
// computes its own block.  INFLIGHT: draws a lane has in flight at once (every
// load is issued before any is decoded).  MODE 2 is the CSR (one column load
// per draw).
template <int MODE, int INFLIGHT = 1>
__device__ __forceinline__ void khop_seed_warp(const DevGraph &g, const uint32_t *seeds,
                                               const KhopArgs &A, uint64_t s, SmemHdr &my,
                                               uint32_t *dbuf, uint64_t &cnt, bool &bad,
                                               uint32_t part = 0, uint32_t parts = 1) {
  static_assert(INFLIGHT == 1 || INFLIGHT == 2 || INFLIGHT == 4, "INFLIGHT in {1, 2, 4}");
  const int lane = threadIdx.x & 31;
  for (uint32_t hop = 0; hop < A.hops; hop++) {
    const uint32_t f = A.fan[hop];
    const uint64_t Mf = div_magic(f);
    const uint64_t Pall = hop ? A.width[hop - 1] : 1;
    // this part's parents: Q consecutive ones under each of its first-hop children
    const uint64_t Q = hop ? Pall / A.fan[0] : 1;
    const uint64_t mine = hop ? (part < A.fan[0] ? (A.fan[0] - part + parts - 1) / parts : 0) : 1;
    const uint64_t P = mine * Q;
    auto parent = [&](uint64_t k) -> uint64_t {
      return hop ? (part + (k / Q) * parts) * Q + k % Q : 0;
    };
    const bool count = hop || part == 0;
    const bool last_hop = hop + 1 == A.hops;
    const uint32_t G = f < (1u << 27) ? 32u : (uint32_t)max(1ull, 0xFFFFFFFFull / f);
    const bool contig = parts == 1 && G == 32;
    uint32_t *out = A.out[hop] + s * A.width[hop];
    const uint32_t *prev = hop ? A.out[hop - 1] + s * A.width[hop - 1] : nullptr;
    for (uint64_t pc = 0; pc < P; pc += G) {
      const uint64_t p = pc + lane;
      uint32_t t = INVALID_VERTEX;
      uint64_t ob = 0;
      if (lane < (int)G && p < P) {
        const uint64_t par = parent(p);
        ob = par * f;
        t = hop ? prev[par] : seeds[s];
      }
      VHdr h;
      if (t < g.n) {
        h = header<MODE>(g, t);
      } else {
        h.d = 0;
        h.P = 0;
        h.v = t;
        h.bn = h.bl = h.om = h.fp = 0;
        h.cx = 0;
        h.a = h.b = 0;
      }
      my.put(lane, h);
      my.ob[lane] = ob;
      __syncwarp();
      const uint32_t nP = (uint32_t)min((uint64_t)G, P - pc);
      const uint32_t total = nP * f;  // < 2^32 by the choice of G
      const uint64_t sbase = pc * f;  // contiguous groups: slot = sbase + j
      u32x4 rw = u32x4{0, 0, 0, 0};
      for (uint64_t j0 = 0; j0 < total; j0 += 32 * INFLIGHT) {  // warp-uniform
        if (contig && (j0 & 127u) == 0)
          rw = philox4x32_10(A.seed, (uint32_t)(((sbase + j0) >> 2) + (uint64_t)lane), (uint32_t)s,
                             (uint32_t)(s >> 32), TAG_KHOP | hop);
        uint32_t rnd[INFLIGHT];
#pragma unroll
        for (int u = 0; u < INFLIGHT; u++) {
          rnd[u] = 0;
          if (contig) {  // warp-uniform
            // block ((j0 mod 128) + 32 u + lane) / 4 of the window, word lane & 3
            const int src = (int)((((uint32_t)j0 & 127u) + 32u * u + (uint32_t)lane) >> 2);
            const uint32_t x = __shfl_sync(kFull, rw.x, src), y = __shfl_sync(kFull, rw.y, src);
            const uint32_t z = __shfl_sync(kFull, rw.z, src), w = __shfl_sync(kFull, rw.w, src);
            rnd[u] = pick4(x, y, z, w, lane & 3);
          }
        }
        if constexpr (MODE != 2) {
          // phase 1: each draw's slot, its sector copied into this lane's buffer u
          uint32_t di[INFLIGHT], dc[INFLIGHT], doff[INFLIGHT];
#pragma unroll
          for (int u = 0; u < INFLIGHT; u++) {
            const uint64_t j = j0 + (uint64_t)u * 32 + lane;
            di[u] = dc[u] = doff[u] = 0;
            if (j < total) {
              const uint32_t pl = div_by((uint32_t)j, f, Mf);
              const uint32_t d = my.d[pl];
              if (d > (MODE == 1 ? 1u : 0u)) {  // (LE degree 1: the record holds it)
                if (!contig) {
                  const uint64_t slot = my.ob[pl] + ((uint32_t)j - pl * f);
                  rnd[u] = pick(philox4x32_10(A.seed, (uint32_t)(slot >> 2), (uint32_t)s,
                                              (uint32_t)(s >> 32), TAG_KHOP | hop),
                                (int)(slot & 3));
                }
                const uint32_t i = mulhi_u32(rnd[u], d), T = my.bl[pl], K = my.om[pl];
                // slot c of neighbor i (LE: neighbor d-1 is slot C-1's right rock)
                const uint32_t c = div_small(MODE == 1 ? min(i, d - 2) : i, T);
                const uint32_t q = div_small(c, K);
                const uint64_t pos = my.P[pl] + (uint64_t)q * 256u + (uint64_t)(c - q * K) * (uint32_t)my.cx[pl];
                draw_copy(dbuf + ((uint32_t)u * 32 + lane) * kDrawBufWords, g.words, pos >> 8);
                di[u] = i;
                dc[u] = c;
                doff[u] = (uint32_t)pos & 255u;
              }
            }
          }
          draw_copy_wait();
          // phase 2: decode from the buffers, store
#pragma unroll
          for (int u = 0; u < INFLIGHT; u++) {
            const uint64_t j = j0 + (uint64_t)u * 32 + lane;
            if (j >= total) continue;
            const uint32_t pl = div_by((uint32_t)j, f, Mf);
            const uint32_t d = my.d[pl];
            const uint64_t slot = contig ? sbase + j : my.ob[pl] + ((uint32_t)j - pl * f);
            uint32_t nv = INVALID_VERTEX;
            if (d > (MODE == 1 ? 1u : 0u)) {
              const uint32_t *w = dbuf + ((uint32_t)u * 32 + lane) * kDrawBufWords;
              const uint32_t T = my.bl[pl], id = di[u] - dc[u] * T;
              if constexpr (MODE == 0) {
                nv = gt_draw_w(w, doff[u], my.v[pl], my.fp[pl], my.a[pl], my.b[pl], dc[u], id);
              } else {
                const uint32_t L = min(T, d - 1 - dc[u] * T);
                nv = le_draw_w(w, doff[u], my.v[pl], my.fp[pl], my.a[pl], my.b[pl], T, dc[u], id,
                               L);
              }
            } else if (d == 1) {
              nv = my.fp[pl];  // LE degree 1
            }
            if (d) {
              if (nv >= g.n) {
                bad = true;
                nv = INVALID_VERTEX;
              } else if (count) {
                cnt++;
              }
            }
            if (last_hop) store_out_u32(out + slot, nv);
            else out[slot] = nv;  // read back by the next hop
          }
        } else {  // CSR: one column load per draw
          uint32_t col[INFLIGHT];
#pragma unroll
          for (int u = 0; u < INFLIGHT; u++) {
            const uint64_t j = j0 + (uint64_t)u * 32 + lane;
            col[u] = INVALID_VERTEX;
            if (j < total) {
              const uint32_t pl = div_by((uint32_t)j, f, Mf);
              const uint32_t d = my.d[pl];
              if (d) {
                if (!contig) {
                  const uint64_t slot = my.ob[pl] + ((uint32_t)j - pl * f);
                  rnd[u] = pick(philox4x32_10(A.seed, (uint32_t)(slot >> 2), (uint32_t)s,
                                              (uint32_t)(s >> 32), TAG_KHOP | hop),
                                (int)(slot & 3));
                }
                col[u] = load_cold_u32(g.cols + my.P[pl] + mulhi_u32(rnd[u], d));
              }
            }
          }
#pragma unroll
          for (int u = 0; u < INFLIGHT; u++) {
            const uint64_t j = j0 + (uint64_t)u * 32 + lane;
            if (j >= total) continue;
            const uint32_t pl = div_by((uint32_t)j, f, Mf);
            const uint64_t slot = contig ? sbase + j : my.ob[pl] + ((uint32_t)j - pl * f);
            uint32_t nv = col[u];
            if (my.d[pl]) {
              if (nv >= g.n) {
                bad = true;
                nv = INVALID_VERTEX;
              } else if (count) {
                cnt++;
              }
            }
            if (last_hop) store_out_u32(out + slot, nv);
            else out[slot] = nv;  // read back by the next hop
          }
        }
      }
      __syncwarp();
    }
  }
}

// Start vertex i of a multi-RW job whose roots are drawn from its seed: the
// stream of grass_mrw_roots (word i & 3 of Philox(seed; i >> 2, 0, 0,
// TAG_MRW_ROOT), mapped to [0, n)).
__device__ __forceinline__ uint32_t mrw_root(uint32_t n, uint64_t seed, uint64_t i) {
  const u32x4 r = philox4x32_10(seed, (uint32_t)(i >> 2), 0u, 0u, TAG_MRW_ROOT);
  return mulhi_u32(pick(r, (int)(i & 3)), n);
}

// Multi random walk of one sample (MultiRWApp, GT/src/apps/multiRW/multiRW.cu:3-112).
// The sample's state is vtx[0..R), the walkers' vertices (updated in place),
// and rec[0..R), each walker's 16-byte vertex record (all zero for a vertex
// out of range), in shared or global memory.  Keeping the record makes a
// step cost two dependent DRAM reads (payload, then the new vertex's record)
// instead of three.  Lane j keeps the total degree of walkers [j*B, (j+1)*B),
// B = ceil(R/32); a degree-proportional pick scans the 32 bucket sums with
// shuffles, then the chosen bucket 32 entries at a time.  Step t draws from
// Philox(seed; t, sample, .., TAG_MRW): word 0 (+ word 2 as high half) picks
// the walker, word 1 the neighbor.  Lane k computes the block of step
// t0 + k, so one Philox evaluation per lane serves 32 steps.
template <int MODE>
__device__ __forceinline__ void mrw_warp(const DevGraph &g, uint32_t *vtx, uint4 *rec, uint32_t R,
                                         uint32_t T, int select, uint64_t seed, uint64_t sample,
                                         uint32_t *src, uint32_t *dst, uint64_t &cnt, bool &bad) {
  const int lane = threadIdx.x & 31;
  const uint32_t B = (R + 31) / 32;
  // Records of the start vertices: four independent loads in flight per lane.
  for (uint32_t c0 = 0; c0 < R; c0 += 128) {
    uint4 r[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t i = c0 + k * 32 + lane;
      const uint32_t x = i < R ? vtx[i] : INVALID_VERTEX;
      r[k] = x < g.n ? graph_record<MODE>(g, x) : make_uint4(0u, 0u, 0u, 0u);
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t i = c0 + k * 32 + lane;
      if (i < R) rec[i] = r[k];
    }
  }
  __syncwarp();
  uint64_t bsum = 0;  // this lane's bucket
  for (uint32_t i = lane * B; i < min(R, (lane + 1) * B); i++) bsum += rec[i].z;
  uint64_t wsum = bsum;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(kFull, wsum, o);
  for (uint32_t t0 = 0; t0 < T; t0 += 32) {
    const u32x4 mine =
        philox4x32_10(seed, t0 + lane, (uint32_t)sample, (uint32_t)(sample >> 32), TAG_MRW);
    const uint32_t tn = min(32u, T - t0);
    for (uint32_t k = 0; k < tn; k++) {
      const uint32_t rx = __shfl_sync(kFull, mine.x, k), ry = __shfl_sync(kFull, mine.y, k),
                     rz = __shfl_sync(kFull, mine.z, k);
      const uint64_t io = sample * T + t0 + k;
      uint32_t x;
      if (select == GRASS_SELECT_DEGREE) {
        if (wsum == 0) {
          if (lane == 0) {
            src[io] = INVALID_VERTEX;
            dst[io] = INVALID_VERTEX;
          }
          continue;
        }
        const uint64_t u = mulhi_u64(((uint64_t)rz << 32) | rx, wsum);
        // bucket: first lane whose inclusive prefix exceeds u
        uint64_t incl = bsum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const uint64_t y = __shfl_up_sync(kFull, incl, o);
          if (lane >= o) incl += y;
        }
        const int Lb = __ffs(__ballot_sync(kFull, incl > u)) - 1;
        uint64_t acc = __shfl_sync(kFull, incl - bsum, Lb);  // prefix before the bucket
        const uint32_t b0 = (uint32_t)Lb * B, b1 = min(R, b0 + B);
        x = b1 - 1;
        for (uint32_t c0 = b0; c0 < b1; c0 += 32) {  // two passes for R <= 2048
          const uint32_t i = c0 + lane;
          const uint64_t d = i < b1 ? rec[i].z : 0u;
          uint64_t ci = d;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const uint64_t y = __shfl_up_sync(kFull, ci, o);
            if (lane >= o) ci += y;
          }
          const unsigned hit = __ballot_sync(kFull, i < b1 && acc + ci > u);
          if (hit) {
            x = c0 + (uint32_t)(__ffs(hit) - 1);
            break;
          }
          acc += __shfl_sync(kFull, ci, 31);
        }
      } else {
        x = mulhi_u32(rx, R);
      }
      // lane 0 moves walker x
      uint32_t nd = 0, od = 0;
      bool moved = false;
      if (lane == 0) {
        const uint32_t v = vtx[x];
        const uint4 r = rec[x];
        od = r.z;
        src[io] = v;
        if (od == 0) {
          dst[io] = INVALID_VERTEX;
        } else {
          const VHdr h = record_header<MODE>(r, v);
          const uint32_t nv = neighbor<MODE>(g, h, mulhi_u32(ry, h.d));
          if (nv >= g.n) {
            bad = true;
            dst[io] = INVALID_VERTEX;
          } else {
            dst[io] = nv;
            cnt++;
            const uint4 nr = graph_record<MODE>(g, nv);
            vtx[x] = nv;
            rec[x] = nr;
            nd = nr.z;
            moved = true;
          }
        }
      }
      moved = __shfl_sync(kFull, moved, 0);
      if (moved) {
        nd = __shfl_sync(kFull, nd, 0);
        od = __shfl_sync(kFull, od, 0);
        if (lane == (int)(x / B)) bsum = bsum - od + nd;
        wsum = wsum - od + nd;
      }
      __syncwarp();
    }
  }
}

}  // namespace grass
