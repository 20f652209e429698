// graphgen.cpp -- host graph tools: synthetic generators, graph_sort
// semantics and the GT/LE writers that produce the reference's on-disk format.
//
// The writers are byte-identical to the reference compressor
// (GT/chunk_compress/compressor.hpp, LE/chunk_compress/compressor.hpp) but are
// organised for many cores: one parallel pass computes every vertex's fields
// and bit length, a scan places the vertices, and a second parallel pass
// writes the fields with atomic ORs into a zeroed word buffer.  The reference
// instead builds a std::vector<bool> per vertex and concatenates them.
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <parallel/algorithm>
#include <vector>

#include "internal.h"
#include "rng.h"

using namespace grass;

struct grass_host_csr {
  uint64_t n = 0;
  std::vector<uint64_t> rowptr;
  std::vector<uint32_t> cols;
};

// ---------------------------------------------------------------------------
// Generators.

extern "C" int grass_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                              uint64_t seed, uint32_t *src, uint32_t *dst) {
  clear_error();
  if (scale == 0 || scale > 31 || !src || !dst || a < 0 || b < 0 || c < 0 || a + b + c > 1.0)
    return set_error(GRASS_E_ARG, "grass_gen_rmat: bad arguments");
  const uint64_t m = (uint64_t)edge_factor << scale;
  const uint32_t A = (uint32_t)llround(a * 65536.0);
  const uint32_t AB = (uint32_t)llround((a + b) * 65536.0);
  const uint32_t ABC = (uint32_t)llround((a + b + c) * 65536.0);
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)m; k++) {
    uint32_t u = 0, v = 0;
    u32x4 r{0, 0, 0, 0};
    for (uint32_t l = 0; l < scale; l++) {
      // 16 bits per level: eight levels per Philox block.
      if ((l & 7) == 0)
        r = philox4x32_10(seed, l >> 3, (uint32_t)k, (uint32_t)((uint64_t)k >> 32), TAG_GEN);
      uint32_t word = pick(r, (int)((l & 7) >> 1));
      uint32_t r16 = (l & 1) ? (word >> 16) : (word & 0xFFFFu);
      uint32_t ub = r16 >= AB, vb = (r16 >= A && r16 < AB) || r16 >= ABC;
      u = (u << 1) | ub;
      v = (v << 1) | vb;
    }
    src[k] = u;
    dst[k] = v;
  }
  return GRASS_OK;
}

extern "C" int grass_gen_chung_lu(uint64_t n, double exponent, double mean_degree,
                                  uint64_t max_degree, uint64_t seed, uint64_t m, uint32_t *src,
                                  uint32_t *dst) {
  clear_error();
  if (n < 2 || n > 0xFFFFFFFFull || exponent <= 2.0 || mean_degree <= 0 || !src || !dst)
    return set_error(GRASS_E_ARG, "grass_gen_chung_lu: bad arguments");
  // Continuous power law w(x) ~ (x + i0)^-alpha on [0, n), alpha = 1/(exponent-1).
  // i0 is chosen so that the expected degree of vertex 0 equals max_degree:
  // d(0) = 2m * p(0) with p the normalised density; solved by bisection.
  const double alpha = 1.0 / (exponent - 1.0);
  const double beta = 1.0 - alpha;
  auto p0 = [&](double i0) {
    double norm = (pow((double)n + i0, beta) - pow(i0, beta)) / beta;
    return pow(i0, -alpha) / norm;
  };
  double target = max_degree ? (double)max_degree / (2.0 * (double)m) : 1.0;
  double lo = 1e-9, hi = (double)n;
  for (int it = 0; it < 200; it++) {
    double mid = sqrt(lo * hi);
    if (p0(mid) > target) lo = mid; else hi = mid;
  }
  const double i0 = max_degree ? hi : 1.0;
  const double base = pow(i0, beta);
  const double span = pow((double)n + i0, beta) - base;
  (void)mean_degree;
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < (int64_t)m; k++) {
    u32x4 r = philox4x32_10(seed, 0, (uint32_t)k, (uint32_t)((uint64_t)k >> 32), TAG_GEN);
    double u1 = ((double)r.x * 4294967296.0 + r.y) * (1.0 / 18446744073709551616.0);
    double u2 = ((double)r.z * 4294967296.0 + r.w) * (1.0 / 18446744073709551616.0);
    double x1 = pow(u1 * span + base, 1.0 / beta) - i0;
    double x2 = pow(u2 * span + base, 1.0 / beta) - i0;
    uint64_t a = (uint64_t)x1, b = (uint64_t)x2;
    src[k] = (uint32_t)(a < n ? a : n - 1);
    dst[k] = (uint32_t)(b < n ? b : n - 1);
  }
  return GRASS_OK;
}

// ---------------------------------------------------------------------------
// graph_sort (GT/chunk_compress/graph_sort.cpp:47-72).

extern "C" int grass_graph_sort(const uint32_t *src, const uint32_t *dst, uint64_t m,
                                int directed, grass_host_csr **out) {
  clear_error();
  if (!out || (m && (!src || !dst))) return set_error(GRASS_E_ARG, "grass_graph_sort: bad args");
  *out = nullptr;
  uint32_t maxid = 0;
#pragma omp parallel for reduction(max : maxid)
  for (int64_t k = 0; k < (int64_t)m; k++) maxid = std::max(maxid, std::max(src[k], dst[k]));
  if (maxid >= 0x7FFFFFFFu) return set_error(GRASS_E_ARG, "vertex ids must fit int32");
  // Relabel in order of first appearance; self-loops are skipped before
  // relabelling (graph_sort.cpp:48-52).
  std::vector<int32_t> o2n((size_t)maxid + 1, -1);
  int32_t tot = 0;
  for (uint64_t k = 0; k < m; k++) {
    uint32_t u = src[k], v = dst[k];
    if (u == v) continue;
    if (o2n[u] < 0) o2n[u] = tot++;
    if (o2n[v] < 0) o2n[v] = tot++;
  }
  std::vector<uint64_t> keys;
  keys.reserve(m);
  for (uint64_t k = 0; k < m; k++) {
    uint32_t u = src[k], v = dst[k];
    if (u == v) continue;
    uint64_t a = (uint32_t)o2n[u], b = (uint32_t)o2n[v];
    if (!directed && a > b) std::swap(a, b);
    keys.push_back((a << 32) | b);
  }
  __gnu_parallel::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());

  auto *csr = new (std::nothrow) grass_host_csr();
  if (!csr) return set_error(GRASS_E_OOM, "host allocation failed");
  const uint64_t n = (uint64_t)tot;
  csr->n = n;
  csr->rowptr.assign(n + 1, 0);
  if (directed) {
    for (uint64_t e : keys) csr->rowptr[(e >> 32) + 1]++;
    for (uint64_t v = 0; v < n; v++) csr->rowptr[v + 1] += csr->rowptr[v];
    csr->cols.resize(keys.size());
#pragma omp parallel for
    for (int64_t i = 0; i < (int64_t)keys.size(); i++) csr->cols[i] = (uint32_t)keys[i];
  } else {
    // Symmetrize (graph_sort.cpp:63-72) by counting both directions, then
    // sorting each row; equal to appending mirrored edges and re-sorting.
    std::vector<uint32_t> deg(n, 0);
    for (uint64_t e : keys) { deg[e >> 32]++; deg[(uint32_t)e]++; }
    for (uint64_t v = 0; v < n; v++) csr->rowptr[v + 1] = csr->rowptr[v] + deg[v];
    csr->cols.resize(csr->rowptr[n]);
    std::vector<uint64_t> fill(csr->rowptr.begin(), csr->rowptr.end() - 1);
    for (uint64_t e : keys) {
      uint32_t a = (uint32_t)(e >> 32), b = (uint32_t)e;
      csr->cols[fill[a]++] = b;
      csr->cols[fill[b]++] = a;
    }
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t v = 0; v < (int64_t)n; v++)
      std::sort(csr->cols.begin() + csr->rowptr[v], csr->cols.begin() + csr->rowptr[v + 1]);
  }
  *out = csr;
  return GRASS_OK;
}

extern "C" int grass_host_csr_view(const grass_host_csr *csr, uint64_t *n, uint64_t *nnz,
                                   const uint64_t **rowptr, const uint32_t **cols) {
  if (!csr) return set_error(GRASS_E_ARG, "null csr");
  if (n) *n = csr->n;
  if (nnz) *nnz = csr->cols.size();
  if (rowptr) *rowptr = csr->rowptr.data();
  if (cols) *cols = csr->cols.data();
  return GRASS_OK;
}

extern "C" void grass_host_csr_free(grass_host_csr *csr) { delete csr; }

// ---------------------------------------------------------------------------
// Writers.

namespace {

inline int gamma_len(uint64_t x) {  // length of gamma(x) = code of x+1
  int L = 63 - __builtin_clzll(x + 1);
  return 2 * L + 1;
}

struct VParams {
  uint64_t d;
  int a_bit, b_bit;  // GT head/body bits; LE rock/sea bits
  uint64_t fp;
  uint64_t bn, bl, om;  // GT blocks; LE chunks (bl = the compressor's chunk_len)
  uint64_t len;         // bits
  int ok;
};

// GT encode_node_s1 (GT/chunk_compress/compressor.hpp:245-282) sizing.
VParams gt_params(uint64_t v, const uint32_t *nb, uint64_t d) {
  VParams p{};
  p.d = d;
  p.ok = 1;
  if (d == 0) {
    p.len = 4;  // gamma(0) x 4
    return p;
  }
  uint64_t s = isqrt_floor(d);
  if (s * s == d) { p.bn = p.bl = s; p.om = 0; }
  else { p.bn = s + 1; p.bl = d / p.bn; p.om = d - p.bn * p.bl; }
  int64_t fp = -1;
  int hb = 0, bb = 0;
  uint64_t k = 0;
  for (uint64_t blk = 0; blk < p.bn; blk++) {
    int64_t cur = (int64_t)nb[k] - (int64_t)v;
    if (cur < 0) { fp = (int64_t)blk; cur = -cur; }
    if (cur == 0) p.ok = 0;  // a self-loop cannot lead a GT block (head = |n-v|-1)
    hb = std::max(hb, bit_count((uint64_t)(cur - 1)));
    k++;
    uint64_t len = p.bl + (blk < p.om);
    for (uint64_t i = 1; i < len && k < d; i++, k++) {
      int64_t gap = (int64_t)nb[k] - (int64_t)nb[k - 1] - 1;
      if (gap < 0) p.ok = 0;
      bb = std::max(bb, bit_count((uint64_t)gap));
    }
  }
  p.fp = (uint64_t)(fp + 1);
  p.a_bit = hb;
  p.b_bit = bb;
  p.len = gamma_len(d) + gamma_len(hb) + gamma_len(bb) + gamma_len(p.fp) + p.bn * hb +
          (d - p.bn) * bb;
  return p;
}

// LE set_chunks + encode_node_s1 (LE/chunk_compress/compressor.hpp:49-71, 288-327).
VParams le_params(uint64_t v, const uint32_t *nb, uint64_t d) {
  VParams p{};
  p.d = d;
  p.ok = 1;
  if (d == 0) { p.len = 1; return p; }
  if (d == 1) {
    p.a_bit = 0;
    p.fp = nb[0];  // the single neighbor is stored as the rock_bit field
    p.len = gamma_len(1) + gamma_len(nb[0]);
    return p;
  }
  uint64_t D = d - 1;
  uint64_t s = isqrt_floor(D);
  uint64_t om = D - s * s;
  p.bn = s + (om > s);
  uint64_t cl = D / p.bn;
  p.om = D - p.bn * cl;
  p.bl = cl - 1;
  int64_t r0 = (int64_t)nb[0] - (int64_t)v, rl = (int64_t)nb[d - 1] - (int64_t)v;
  p.a_bit = bit_count((uint64_t)std::max(r0 < 0 ? -r0 : r0, rl < 0 ? -rl : rl));
  int64_t fp = -1;
  int sb = 0;
  uint64_t k = 0;
  for (uint64_t c = 0; c < p.bn; c++) {
    int64_t rock_l = nb[k];
    uint64_t cur_len = p.bl + (c < p.om);
    int64_t rock_r = nb[k + cur_len + 1];
    int64_t dist = (rock_r - rock_l) / (int64_t)(cur_len + 1);
    if (rock_l - (int64_t)v < 0) fp = (int64_t)c;
    k++;
    for (uint64_t i = 1; i <= cur_len && k < d; i++, k++) {
      int64_t sea = (int64_t)nb[k] - (rock_l + (int64_t)i * dist);
      sb = std::max(sb, bit_count((uint64_t)(sea < 0 ? -sea : sea)));
    }
  }
  if ((int64_t)nb[k] - (int64_t)v < 0) fp = (int64_t)p.bn;
  p.fp = (uint64_t)(fp + 1);
  p.b_bit = sb;
  p.len = gamma_len(d) + gamma_len(p.a_bit) + gamma_len(sb) + gamma_len(p.fp) +
          (p.bn + 1) * p.a_bit + (d - p.bn - 1) * (sb + 1);
  return p;
}

// MSB-first bit writer over a zeroed u64 buffer.  Writers of different
// vertices may share a word, so every store is an atomic OR.
struct BitSink {
  uint64_t *buf;
  uint64_t pos;
  inline void put(uint64_t val, int width) {
    if (width <= 0) return;
    uint64_t w = pos >> 6;
    int off = (int)(pos & 63);
    int room = 64 - off;
    if (width <= room) {
      __atomic_fetch_or(&buf[w], val << (room - width), __ATOMIC_RELAXED);
    } else {
      int rest = width - room;
      __atomic_fetch_or(&buf[w], val >> rest, __ATOMIC_RELAXED);
      __atomic_fetch_or(&buf[w + 1], val << (64 - rest), __ATOMIC_RELAXED);
    }
    pos += (uint64_t)width;
  }
  inline void gamma(uint64_t x) { put(x + 1, gamma_len(x)); }
};

void gt_write(BitSink &o, uint64_t v, const uint32_t *nb, const VParams &p) {
  // encode_node_s2, GT/chunk_compress/compressor.hpp:297-349 (non-ZETA,
  // per-vertex widths, blocks interleaved head then gaps).
  o.gamma(p.d);
  o.gamma((uint64_t)p.a_bit);
  o.gamma((uint64_t)p.b_bit);
  o.gamma(p.fp);
  uint64_t k = 0;
  for (uint64_t blk = 0; blk < p.bn; blk++) {
    int64_t cur = (int64_t)nb[k] - (int64_t)v;
    if (cur < 0) cur = -cur;
    o.put((uint64_t)(cur - 1), p.a_bit);
    k++;
    uint64_t len = p.bl + (blk < p.om);
    for (uint64_t i = 1; i < len && k < p.d; i++, k++)
      o.put((uint64_t)nb[k] - nb[k - 1] - 1, p.b_bit);
  }
}

void le_write(BitSink &o, uint64_t v, const uint32_t *nb, const VParams &p) {
  // encode_node_s2, LE/chunk_compress/compressor.hpp:329-390 (GATHER_HEAD:
  // all rocks, then all signed seas).
  o.gamma(p.d);
  if (p.d == 0) return;
  if (p.d == 1) { o.gamma(p.fp); return; }
  o.gamma((uint64_t)p.a_bit);
  o.gamma((uint64_t)p.b_bit);
  o.gamma(p.fp);
  uint64_t k = 0;
  for (uint64_t c = 0; c < p.bn; c++) {
    int64_t r = (int64_t)nb[k] - (int64_t)v;
    o.put((uint64_t)(r < 0 ? -r : r), p.a_bit);
    k += p.bl + (c < p.om) + 1;
  }
  int64_t r = (int64_t)nb[p.d - 1] - (int64_t)v;
  o.put((uint64_t)(r < 0 ? -r : r), p.a_bit);
  k = 0;
  for (uint64_t c = 0; c < p.bn; c++) {
    int64_t rock_l = nb[k];
    uint64_t cur_len = p.bl + (c < p.om);
    int64_t dist = ((int64_t)nb[k + cur_len + 1] - rock_l) / (int64_t)(cur_len + 1);
    k++;
    for (uint64_t i = 1; i <= cur_len; i++, k++) {
      int64_t sea = (int64_t)nb[k] - (rock_l + (int64_t)i * dist);
      uint64_t mag = (uint64_t)(sea < 0 ? -sea : sea);
      o.put((mag << 1) | (sea < 0 ? 1u : 0u), p.b_bit + 1);
    }
  }
}

}  // namespace

extern "C" int grass_compress(const uint64_t *rowptr, const uint32_t *cols, uint64_t n, int mode,
                              uint8_t *graph_buf, uint64_t *graph_size, uint8_t *offset_buf,
                              uint64_t *offset_size) {
  clear_error();
  if (!rowptr || !graph_size || !offset_size || (mode != GRASS_MODE_GT && mode != GRASS_MODE_LE))
    return set_error(GRASS_E_ARG, "grass_compress: bad arguments");
  if (n == 0) return set_error(GRASS_E_ARG, "grass_compress: empty graph");
  std::vector<VParams> P(n);
  int bad = 0;
#pragma omp parallel for schedule(dynamic, 4096) reduction(| : bad)
  for (int64_t v = 0; v < (int64_t)n; v++) {
    const uint32_t *nb = cols + rowptr[v];
    uint64_t d = rowptr[v + 1] - rowptr[v];
    for (uint64_t i = 0; i < d; i++) {
      if (nb[i] >= n || (i && nb[i] <= nb[i - 1])) bad = 1;
    }
    if (d > 0xFFFFFFFEull) bad = 1;
    if (bad) continue;
    P[v] = mode == GRASS_MODE_GT ? gt_params((uint64_t)v, nb, d) : le_params((uint64_t)v, nb, d);
    if (!P[v].ok) bad = 1;
  }
  if (bad)
    return set_error(GRASS_E_ARG,
                     "grass_compress: rows must be strictly increasing and < n (GT: no self-loop at a block head)");
  uint64_t max_len = 0, total = 0;
  std::vector<uint64_t> off(n + 1);
  for (uint64_t v = 0; v < n; v++) {
    off[v] = total;
    total += P[v].len;
    max_len = std::max(max_len, P[v].len);
  }
  off[n] = total;
  const int ubl = bit_count(max_len);
  const uint64_t gbytes = (total + 7) / 8;
  const uint64_t obytes = 1 + (n * (uint64_t)ubl + 7) / 8;
  if (!graph_buf || !offset_buf) {
    *graph_size = gbytes;
    *offset_size = obytes;
    return GRASS_OK;
  }
  if (*graph_size < gbytes || *offset_size < obytes)
    return set_error(GRASS_E_ARG, "grass_compress: buffers too small (%llu, %llu needed)",
                     (unsigned long long)gbytes, (unsigned long long)obytes);
  // Graph stream.
  std::vector<uint64_t> gw((total + 63) / 64 + 2, 0);
#pragma omp parallel for schedule(dynamic, 4096)
  for (int64_t v = 0; v < (int64_t)n; v++) {
    BitSink o{gw.data(), off[v]};
    const uint32_t *nb = cols + rowptr[v];
    if (mode == GRASS_MODE_GT) gt_write(o, (uint64_t)v, nb, P[v]);
    else le_write(o, (uint64_t)v, nb, P[v]);
  }
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)gbytes; i++)
    graph_buf[i] = (uint8_t)(gw[(uint64_t)i >> 3] >> (56 - 8 * ((uint64_t)i & 7)));
  // Offset file: byte 0 = ubl, then n ubl-bit lengths (write_offset3,
  // GT/chunk_compress/compressor.hpp:146-210).
  std::vector<uint64_t> ow(((uint64_t)n * ubl + 63) / 64 + 2, 0);
#pragma omp parallel for schedule(static, 8192)
  for (int64_t v = 0; v < (int64_t)n; v++) {
    BitSink o{ow.data(), (uint64_t)v * ubl};
    o.put(P[v].len, ubl);
  }
  offset_buf[0] = (uint8_t)ubl;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)obytes - 1; i++)
    offset_buf[1 + i] = (uint8_t)(ow[(uint64_t)i >> 3] >> (56 - 8 * ((uint64_t)i & 7)));
  *graph_size = gbytes;
  *offset_size = obytes;
  return GRASS_OK;
}

extern "C" int grass_compress_to_files(const uint64_t *rowptr, const uint32_t *cols, uint64_t n,
                                       int mode, const char *prefix) {
  clear_error();
  if (!prefix) return set_error(GRASS_E_ARG, "null prefix");
  uint64_t gs = 0, os = 0;
  int rc = grass_compress(rowptr, cols, n, mode, nullptr, &gs, nullptr, &os);
  if (rc) return rc;
  std::vector<uint8_t> gb(gs), ob(os);
  rc = grass_compress(rowptr, cols, n, mode, gb.data(), &gs, ob.data(), &os);
  if (rc) return rc;
  std::string p(prefix);
  FILE *f = fopen((p + ".graph").c_str(), "wb");
  if (!f) return set_error(GRASS_E_IO, "cannot create %s.graph", prefix);
  bool ok = fwrite(gb.data(), 1, gs, f) == gs;
  ok = (fclose(f) == 0) && ok;
  f = fopen((p + ".offset").c_str(), "wb");
  if (!f) return set_error(GRASS_E_IO, "cannot create %s.offset", prefix);
  ok = fwrite(ob.data(), 1, os, f) == os && ok;
  ok = (fclose(f) == 0) && ok;
  return ok ? GRASS_OK : set_error(GRASS_E_IO, "short write under %s", prefix);
}
