/*
 * grass_oracle.c -- CPU oracle (test infrastructure only; see grass_oracle.h).
 *
 * Plain C11 + OpenMP.  Every function states the reference file:line whose
 * behaviour it restates.  Nothing here is tuned for speed beyond OpenMP over
 * independent walkers/samples: it is the checker and the timed CPU baseline.
 */
#include "grass_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------ */
/* Bit access.  The stream is MSB-first; words hold 4 file bytes big-endian
 * (GT/src/grass.cu:1147-1159).  A field of width w <= 32 at bit offset off is
 * the reference's get_32b(off) >> (32 - w) (GT/src/bcg.cuh:64-70, 90-95).   */
static inline uint32_t fld(const uint32_t *w, uint64_t off, int width) {
  if (width <= 0) return 0;
  uint64_t wi = off >> 5;
  int s = (int)(off & 31);
  uint64_t win = ((uint64_t)w[wi] << 32) | (uint64_t)w[wi + 1];
  return (uint32_t)((win << s) >> (64 - width));
}

/* Elias-gamma of x+1, returns x (GT/src/bcg.cuh:82-107): count the leading
 * zeros z of the 32-bit window, then read z+1 bits and subtract 1.  Valid for
 * z <= 31 as in the reference; returns -1 when the window is all zeros. */
static inline int64_t gam(const uint32_t *w, uint64_t *off) {
  uint32_t win = fld(w, *off, 32);
  if (win == 0) return -1;
  int z = __builtin_clz(win);
  uint32_t v = fld(w, *off + (uint64_t)z, z + 1);
  *off += (uint64_t)(2 * z + 1);
  return (int64_t)v - 1;
}

static inline uint64_t isqrt_u64(uint64_t x) {
  /* floor(sqrt(x)); the compressor uses (int64)sqrt((double)x)
   * (GT/chunk_compress/compressor.hpp:50, LE/chunk_compress/compressor.hpp:62),
   * which equals the exact floor square root for every x < 2^52. */
  uint64_t r = (uint64_t)sqrt((double)x);
  while (r * r > x) r--;
  while ((r + 1) * (r + 1) <= x) r++;
  return r;
}

/* ------------------------------------------------------------------------ */
/* Loading (GT/src/grass.cu:1126-1215; identical in LE/src/grass.cu:1015-1095)
 * plus the device offset expansion (GT/src/bcg.cuh:368-412) and the exclusive
 * scan over n+1 entries (GT/src/utils.hpp:363-375).
 *
 * Deviation (documented): the reference counts n = (size-1)*8/ubl, which
 * includes zero-length fields that are only byte padding.  A real vertex
 * always encodes at least one bit, so trailing zero-length fields are
 * trimmed; n_file keeps the reference's count. */
static uint32_t *pack_words(const uint8_t *b, uint64_t size, uint64_t *n_words_out) {
  uint64_t nw = (size + 3) / 4;
  uint32_t *w = (uint32_t *)calloc(nw + 2, sizeof(uint32_t));
  if (!w) return NULL;
  for (uint64_t i = 0; i < size; i++) w[i >> 2] |= (uint32_t)b[i] << (24 - 8 * (i & 3));
  *n_words_out = nw;
  return w;
}

int og_load_mem(const uint8_t *gb, uint64_t gsize, const uint8_t *ob, uint64_t osize,
                og_graph *g) {
  memset(g, 0, sizeof(*g));
  if (osize < 1) return OG_E_FORMAT;
  uint32_t ubl = ob[0];
  if (ubl < 1 || ubl > 64) return OG_E_FORMAT;
  uint64_t onw = 0;
  uint32_t *ow = pack_words(ob + 1, osize - 1, &onw);
  if (!ow) return OG_E_OOM;
  uint64_t n_file = ((osize - 1) * 8) / ubl;
  if (n_file > 0xFFFFFFFEull) { free(ow); return OG_E_FORMAT; }
  uint64_t *lens = (uint64_t *)malloc((n_file + 1) * sizeof(uint64_t));
  if (!lens) { free(ow); return OG_E_OOM; }
  for (uint64_t u = 0; u < n_file; u++) {
    /* field u occupies bits [u*ubl, (u+1)*ubl) of the payload, MSB first */
    uint64_t off = u * ubl;
    uint64_t val;
    if (ubl <= 32) {
      val = fld(ow, off, (int)ubl);
    } else {
      val = ((uint64_t)fld(ow, off, (int)ubl - 32) << 32) | fld(ow, off + ubl - 32, 32);
    }
    lens[u] = val;
  }
  free(ow);
  uint64_t n = n_file;
  while (n > 0 && lens[n - 1] == 0) n--;
  uint64_t *offs = (uint64_t *)malloc((n + 1) * sizeof(uint64_t));
  if (!offs) { free(lens); return OG_E_OOM; }
  uint64_t acc = 0;
  for (uint64_t u = 0; u < n; u++) { offs[u] = acc; acc += lens[u]; }
  offs[n] = acc;
  free(lens);
  if (acc > gsize * 8) { free(offs); return OG_E_FORMAT; }
  uint64_t gnw = 0;
  uint32_t *gw = pack_words(gb, gsize, &gnw);
  if (!gw) { free(offs); return OG_E_OOM; }
  g->words = gw;
  g->n_words = gnw;
  g->offsets = offs;
  g->n = (uint32_t)n;
  g->n_file = (uint32_t)n_file;
  g->ubl = ubl;
  g->graph_bits = gsize * 8;
  return OG_OK;
}

static uint8_t *read_file(const char *path, uint64_t *size) {
  FILE *f = fopen(path, "rb");
  if (!f) return NULL;
  fseek(f, 0, SEEK_END);
  long s = ftell(f);
  fseek(f, 0, SEEK_SET);
  uint8_t *b = (uint8_t *)malloc(s > 0 ? (size_t)s : 1);
  if (b && s > 0 && fread(b, 1, (size_t)s, f) != (size_t)s) { free(b); b = NULL; }
  fclose(f);
  *size = (uint64_t)(s > 0 ? s : 0);
  return b;
}

int og_load(const char *prefix, og_graph *g) {
  char path[4096];
  uint64_t gs = 0, os = 0;
  snprintf(path, sizeof path, "%s.graph", prefix);
  uint8_t *gb = read_file(path, &gs);
  if (!gb) return OG_E_IO;
  snprintf(path, sizeof path, "%s.offset", prefix);
  uint8_t *ob = read_file(path, &os);
  if (!ob) { free(gb); return OG_E_IO; }
  int rc = og_load_mem(gb, gs, ob, os, g);
  free(gb);
  free(ob);
  return rc;
}

void og_free(og_graph *g) {
  free(g->words);
  free(g->offsets);
  memset(g, 0, sizeof(*g));
}

uint32_t og_n(const og_graph *g) { return g->n; }
uint64_t og_offset(const og_graph *g, uint32_t v) { return g->offsets[v]; }

/* ------------------------------------------------------------------------ */
/* Headers. */
typedef struct {
  uint32_t v, d;
  int a_bit;   /* GT head_bit / LE rock_bit (LE d==1: the neighbor itself) */
  int b_bit;   /* GT body_bit / LE sea_bit */
  int64_t fp;  /* first_pos */
  int64_t bn;  /* GT block_num / LE chunk_num */
  int64_t bl;  /* GT block_len / LE chunk_len (decoder's value) */
  int64_t om;  /* om_num */
  uint64_t P;  /* bit offset of the payload */
  int ok;
} hdr_t;

/* GT: BCGVertex ctor, GT/src/bcg.cuh:109-136. */
static hdr_t gt_header(const og_graph *g, uint32_t v) {
  hdr_t h;
  memset(&h, 0, sizeof h);
  h.v = v;
  uint64_t off = g->offsets[v];
  int64_t d = gam(g->words, &off), hb = gam(g->words, &off), bb = gam(g->words, &off),
          fp = gam(g->words, &off);
  if (d < 0 || hb < 0 || bb < 0 || fp < 0 || hb > 32 || bb > 32) return h;
  h.d = (uint32_t)d;
  h.a_bit = (int)hb;
  h.b_bit = (int)bb;
  h.fp = fp;
  int64_t s = (int64_t)isqrt_u64((uint64_t)d);
  if (s * s == d) {
    h.bn = h.bl = s;
    h.om = 0;
  } else {
    h.bn = s + 1;
    h.bl = d / h.bn;
    h.om = d - h.bn * h.bl;
  }
  h.P = off;
  h.ok = 1;
  return h;
}

/* GT get_vertex, GT/src/bcg.cuh:138-168. */
static uint32_t gt_get(const og_graph *g, const hdr_t *h, uint32_t i) {
  int64_t nb = i;
  int flag = nb < (h->bl + 1) * h->om;
  if (!flag) nb -= (h->bl + 1) * h->om;
  int64_t blk = nb / (h->bl + flag);
  int64_t id = nb - blk * (h->bl + flag);
  if (!flag) blk += h->om;
  uint64_t pos = h->P + (uint64_t)(blk * ((int64_t)h->b_bit * h->bl - h->b_bit + h->a_bit)) +
                 (uint64_t)((blk < h->om ? blk : h->om) * h->b_bit);
  int64_t hv = fld(g->words, pos, h->a_bit);
  pos += (uint64_t)h->a_bit;
  int64_t cur = (blk >= h->fp) ? (int64_t)h->v + hv + 1 : (int64_t)h->v - hv - 1;
  while (id-- > 0) {
    cur += (int64_t)fld(g->words, pos, h->b_bit) + 1;
    pos += (uint64_t)h->b_bit;
  }
  return (uint32_t)cur;
}

/* LE: BCGVertex ctor, LE/src/bcg.cuh:130-152 (chunk geometry of the
 * compressor's set_chunks, LE/chunk_compress/compressor.hpp:49-71). */
static hdr_t le_header(const og_graph *g, uint32_t v) {
  hdr_t h;
  memset(&h, 0, sizeof h);
  h.v = v;
  uint64_t off = g->offsets[v];
  int64_t d = gam(g->words, &off);
  if (d < 0) return h;
  h.d = (uint32_t)d;
  if (d == 0) { h.ok = 1; h.P = off; return h; }
  int64_t rb = gam(g->words, &off);
  if (rb < 0) return h;
  h.a_bit = (int)(d == 1 ? 0 : rb);
  if (d == 1) { h.fp = rb; /* the neighbor ID */ h.ok = 1; h.P = off; return h; }
  int64_t sb = gam(g->words, &off), fp = gam(g->words, &off);
  if (sb < 0 || fp < 0 || rb > 32 || sb > 31) return h;
  h.b_bit = (int)sb;
  h.fp = fp;
  int64_t D = d - 1;
  int64_t s = (int64_t)isqrt_u64((uint64_t)D);
  int64_t om = D - s * s;
  h.bn = s + (om > s);
  h.bl = D / h.bn;
  h.om = D - h.bn * h.bl;
  h.P = off;
  h.ok = 1;
  return h;
}

/* LE get_vertex, LE/src/bcg.cuh:195-261. */
static uint32_t le_get(const og_graph *g, const hdr_t *h, uint32_t i) {
  if (h->d == 1) return (uint32_t)h->fp;
  int64_t nb = i;
  int64_t this_len = h->bl + 1;
  int flag = nb >= h->om * this_len;
  if (flag) { nb -= h->om * this_len; this_len -= 1; }
  int64_t c = this_len ? nb / this_len : 0;
  int64_t id = nb - c * this_len;
  if (flag) c += h->om;
  int64_t r1 = fld(g->words, h->P + (uint64_t)(c * h->a_bit), h->a_bit);
  r1 = (c < h->fp) ? (int64_t)h->v - r1 : (int64_t)h->v + r1;
  if (id == 0) return (uint32_t)r1;
  int64_t r2 = fld(g->words, h->P + (uint64_t)((c + 1) * h->a_bit), h->a_bit);
  r2 = (c + 1 < h->fp) ? (int64_t)h->v - r2 : (int64_t)h->v + r2;
  uint64_t spos = h->P + (uint64_t)((h->bn + 1) * h->a_bit) +
                  (uint64_t)(((h->bl - 1) * c + (h->om < c ? h->om : c) + id - 1) * (h->b_bit + 1));
  uint32_t raw = fld(g->words, spos, h->b_bit + 1);
  int64_t mag = raw >> 1;
  int neg = raw & 1;
  /* (r2 - r1) >= 0 for sorted lists, so C's truncating division is the floor
   * the compressor used (LE/chunk_compress/compressor.hpp:300). */
  return (uint32_t)(((r2 - r1) / this_len) * id + r1 + (neg ? -mag : mag));
}

static inline hdr_t header(const og_graph *g, int mode, uint32_t v) {
  return mode == OG_MODE_GT ? gt_header(g, v) : le_header(g, v);
}
static inline uint32_t getv(const og_graph *g, int mode, const hdr_t *h, uint32_t i) {
  return mode == OG_MODE_GT ? gt_get(g, h, i) : le_get(g, h, i);
}

uint32_t og_degree(const og_graph *g, int mode, uint32_t v) {
  if (v >= g->n) return OG_INVALID;
  hdr_t h = header(g, mode, v);
  return h.ok ? h.d : OG_INVALID;
}

uint32_t og_get_vertex(const og_graph *g, int mode, uint32_t v, uint32_t i) {
  if (v >= g->n) return OG_INVALID;
  hdr_t h = header(g, mode, v);
  if (!h.ok || i >= h.d) return OG_INVALID;
  return getv(g, mode, &h, i);
}

int og_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

static void set_threads(int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#else
  (void)threads;
#endif
}

int og_degrees(const og_graph *g, int mode, uint32_t *deg, int threads) {
  set_threads(threads);
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for (int64_t v = 0; v < (int64_t)g->n; v++) {
    hdr_t h = header(g, mode, (uint32_t)v);
    if (!h.ok) bad = 1;
    deg[v] = h.ok ? h.d : 0;
  }
  return bad ? OG_E_FORMAT : OG_OK;
}

/* Whole-vertex decode.  GT walks each block head-then-gaps, the order the
 * block-cooperative GlobalDecoder produces (GT/src/bcg.cuh:254-298); LE uses
 * the O(1) random access for each index. */
static void decode_vertex(const og_graph *g, int mode, const hdr_t *h, uint32_t *out) {
  if (mode == OG_MODE_LE) {
    for (uint32_t i = 0; i < h->d; i++) out[i] = le_get(g, h, i);
    return;
  }
  uint64_t pos = h->P;
  uint32_t k = 0;
  for (int64_t b = 0; b < h->bn; b++) {
    int64_t len = h->bl + (b < h->om);
    int64_t hv = fld(g->words, pos, h->a_bit);
    pos += (uint64_t)h->a_bit;
    int64_t cur = (b >= h->fp) ? (int64_t)h->v + hv + 1 : (int64_t)h->v - hv - 1;
    out[k++] = (uint32_t)cur;
    for (int64_t j = 1; j < len; j++) {
      cur += (int64_t)fld(g->words, pos, h->b_bit) + 1;
      pos += (uint64_t)h->b_bit;
      out[k++] = (uint32_t)cur;
    }
  }
}

int og_decode_all(const og_graph *g, int mode, uint64_t *rowptr, uint32_t *cols, int threads) {
  uint32_t *deg = (uint32_t *)malloc(((size_t)g->n + 1) * sizeof(uint32_t));
  if (!deg) return OG_E_OOM;
  int rc = og_degrees(g, mode, deg, threads);
  if (rc) { free(deg); return rc; }
  uint64_t acc = 0;
  for (uint32_t v = 0; v < g->n; v++) { rowptr[v] = acc; acc += deg[v]; }
  rowptr[g->n] = acc;
  free(deg);
  if (!cols) return OG_OK;
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t v = 0; v < (int64_t)g->n; v++) {
    hdr_t h = header(g, mode, (uint32_t)v);
    decode_vertex(g, mode, &h, cols + rowptr[v]);
  }
  return OG_OK;
}

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel Random Numbers: As
 * Easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with the
 * published multipliers, key schedule bumped by the published Weyl
 * constants between rounds. */
void og_philox4x32_10(uint32_t k0, uint32_t k1, const uint32_t c[4], uint32_t out[4]) {
  uint32_t x0 = c[0], x1 = c[1], x2 = c[2], x3 = c[3];
  for (int r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * x0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
    uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ k0;
    uint32_t y1 = (uint32_t)p1;
    uint32_t y2 = (uint32_t)(p0 >> 32) ^ x3 ^ k1;
    uint32_t y3 = (uint32_t)p0;
    x0 = y0; x1 = y1; x2 = y2; x3 = y3;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = x0; out[1] = x1; out[2] = x2; out[3] = x3;
}

static inline uint32_t mulhi32(uint32_t r, uint32_t d) {
  return (uint32_t)(((uint64_t)r * d) >> 32);
}

static inline uint32_t draw(uint64_t seed, uint32_t c0, uint64_t id, uint32_t tag, int word) {
  uint32_t c[4] = {c0, (uint32_t)id, (uint32_t)(id >> 32), tag}, o[4];
  og_philox4x32_10((uint32_t)seed, (uint32_t)(seed >> 32), c, o);
  return o[word];
}

void og_uniform_starts(uint32_t n, uint64_t count, uint64_t seed, uint32_t *out) {
  for (uint64_t i = 0; i < count; i++)
    out[i] = mulhi32(draw(seed, (uint32_t)(i >> 2), 0, OG_TAG_START, (int)(i & 3)), n);
}

void og_mrw_roots(uint32_t n, uint64_t S, uint32_t R, uint64_t seed, uint32_t *roots) {
  uint64_t tot = S * (uint64_t)R;
  for (uint64_t i = 0; i < tot; i++)
    roots[i] = mulhi32(draw(seed, (uint32_t)(i >> 2), 0, OG_TAG_MRW_ROOT, (int)(i & 3)), n);
}

/* ------------------------------------------------------------------------ */
/* Random walk: DeepWalkApp::next (GT/src/apps/randomwalk/randomWalks.cu:49-81,
 * LE/src/apps/randomwalk/randomWalks.cu) run for L steps per walker.  A vertex
 * with no edges ends the walk (next returns -1, the engine stores the invalid
 * vertex, GT/src/grass.cu:180-183); later entries stay invalid.
 * Draw of step s for walker w: word s&3 of Philox(seed; s>>2, w, w>>32, TAG_RW). */
uint64_t og_rw(const og_graph *g, int mode, const uint32_t *starts, uint64_t W, uint32_t L,
               uint64_t seed, uint32_t *paths, int threads) {
  set_threads(threads);
  uint64_t total = 0;
  const uint64_t pitch = (uint64_t)L + 1;
#pragma omp parallel for schedule(static) reduction(+ : total)
  for (int64_t w = 0; w < (int64_t)W; w++) {
    uint32_t *row = paths + (uint64_t)w * pitch;
    uint32_t v = starts[w];
    if (v >= g->n) v = OG_INVALID;
    row[0] = starts[w];
    uint32_t o[4] = {0, 0, 0, 0};
    for (uint32_t s = 0; s < L; s++) {
      if ((s & 3) == 0) {
        uint32_t c[4] = {s >> 2, (uint32_t)w, (uint32_t)((uint64_t)w >> 32), OG_TAG_RW};
        og_philox4x32_10((uint32_t)seed, (uint32_t)(seed >> 32), c, o);
      }
      if (v != OG_INVALID) {
        hdr_t h = header(g, mode, v);
        if (!h.ok || h.d == 0) {
          v = OG_INVALID;
        } else {
          v = getv(g, mode, &h, mulhi32(o[s & 3], h.d));
          total++;
        }
      }
      row[s + 1] = v;
    }
  }
  return total;
}

/* ------------------------------------------------------------------------ */
/* Second-order (node2vec) walk, beyond the reference (its apps are first
 * order, GT/src/apps/randomwalk/randomWalks.cu:49-81).  Membership of x in
 * N(u): a binary search of u's sorted list through get_vertex. */
static int og_has_neighbor(const og_graph *g, int mode, uint32_t u, uint32_t x) {
  if (u >= g->n) return 0;
  hdr_t h = header(g, mode, u);
  if (!h.ok || h.d == 0 || getv(g, mode, &h, 0) > x) return 0;
  uint32_t lo = 0, hi = h.d - 1;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo + 1) / 2;
    if (getv(g, mode, &h, mid) <= x) lo = mid;
    else hi = mid - 1;
  }
  return getv(g, mode, &h, lo) == x;
}

uint64_t og_node2vec(const og_graph *g, int mode, const uint32_t *starts, uint64_t W,
                     uint32_t L, uint64_t seed, double p, double q, uint32_t max_tries,
                     uint32_t *paths, int threads) {
  set_threads(threads);
  if (!max_tries) max_tries = 64;
  const double a[3] = {1.0 / p, 1.0, 1.0 / q};
  double amax = a[0] > a[1] ? a[0] : a[1];
  if (a[2] > amax) amax = a[2];
  uint64_t t[3];
  for (int k = 0; k < 3; k++) t[k] = (uint64_t)(a[k] / amax * 4294967296.0);
  uint64_t total = 0;
  const uint64_t pitch = (uint64_t)L + 1;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : total)
  for (int64_t w = 0; w < (int64_t)W; w++) {
    uint32_t *row = paths + (uint64_t)w * pitch;
    uint32_t v = starts[w], u = OG_INVALID;
    if (v >= g->n) v = OG_INVALID;
    row[0] = starts[w];
    for (uint32_t s = 0; s < L; s++) {
      if (v != OG_INVALID) {
        hdr_t h = header(g, mode, v);
        if (!h.ok || h.d == 0) {
          v = OG_INVALID;
        } else {
          uint32_t x = OG_INVALID;
          for (uint32_t k = 0; k < max_tries; k++) {
            uint32_t c[4] = {s, (uint32_t)w, (uint32_t)((uint64_t)w >> 32), OG_TAG_N2V | k}, o[4];
            og_philox4x32_10((uint32_t)seed, (uint32_t)(seed >> 32), c, o);
            x = getv(g, mode, &h, mulhi32(o[0], h.d));
            if (s == 0 || k + 1 == max_tries) break;
            const uint64_t th = x == u ? t[0] : og_has_neighbor(g, mode, u, x) ? t[1] : t[2];
            if ((uint64_t)o[1] < th) break;
          }
          u = v;
          v = x;
          total++;
        }
      }
      row[s + 1] = v;
    }
  }
  return total;
}

uint64_t og_rw_csr(const uint64_t *rowptr, const uint32_t *cols, uint32_t n,
                   const uint32_t *starts, uint64_t W, uint32_t L, uint64_t seed,
                   uint32_t *paths, int threads) {
  set_threads(threads);
  uint64_t total = 0;
  const uint64_t pitch = (uint64_t)L + 1;
#pragma omp parallel for schedule(static) reduction(+ : total)
  for (int64_t w = 0; w < (int64_t)W; w++) {
    uint32_t *row = paths + (uint64_t)w * pitch;
    uint32_t v = starts[w];
    if (v >= n) v = OG_INVALID;
    row[0] = starts[w];
    uint32_t o[4] = {0, 0, 0, 0};
    for (uint32_t s = 0; s < L; s++) {
      if ((s & 3) == 0) {
        uint32_t c[4] = {s >> 2, (uint32_t)w, (uint32_t)((uint64_t)w >> 32), OG_TAG_RW};
        og_philox4x32_10((uint32_t)seed, (uint32_t)(seed >> 32), c, o);
      }
      if (v != OG_INVALID) {
        uint64_t b = rowptr[v], d = rowptr[v + 1] - b;
        if (d == 0) {
          v = OG_INVALID;
        } else {
          v = cols[b + mulhi32(o[s & 3], (uint32_t)d)];
          total++;
        }
      }
      row[s + 1] = v;
    }
  }
  return total;
}

/* ------------------------------------------------------------------------ */
/* k-hop: KHopApp::next (GT/src/apps/khop/khop.cu:1-79) with runtime fanouts.
 * Hop h expands every entry p of the previous hop's frontier into fanouts[h]
 * draws with replacement; an invalid transit or one with no edges yields
 * invalid children.  Draw of slot j = p*f_h + k of sample s at hop h:
 * word j&3 of Philox(seed; j>>2, s, s>>32, TAG_KHOP | h). */
uint64_t og_khop(const og_graph *g, int mode, const uint32_t *seeds, uint64_t S,
                 const uint32_t *fanouts, int hops, uint64_t seed, uint32_t **hop_out,
                 int threads) {
  set_threads(threads);
  uint64_t width[16];
  uint64_t wcur = 1;
  for (int h = 0; h < hops; h++) { wcur *= fanouts[h]; width[h] = wcur; }
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
  for (int64_t s = 0; s < (int64_t)S; s++) {
    uint64_t prev_w = 1;
    for (int h = 0; h < hops; h++) {
      uint32_t f = fanouts[h];
      uint32_t *out = hop_out[h] + (uint64_t)s * width[h];
      const uint32_t *prev = h ? hop_out[h - 1] + (uint64_t)s * width[h - 1] : NULL;
      for (uint64_t p = 0; p < prev_w; p++) {
        uint32_t t = h ? prev[p] : seeds[s];
        hdr_t hd;
        int valid = t < g->n;
        if (valid) { hd = header(g, mode, t); valid = hd.ok && hd.d > 0; }
        for (uint32_t k = 0; k < f; k++) {
          uint64_t j = p * f + k;
          if (!valid) { out[j] = OG_INVALID; continue; }
          uint32_t r = draw(seed, (uint32_t)(j >> 2), (uint64_t)s, OG_TAG_KHOP | (uint32_t)h,
                            (int)(j & 3));
          out[j] = getv(g, mode, &hd, mulhi32(r, hd.d));
          total++;
        }
      }
      prev_w = width[h];
    }
  }
  return total;
}

/* ------------------------------------------------------------------------ */
/* Multi random walk (frontier sampling): MultiRWApp (GT/src/apps/multiRW/
 * multiRW.cu:3-112).  Each step picks one of R walkers -- uniformly, as the
 * reference's stepTransits does (:93-101), or proportionally to the walker's
 * current degree -- moves it to a uniform neighbor and records the edge.
 * Step t of sample s uses Philox(seed; t, s, s>>32, TAG_MRW): word 0 (and
 * word 2 as the high half for degree-proportional selection) picks the
 * walker, word 1 the neighbor.  A walker on a vertex with no edges records
 * an invalid destination and stays. */
/* ------------------------------------------------------------------------ */
/* Continuous-time multi-RW (select 2).  Degree-proportional walker choice is
 * the jump chain of R independent continuous-time walks in which a walker at
 * a vertex of degree d waits Exp(d) and then moves to a uniform neighbor
 * (competing exponentials: the next walker to move is x with probability
 * d_x / sum d, independently of the past).  Each walker's events are then a
 * stream of its own: event k of walker w draws Philox(seed; k, sample, w,
 * TAG_MRW_CT), words 0-1 for the holding time before it, word 2 for the
 * neighbor.  The sample's output is the first T events in (time, walker)
 * order.  Here a binary heap pops them one by one.
 *
 * det_log: ln u for u in (0, 1) from correctly rounded +, *, / in a fixed
 * order (compiled without FP contraction), bit-identical to the device:
 * u = m 2^e, m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1), z = s^2,
 * ln u = e ln2 + 2 s (1 + z/3 + ... + z^10/21). */
static double det_log(double u) {
  uint64_t b;
  memcpy(&b, &u, 8);
  int e = (int)((b >> 52) & 0x7FF) - 1023;
  uint64_t mb = (b & 0x000FFFFFFFFFFFFFull) | 0x3FF0000000000000ull;
  double m;
  memcpy(&m, &mb, 8);
  if (m > 0x1.6a09e667f3bcdp+0) {
    m = m * 0.5;
    e += 1;
  }
  const double s = (m + -1.0) / (m + 1.0);
  const double z = s * s;
  static const double c[10] = {0x1.8618618618618p-5, 0x1.af286bca1af28p-5, 0x1.e1e1e1e1e1e1ep-5,
                               0x1.1111111111111p-4, 0x1.3b13b13b13b14p-4, 0x1.745d1745d1746p-4,
                               0x1.c71c71c71c71cp-4, 0x1.2492492492492p-3, 0x1.999999999999ap-3,
                               0x1.5555555555555p-2}; /* 1/21 ... 1/3 */
  double p = c[0];
  for (int i = 1; i < 10; i++) p = c[i] + z * p;
  const double t = s + s * (z * p);
  return (double)e * 0x1.62e42fefa39efp-1 + 2.0 * t;
}

static double exp_variate(uint32_t w0, uint32_t w1) {
  const uint64_t u52 = ((uint64_t)w0 << 20) | (w1 >> 12);
  return -det_log(((double)u52 + 0.5) * 0x1p-52);
}

static double next_event_time(double t, double E, uint32_t d) {
  double nt = t + E / (double)d;
  if (nt > t) return nt;
  uint64_t b;
  memcpy(&b, &t, 8);
  b += 1;
  memcpy(&nt, &b, 8);
  return nt;
}

double og_det_log(double u) { return det_log(u); }

typedef struct {
  uint32_t v, d, k, z;
  double t;
} ct_walker;

static int ct_less(const ct_walker *W, uint32_t a, uint32_t b) {
  return W[a].t < W[b].t || (W[a].t == W[b].t && a < b);
}

static void ct_push(uint32_t *heap, uint32_t *n, const ct_walker *W, uint32_t w) {
  uint32_t i = (*n)++;
  heap[i] = w;
  while (i && ct_less(W, heap[i], heap[(i - 1) / 2])) {
    uint32_t p = (i - 1) / 2, x = heap[p];
    heap[p] = heap[i];
    heap[i] = x;
    i = p;
  }
}

static uint32_t ct_pop(uint32_t *heap, uint32_t *n, const ct_walker *W) {
  uint32_t top = heap[0];
  heap[0] = heap[--(*n)];
  uint32_t i = 0;
  for (;;) {
    uint32_t l = 2 * i + 1, r = l + 1, m = i;
    if (l < *n && ct_less(W, heap[l], heap[m])) m = l;
    if (r < *n && ct_less(W, heap[r], heap[m])) m = r;
    if (m == i) break;
    uint32_t x = heap[m];
    heap[m] = heap[i];
    heap[i] = x;
    i = m;
  }
  return top;
}

static void ct_arm(const og_graph *g, int mode, ct_walker *w, uint32_t wid, uint64_t s,
                   uint64_t seed, double t0) {
  (void)g;
  (void)mode;
  uint32_t c[4] = {w->k, (uint32_t)s, wid, OG_TAG_MRW_CT}, o[4];
  og_philox4x32_10((uint32_t)seed, (uint32_t)(seed >> 32), c, o);
  w->z = o[2];
  w->t = next_event_time(t0, exp_variate(o[0], o[1]), w->d);
}

static uint64_t mrw_ct_sample(const og_graph *g, int mode, uint32_t *rt, uint64_t s, uint32_t R,
                              uint32_t T, uint64_t seed, uint32_t *src, uint32_t *dst) {
  ct_walker *W = (ct_walker *)malloc((size_t)R * sizeof(ct_walker));
  uint32_t *heap = (uint32_t *)malloc((size_t)R * sizeof(uint32_t));
  uint32_t hn = 0;
  uint64_t total = 0;
  for (uint32_t w = 0; w < R; w++) {
    W[w].v = rt[w];
    W[w].d = rt[w] < g->n ? og_degree(g, mode, rt[w]) : 0;
    if (W[w].d == OG_INVALID) W[w].d = 0;
    W[w].k = 0;
    if (W[w].d) {
      ct_arm(g, mode, &W[w], w, s, seed, 0.0);
      ct_push(heap, &hn, W, w);
    }
  }
  for (uint32_t r = 0; r < T; r++) {
    if (!hn) {
      src[r] = OG_INVALID;
      dst[r] = OG_INVALID;
      continue;
    }
    const uint32_t w = ct_pop(heap, &hn, W);
    ct_walker *x = &W[w];
    hdr_t h = header(g, mode, x->v);
    const uint32_t nv = getv(g, mode, &h, mulhi32(x->z, x->d));
    src[r] = x->v;
    dst[r] = nv;
    total++;
    x->v = nv;
    x->d = og_degree(g, mode, nv);
    if (x->d == OG_INVALID) x->d = 0;
    x->k++;
    if (x->d) {
      ct_arm(g, mode, x, w, s, seed, x->t);
      ct_push(heap, &hn, W, w);
    }
  }
  for (uint32_t w = 0; w < R; w++) rt[w] = W[w].v;
  free(W);
  free(heap);
  return total;
}

uint64_t og_mrw(const og_graph *g, int mode, uint32_t *roots, uint64_t S, uint32_t R,
                uint32_t T, uint64_t seed, int select, uint32_t *src, uint32_t *dst,
                int threads) {
  set_threads(threads);
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total)
  for (int64_t s = 0; s < (int64_t)S; s++) {
    uint32_t *rt = roots + (uint64_t)s * R;
    if (select == 2) {
      total += mrw_ct_sample(g, mode, rt, (uint64_t)s, R, T, seed, src + (uint64_t)s * T,
                             dst + (uint64_t)s * T);
      continue;
    }
    uint32_t *deg = (uint32_t *)malloc((size_t)R * sizeof(uint32_t));
    uint64_t wsum = 0;
    for (uint32_t r = 0; r < R; r++) {
      deg[r] = rt[r] < g->n ? og_degree(g, mode, rt[r]) : 0;
      if (deg[r] == OG_INVALID) deg[r] = 0;
      wsum += deg[r];
    }
    for (uint32_t t = 0; t < T; t++) {
      uint32_t c[4] = {t, (uint32_t)s, (uint32_t)((uint64_t)s >> 32), OG_TAG_MRW}, o[4];
      og_philox4x32_10((uint32_t)seed, (uint32_t)(seed >> 32), c, o);
      uint64_t i_out = (uint64_t)s * T + t;
      uint32_t x;
      if (select == 0) {
        x = mulhi32(o[0], R);
      } else {
        if (wsum == 0) { src[i_out] = OG_INVALID; dst[i_out] = OG_INVALID; continue; }
        uint64_t r64 = ((uint64_t)o[2] << 32) | o[0];
        uint64_t u = (uint64_t)(((unsigned __int128)r64 * wsum) >> 64);
        uint64_t acc = 0;
        x = 0;
        for (uint32_t r = 0; r < R; r++) {
          acc += deg[r];
          if (u < acc) { x = r; break; }
        }
      }
      uint32_t v = rt[x];
      src[i_out] = v;
      if (deg[x] == 0) { dst[i_out] = OG_INVALID; continue; }
      hdr_t h = header(g, mode, v);
      uint32_t nv = getv(g, mode, &h, mulhi32(o[1], h.d));
      dst[i_out] = nv;
      total++;
      rt[x] = nv;
      uint32_t nd = og_degree(g, mode, nv);
      if (nd == OG_INVALID) nd = 0;
      wsum = wsum - deg[x] + nd;
      deg[x] = nd;
    }
    free(deg);
  }
  return total;
}
