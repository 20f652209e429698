/*
 * grass_oracle.h -- CPU oracle for the compressed-graph sampling path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker that the CUDA library is
 * compared against; it is never linked into, called by, or shipped with the
 * product library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg load it.
 *
 * What it restates (file:line within the GraSS reference project):
 *   - file loading and word packing      GT/src/grass.cu:1126-1215
 *   - offset-field expansion + scan      GT/src/bcg.cuh:368-412, GT/src/utils.hpp:360-386
 *   - Elias-gamma header decode          GT/src/bcg.cuh:64-107, LE/src/bcg.cuh:65-98
 *   - GT header/geometry + get_vertex    GT/src/bcg.cuh:109-168
 *   - LE header/geometry + get_vertex    LE/src/bcg.cuh:130-152, 195-261
 *   - app next() semantics (RW/k-hop/MRW) GT/src/apps/{randomwalk,khop,multiRW}/*.cu
 * and the counter-based Philox4x32-10 stream that replaces cuRAND (Salmon et
 * al., SC'11), with the index map idx = (r * d) >> 32.
 *
 * Parity pins: decode is pinned against the reference compressor's output
 * and the reference's own bcg.cuh decoder compiled for the host (oracle/_ref),
 * Philox against an independent open-source implementation (fixtures under
 * tests/golden/).  The reference's sampled paths cannot be pinned (cuRAND
 * XORWOW, outputs never materialised), so sampling parity is anchored on the
 * shared Philox stream plus a chi-square test of visit distributions.
 */
#ifndef GRASS_ORACLE_H
#define GRASS_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define OG_MODE_GT 0
#define OG_MODE_LE 1
#define OG_INVALID 0xFFFFFFFFu

#define OG_OK 0
#define OG_E_IO 1
#define OG_E_FORMAT 2
#define OG_E_ARG 3
#define OG_E_OOM 4

/* Stream tags (counter word 3); must agree with the product's RNG spec. */
#define OG_TAG_RW 0x52570001u
#define OG_TAG_KHOP 0x4b480000u /* | hop */
#define OG_TAG_MRW 0x4d520001u
#define OG_TAG_START 0x53540001u
#define OG_TAG_MRW_ROOT 0x4d520002u
#define OG_TAG_MRW_CT 0x4d520003u
#define OG_TAG_N2V 0x4e320000u /* | try */

typedef struct {
  uint32_t *words;    /* big-endian packed graph words + 2 zero guard words */
  uint64_t n_words;   /* words excluding the guard words */
  uint64_t *offsets;  /* bit offset of each vertex, n + 1 entries */
  uint32_t n;         /* vertices after trimming zero-length padding fields */
  uint32_t n_file;    /* the reference's vertex count, (size-1)*8/ubl */
  uint32_t ubl;       /* width of one length field */
  uint64_t graph_bits;/* 8 * .graph size */
} og_graph;

int og_load_mem(const uint8_t *graph_bytes, uint64_t graph_size,
                const uint8_t *offset_bytes, uint64_t offset_size, og_graph *g);
int og_load(const char *prefix, og_graph *g);
void og_free(og_graph *g);

uint32_t og_n(const og_graph *g);
uint64_t og_offset(const og_graph *g, uint32_t v);

/* Decoding.  Returns degree, or 0xFFFFFFFF on a malformed header. */
uint32_t og_degree(const og_graph *g, int mode, uint32_t v);
/* i-th neighbor of v (0 <= i < degree). */
uint32_t og_get_vertex(const og_graph *g, int mode, uint32_t v, uint32_t i);
/* Full decode into CSR.  rowptr has n+1 entries; cols may be NULL (count only).
 * Returns OG_OK or an error. */
int og_degrees(const og_graph *g, int mode, uint32_t *deg_out, int threads);
int og_decode_all(const og_graph *g, int mode, uint64_t *rowptr, uint32_t *cols,
                  int threads);

/* Philox4x32-10 with key (k0,k1) over counter c[4]. */
void og_philox4x32_10(uint32_t k0, uint32_t k1, const uint32_t c[4], uint32_t out[4]);

/* Uniform start vertices: start[i] = mulhi(word i&3 of Philox(seed; i>>2, 0, 0, TAG_START), n). */
void og_uniform_starts(uint32_t n, uint64_t count, uint64_t seed, uint32_t *out);

/* Random walk.  paths is [W][L+1]; column 0 is the start.  Returns the number
 * of sampled (valid) edges. */
uint64_t og_rw(const og_graph *g, int mode, const uint32_t *starts, uint64_t W,
               uint32_t L, uint64_t seed, uint32_t *paths, int threads);
/* Same walk over a plain CSR (rowptr u64[n+1], cols u32). */
uint64_t og_rw_csr(const uint64_t *rowptr, const uint32_t *cols, uint32_t n,
                   const uint32_t *starts, uint64_t W, uint32_t L, uint64_t seed,
                   uint32_t *paths, int threads);
/* Second-order (node2vec) walk beyond the reference: first step uniform;
 * later steps draw candidates from N(v) and accept with probability
 * alpha / alpha_max (alpha = 1/p back to u, 1 for a neighbor of u, 1/q
 * otherwise), taking the last candidate after max_tries.  Try k of step s of
 * walker w: Philox(seed; s, w, w >> 32, OG_TAG_N2V | k), word 0 the candidate,
 * word 1 against floor(alpha / alpha_max * 2^32).  Paths [W][L+1]. */
uint64_t og_node2vec(const og_graph *g, int mode, const uint32_t *starts, uint64_t W,
                     uint32_t L, uint64_t seed, double p, double q, uint32_t max_tries,
                     uint32_t *paths, int threads);

/* k-hop with replacement.  hop_out[h] is [S][prod_{j<=h} fanouts[j]]. */
uint64_t og_khop(const og_graph *g, int mode, const uint32_t *seeds, uint64_t S,
                 const uint32_t *fanouts, int hops, uint64_t seed,
                 uint32_t **hop_out, int threads);

/* Multi random walk (frontier sampling).  roots is [S][R] (updated in place);
 * src/dst are [S][T].  select: 0 = uniform walker choice, 1 = degree-
 * proportional (one Philox block per step), 2 = degree-proportional as the
 * jump chain of independent continuous-time walks (one stream per walker). */
uint64_t og_mrw(const og_graph *g, int mode, uint32_t *roots, uint64_t S, uint32_t R,
                uint32_t T, uint64_t seed, int select, uint32_t *src, uint32_t *dst,
                int threads);

/* Root initialisation for MRW: roots[s*R + r] = mulhi(Philox(seed; idx>>2, 0, 0, TAG_MRW_ROOT)[idx&3], n), idx = s*R + r. */
void og_mrw_roots(uint32_t n, uint64_t S, uint32_t R, uint64_t seed, uint32_t *roots);

int og_max_threads(void);

/* ln u for u in (0, 1), bit-identical to the device's det_log. */
double og_det_log(double u);

#ifdef __cplusplus
}
#endif
#endif
