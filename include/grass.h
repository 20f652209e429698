/*
 * grass.h -- C ABI of the B200-native compressed-graph sampler.
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes, no
 * exceptions or aborts across the boundary.  Device-pointer entry points are
 * asynchronous on the given CUDA stream (NULL = legacy default stream);
 * "_host" entry points take host buffers, copy in and out inside the call
 * and return when the results are in host memory.
 *
 * Each entry point names the reference (calla212/GraSS) interface it replaces,
 * by file:line within that project.  The reference exposes its hot path as a
 * compile-time App template run by nextdoor<SampleType, App>(graph_file,
 * nruns) (GT/src/grass.cu:2066-2135); here the app becomes a runtime
 * parameter block and the graph a handle that outlives one run.
 */
#ifndef GRASS_B200_H
#define GRASS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace CHK_CU's print-and-assert, GT/src/utils.hpp:17) ---- */
#define GRASS_OK 0
#define GRASS_E_IO 1          /* file missing or unreadable */
#define GRASS_E_FORMAT 2      /* malformed .graph/.offset content */
#define GRASS_E_CUDA 3        /* a CUDA runtime call failed */
#define GRASS_E_OOM 4         /* host or device allocation failed */
#define GRASS_E_BUDGET 5      /* request exceeds the scratch budget */
#define GRASS_E_TIMEOUT 6     /* a bounded wait ran out */
#define GRASS_E_ARG 7         /* invalid argument */
#define GRASS_E_DATA 8        /* decoded vertex id out of range (corrupt payload) */

/* ---- decode modes: the reference's two source trees / file formats ---- */
#define GRASS_MODE_GT 0 /* GT/: gamma header + per-block head and gaps   */
#define GRASS_MODE_LE 1 /* LE/: gamma header + rocks and signed seas     */

#define GRASS_INVALID_VERTEX 0xFFFFFFFFu

/* Output layouts of random-walk paths. */
#define GRASS_LAYOUT_WALK_MAJOR 0 /* paths[w * (L+1) + s] */
#define GRASS_LAYOUT_STEP_MAJOR 1 /* paths[s * W + w]     */

/* Multi-RW walker selection. */
#define GRASS_SELECT_UNIFORM 0 /* reference: MultiRWApp::stepTransits, GT/src/apps/multiRW/multiRW.cu:93-101 */
#define GRASS_SELECT_DEGREE 1  /* frontier sampling: proportional to current degree */
/* Degree-proportional as well, computed as the jump chain of independent
 * continuous-time walks (a walker at degree d waits Exp(d), then moves): the
 * same law as GRASS_SELECT_DEGREE with walkers moving in parallel, one
 * Philox stream per walker (TAG_MRW_CT), so a different sample path. */
#define GRASS_SELECT_DEGREE_CT 2

/* Thread-local message for the last failing call on this thread. */
const char *grass_last_error(void);
/* Number of CUDA kernels this library has launched in this process. */
uint64_t grass_launch_count(void);
/* Library version string. */
const char *grass_version(void);

/* =========================================================================
 * Host graph tools.  Replace the offline pipeline GT/chunk_compress/
 * (graph_sort.cpp:22-82, compressor.hpp:24-490, compress.cpp:6-28).
 * ========================================================================= */

/* R-MAT edge generator: m = edge_factor << scale edges into src[m], dst[m].
 * Edge k takes its quadrant choices from Philox(seed; k, 0, 0, TAG_GEN).
 * No reference counterpart (the reference ships no generator). */
int grass_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                   uint64_t seed, uint32_t *src, uint32_t *dst);

/* Chung-Lu power-law generator: m edges between n vertices whose expected
 * degrees follow w_i ~ (i + i0)^(-1/(exponent-1)), scaled to mean_degree and
 * capped at max_degree.  No reference counterpart. */
int grass_gen_chung_lu(uint64_t n, double exponent, double mean_degree, uint64_t max_degree,
                       uint64_t seed, uint64_t m, uint32_t *src, uint32_t *dst);

/* Host CSR produced by grass_graph_sort. */
typedef struct grass_host_csr grass_host_csr;

/* graph_sort semantics (GT/chunk_compress/graph_sort.cpp:47-72): relabel
 * vertices by first appearance, drop self-loops, dedupe, and (directed == 0)
 * symmetrize.  Rows come out sorted. */
int grass_graph_sort(const uint32_t *src, const uint32_t *dst, uint64_t m, int directed,
                     grass_host_csr **out);
int grass_host_csr_view(const grass_host_csr *csr, uint64_t *n, uint64_t *nnz,
                        const uint64_t **rowptr, const uint32_t **cols);
void grass_host_csr_free(grass_host_csr *csr);

/* Compress a sorted CSR into the reference's on-disk format, byte-identical
 * to Compressor::compress + write_cgr (GT/chunk_compress/compressor.hpp:
 * 120-243, 245-362, 422-447; LE/chunk_compress/compressor.hpp:130-187,
 * 217-285, 288-403, 479-502).  Two-call pattern: with NULL buffers, the
 * sizes are returned in *graph_size and *offset_size; then call again with
 * buffers of those sizes. */
int grass_compress(const uint64_t *rowptr, const uint32_t *cols, uint64_t n, int mode,
                   uint8_t *graph_buf, uint64_t *graph_size, uint8_t *offset_buf,
                   uint64_t *offset_size);
/* Same, writing <prefix>.graph and <prefix>.offset. */
int grass_compress_to_files(const uint64_t *rowptr, const uint32_t *cols, uint64_t n, int mode,
                            const char *prefix);

/* =========================================================================
 * Device graph.  Replaces loadGraph (GT/src/grass.cu:1126-1215),
 * transferToGPUs (GT/src/grass.cu:1217-1233) and copyPartitionToGPU +
 * decode_offset + the offset scan (GT/src/utils.hpp:360-386,
 * GT/src/bcg.cuh:368-412).  Unlike the reference's __constant__ partition
 * (GT/src/grass.cu:59), several graphs may be open at once.
 * ========================================================================= */
typedef struct grass_graph grass_graph;
typedef struct grass_csr grass_csr; /* uncompressed-CSR baseline, below */

typedef struct {
  uint64_t n;                 /* vertices (byte-padding fields trimmed)   */
  uint64_t n_file;            /* the reference's count (size-1)*8/ubl     */
  uint64_t num_edges;         /* sum of degrees                           */
  uint32_t max_degree;
  uint32_t ubl;               /* width of one .offset length field        */
  int32_t mode;               /* GRASS_MODE_GT or GRASS_MODE_LE           */
  int32_t device;
  uint64_t graph_file_bytes;  /* .graph size                              */
  uint64_t offset_file_bytes; /* .offset size                             */
  uint64_t device_bytes;      /* resident: stream words + offset index    */
  double read_seconds;        /* file read into pinned memory             */
  double upload_seconds;      /* copies + device index build              */
} grass_graph_info;

/* Load <prefix>.graph / <prefix>.offset onto `device`. */
int grass_open(const char *prefix, int mode, int device, grass_graph **out);
/* Same from in-memory file images. */
int grass_open_mem(const void *graph_bytes, uint64_t graph_size, const void *offset_bytes,
                   uint64_t offset_size, int mode, int device, grass_graph **out);
int grass_close(grass_graph *g);
int grass_get_info(const grass_graph *g, grass_graph_info *info);
/* Waits for `stream`, then reads and clears the graph's device error word,
 * which the asynchronous device-pointer calls (samplers, decode) set instead
 * of aborting (the reference asserts, GT/src/utils.hpp:17, 108-119):
 * GRASS_E_DATA when a decoded id was out of range (corrupt payload),
 * GRASS_E_TIMEOUT when a decode warp's staged copy did not land within its
 * bounded wait (that range was decoded from global memory instead), else
 * GRASS_OK.  The _host calls check it themselves. */
int grass_check_device_error(grass_graph *g, void *stream);
/* Device view of the resident graph (for callers that launch their own
 * kernels): the stream words (n_words + at least 16 zero guard words, each
 * word the next 32 stream bits MSB-first) and the n vertex records, 16 bytes
 * each: {P low 32 bits, P bits 32..47 | a << 16 | b << 22, degree, w}, where
 * P is the bit offset of the vertex's payload, a/b are the GT head/body or LE
 * rock/sea widths, and w is first_pos (LE degree 1: the single neighbor; GT:
 * first_pos in bits 0..15 and the skip-field extra width cx in bits 16..21).
 * The records replace the reference's uint64 bit-offset table
 * (GT/src/utils.hpp:363).  The stream is the .graph stream re-laid for random
 * access, the field values unchanged:
 *   LE: the file's stream; the payload of every vertex whose longest chunk
 *       spans at most 256 bits (2 rock_bit + its seas x (sea_bit + 1)) is in
 *       neighbor order, [rock 0][seas of chunk 0][rock 1]...[last rock],
 *       instead of all rocks then all seas (same bits, same P);
 *   GT: the payloads only, back to back in vertex order; in every block the
 *       field at each position t = 16, 32, ... holds the sum of the block's
 *       raw gaps 1..t in b + cx bits instead of gap t. */
int grass_device_view(const grass_graph *g, const uint32_t **words, uint64_t *n_words,
                      const void **records);

/* Launch shape of the samplers (no reference counterpart: the reference's
 * launch shapes are compile-time constants, GT/src/grass.cu:46-49, 1845,
 * 1886).  Zero fields take the defaults; grass_autotune picks values. */
typedef struct {
  uint32_t rw_depth;          /* walkers interleaved per thread: 1, 2, 4
                                 (default 1 for LE and GT, 4 for CSR)                */
  uint32_t rw_threads;        /* threads per block for walks (default 256)           */
  uint32_t rw_blocks_per_sm;  /* resident blocks per SM for walks (0 = all resident) */
  uint32_t l2_persist;        /* 1: launches mark the vertex records (or CSR row
                                 pointers) persisting in L2 through a per-launch
                                 access-policy window                               */
  uint32_t l2_fetch_bytes;    /* 0 = leave as is; 32/64/128: this process's
                                 cudaLimitMaxL2FetchGranularity hint                 */
  uint32_t decode_stage_depth;/* decode sweep: 0 (default) reads chunk slots
                                 through L1; 1, 2 or 4 copies groups of 32 slots into
                                 shared memory (cp.async.bulk) that many groups ahead
                                 of the one being decoded (measured slower)          */
  uint32_t reserved[2];
} grass_tuning;
int grass_set_tuning(grass_graph *g, const grass_tuning *t);
int grass_get_tuning(const grass_graph *g, grass_tuning *t);

/* Per-vertex degree (BCGVertex::outd, GT/src/bcg.cuh:113 / LE/src/bcg.cuh:132). */
int grass_degrees(const grass_graph *g, uint32_t *d_deg, void *stream);

/* Decode-only sweep: every neighbor list into a device CSR.  d_rowptr has
 * n+1 entries, d_cols num_edges entries.  Replaces the block-cooperative
 * GlobalDecoder (GT/src/bcg.cuh:171-345) and per-index BCGVertex::get_vertex
 * (GT/src/bcg.cuh:153-168, LE/src/bcg.cuh:195-261). */
int grass_decode_all(const grass_graph *g, uint64_t *d_rowptr, uint32_t *d_cols, void *stream);

/* Same as grass_decode_all, but allocates no device memory.  No counterpart
 * in the reference.  For callers that cannot allocate when they decode:
 * applications that reserve the whole device for their own memory pool, and
 * loops that must not pay for allocator calls or the device-wide
 * synchronisation cudaFree implies.  The scan scratch comes from a fixed
 * 512 KiB array that every GPU loading this library holds until exit, which
 * limits graphs to 268,435,456 vertices (larger ones return GRASS_E_ARG).
 * The first call on a device looks up the array's device address, so make it
 * before any stream capture.  All calls share the array: calls that overlap
 * on the GPU (other streams, other threads) race, so the caller serialises
 * them.  Speed: once a grass_decode_all on the same graph has built its
 * decode plan (that call allocates, once), this call runs the same planned
 * sweep; before that it runs an unplanned sweep that needs no set-up, about
 * 3x slower (3.1 ms against 0.94 ms for 250 M neighbors on one B200). */
int grass_decode_all_noalloc(const grass_graph *g, uint64_t *d_rowptr, uint32_t *d_cols,
                             void *stream);

/* Uniform start vertices on the device (Philox TAG_START stream). */
int grass_uniform_starts(uint64_t n, uint64_t count, uint64_t seed, uint32_t *d_out,
                         void *stream);

/* =========================================================================
 * Samplers.  Replace the App plugins run through doTransitParallelSampling
 * (GT/src/grass.cu:1417-2037) with the per-step sort/RLE/partition engine
 * removed: one launch runs all steps.
 * ========================================================================= */

typedef struct {
  uint32_t length;  /* steps per walk; reference RandomWalkApp::steps() = 80 */
  uint32_t layout;  /* GRASS_LAYOUT_*                                        */
  uint64_t seed;    /* Philox key                                            */
} grass_rw_params;

/* Random walk (DeepWalkApp, GT/src/apps/randomwalk/randomWalks.cu:49-81).
 * paths holds W*(L+1) vertices, column 0 the start; a walk that reaches a
 * vertex with no edges continues as GRASS_INVALID_VERTEX.  If d_edge_count
 * is not NULL, the number of sampled edges is added to it. */
int grass_rw(const grass_graph *g, const grass_rw_params *p, const uint32_t *d_starts,
             uint64_t W, uint32_t *d_paths, unsigned long long *d_edge_count, void *stream);
int grass_rw_host(const grass_graph *g, const grass_rw_params *p, const uint32_t *h_starts,
                  uint64_t W, uint32_t *h_paths, uint64_t *edges_out);
/* Traffic accounting for a walk (no reference counterpart; the reference
 * reports only wall times, GT/src/grass.cu:2127-2130).  Replays the walk of
 * grass_rw without writing paths and adds to d_out[0] the algorithmic bytes
 * (per draw: 8 offset + ceil(stream bits read / 8) + 4 path entry; 4 per
 * start entry), to d_out[1] the 32-byte sectors the reads span (+1 per draw
 * for the offset) and to d_out[2] the number of draws. */
int grass_rw_account(const grass_graph *g, const grass_rw_params *p, const uint32_t *d_starts,
                     uint64_t W, unsigned long long *d_out, void *stream);
/* Second-order (node2vec) walk: a biased walk beyond the reference, whose
 * apps are first-order only (its compressor has no edge weights, so a walk
 * is biased by its previous vertex, not weighted; GT/src/apps/randomwalk/
 * randomWalks.cu:49-81 is the first-order step this generalises).  The
 * first step is uniform.  A later step from v, having come from u, draws a
 * candidate x uniformly from N(v) and accepts it with probability
 * alpha(x) / max(1/p, 1, 1/q), alpha = 1/p if x == u, 1 if x is a neighbor
 * of u, 1/q otherwise; after max_tries rejected candidates the last one is
 * taken.  Try k of step s of walker w draws Philox(seed; s, w, w >> 32,
 * GRASS_N2V tag | k): word 0 picks the candidate ((r * d) >> 32), word 1 is
 * compared with the integer threshold floor(alpha / alpha_max * 2^32).
 * Membership in N(u) is a binary search of u's sorted neighbor list.  Paths
 * as grass_rw. */
typedef struct {
  uint32_t length;     /* steps per walk                                      */
  uint32_t layout;     /* GRASS_LAYOUT_*                                      */
  uint64_t seed;       /* Philox key                                          */
  double p, q;         /* return and in-out parameters (> 0)                  */
  uint32_t max_tries;  /* candidates per step, 1..65536 (0: 64)               */
  uint32_t reserved[3];
} grass_node2vec_params;
int grass_node2vec(const grass_graph *g, const grass_node2vec_params *p,
                   const uint32_t *d_starts, uint64_t W, uint32_t *d_paths,
                   unsigned long long *d_edge_count, void *stream);

/* Random-read probe (no reference counterpart): about `reads` independent
 * random 4-byte reads from d_buf[0, n_words) (n_words a power of two), eight
 * in flight per thread, with the loaded values summed into *d_sink; *issued
 * receives the exact number of reads.  Timed on a buffer far larger than L2,
 * it gives the device's ceiling for random 32-byte sector reads, against
 * which the samplers' dependent random reads are compared. */
int grass_random_read_probe(const uint32_t *d_buf, uint64_t n_words, uint64_t reads,
                            uint64_t seed, unsigned long long *d_sink, uint64_t *issued,
                            void *stream);

#define GRASS_MAX_HOPS 8
typedef struct {
  uint32_t hops;                    /* number of hops (reference: 2)       */
  uint32_t fanouts[GRASS_MAX_HOPS]; /* draws per transit per hop (10, 25)  */
  uint64_t seed;
} grass_khop_params;

/* k-hop with replacement (KHopApp, GT/src/apps/khop/khop.cu:1-79).  Hop h
 * output d_hop_out[h] is [S][prod_{j<=h} fanouts[j]]; slot p*f_h + k holds
 * draw k from entry p of the previous hop. */
int grass_khop(const grass_graph *g, const grass_khop_params *p, const uint32_t *d_seeds,
               uint64_t S, uint32_t *const *d_hop_out, unsigned long long *d_edge_count,
               void *stream);
int grass_khop_host(const grass_graph *g, const grass_khop_params *p, const uint32_t *h_seeds,
                    uint64_t S, uint32_t *const *h_hop_out, uint64_t *edges_out);

typedef struct {
  uint32_t walkers; /* R, walkers per sample (reference NUM_ROOT_VERTICES = 80) */
  uint32_t steps;   /* T (reference MultiRWApp::steps() = 100)                 */
  uint32_t select;  /* GRASS_SELECT_*                                          */
  uint32_t reserved;
  uint64_t seed;
} grass_mrw_params;

/* Multi random walk (MultiRWApp, GT/src/apps/multiRW/multiRW.cu:3-112).
 * d_roots [S][R] holds the walkers' start vertices and is updated in place
 * to their final positions; d_src/d_dst [S][T] receive the edge taken at each
 * step (GRASS_INVALID_VERTEX as dst when the walker's vertex has no edges). */
int grass_mrw(const grass_graph *g, const grass_mrw_params *p, uint32_t *d_roots, uint64_t S,
              uint32_t *d_src, uint32_t *d_dst, unsigned long long *d_edge_count, void *stream);
int grass_mrw_host(const grass_graph *g, const grass_mrw_params *p, uint32_t *h_roots,
                   uint64_t S, uint32_t *h_src, uint32_t *h_dst, uint64_t *edges_out);
/* Initial walker vertices for S samples of R walkers, uniform over n from the
 * Philox TAG_MRW_ROOT stream (replaces MultiRWApp::initializeSample's
 * unseeded rand() % n, GT/src/apps/multiRW/multiRW.cu:103-111). */
int grass_mrw_roots(uint64_t n, uint64_t S, uint32_t R, uint64_t seed, uint32_t *d_roots,
                    void *stream);

/* =========================================================================
 * Output compaction: a sampler's fixed-shape output to a dense edge list.
 * The reference cuts invalid walkers out of every step's frontier by a radix
 * sort and a search for the first INVALID_VERTEX (invalidVertexStartPos,
 * GT/src/grass.cu:1085-1117, launched :1641).  The samplers here write
 * fixed-shape outputs with GRASS_INVALID_VERTEX in empty slots; these calls
 * write the valid edges (src, dst) in output order -- an edge is valid when
 * its dst is not GRASS_INVALID_VERTEX -- using per-warp ballot/popc ranks and
 * one scan over 4096-entry tile counts.  Edges past `capacity` are not
 * written; *d_count (a device word) receives the total number of valid
 * edges, which equals the sampler's edge count.  The buffers must be on the
 * current device; each call takes its tile counts from a stream-ordered
 * memory pool private to this library.
 * ========================================================================= */

/* k-hop output (grass_khop / grass_csr_khop) in (hop, seed, slot) order:
 * hop 0 edges are seeds[s] -> hop0[s][k]; hop h edges are
 * hop_{h-1}[s][p] -> hop_h[s][p * fanouts[h] + k]. */
int grass_khop_edges(const grass_khop_params *p, const uint32_t *d_seeds, uint64_t S,
                     const uint32_t *const *d_hop_out, uint32_t *d_src, uint32_t *d_dst,
                     uint64_t capacity, unsigned long long *d_count, void *stream);
/* Walk paths (grass_rw / grass_csr_rw, W walks of p->length steps in
 * p->layout): edge (w, s) is paths(w, s) -> paths(w, s + 1), in (walk, step)
 * order for the walk-major layout and (step, walk) order for step-major. */
int grass_rw_edges(const grass_rw_params *p, const uint32_t *d_paths, uint64_t W,
                   uint32_t *d_src, uint32_t *d_dst, uint64_t capacity,
                   unsigned long long *d_count, void *stream);
/* Multi-RW step edges (grass_mrw, [S][p->steps] each) in (sample, step)
 * order. */
int grass_mrw_edges(const grass_mrw_params *p, uint64_t S, const uint32_t *d_step_src,
                    const uint32_t *d_step_dst, uint32_t *d_src, uint32_t *d_dst,
                    uint64_t capacity, unsigned long long *d_count, void *stream);

/* =========================================================================
 * Batched jobs: many RW / k-hop / multi-RW jobs of uneven size in ONE
 * persistent launch, captured in a CUDA graph.  The reference runs one app
 * per process through nextdoor() (GT/src/grass.cu:2066-2135); here warps of a
 * persistent kernel pull work items (walker tiles, single seeds, single
 * multi-RW samples -- the longest first) from a device queue.  Every job has
 * its own Philox seed, so each job's output equals the standalone call with
 * the same parameters (grass_rw / grass_khop / grass_mrw).
 * ========================================================================= */
#define GRASS_JOB_RW 0
#define GRASS_JOB_KHOP 1
#define GRASS_JOB_MRW 2

typedef struct {
  uint32_t type;                     /* GRASS_JOB_*                                    */
  uint32_t count;                    /* walkers (RW), seeds (k-hop), samples (MRW)     */
  uint64_t seed;                     /* Philox key of the job                          */
  const uint32_t *d_input;           /* RW starts[count] / k-hop seeds[count]          */
  uint32_t *d_roots;                 /* MRW [count][walkers]: initial walker vertices;
                                        each run restores them, then leaves the final
                                        positions                                      */
  uint32_t *d_out0;                  /* RW paths / MRW src[count][steps]               */
  uint32_t *d_out1;                  /* MRW dst[count][steps]                          */
  uint32_t *d_hops[GRASS_MAX_HOPS];  /* k-hop outputs, [count][prod fanouts]           */
  unsigned long long *d_edges;       /* optional: sampled edges of this job are added  */
  uint32_t length, layout;           /* RW                                             */
  uint32_t hops;                     /* k-hop                                          */
  uint32_t fanouts[GRASS_MAX_HOPS];
  uint32_t walkers, steps, select;   /* MRW                                            */
} grass_job;

/* Launch shape of the batched kernel; zero fields take defaults.  The
 * autotuner sweeps walker_tile x depth x warps_per_block x warps_per_vertex. */
typedef struct {
  uint32_t walker_tile;      /* RW walkers per work item: 64, 128, 256 (default 64)           */
  uint32_t depth;            /* RW walkers in flight per lane: 1, 2, 4 (default 1)            */
  uint32_t warps_per_block;  /* 1, 2, 4, 8 (default 8)                                        */
  uint32_t khop_seeds;       /* k-hop seeds per work item (default 1)                         */
  uint32_t use_graph;        /* 1 (default): replay a captured CUDA graph; 2: plain launches  */
  uint32_t warps_per_vertex; /* k-hop: warps sharing one seed vertex's expansion, split by
                                its first hop's subtrees: 1, 2, 4, 8 (default 1); the
                                counterpart of the reference's per-transit thread-block /
                                grid kernels (GT/src/grass.cu:884-1083)                   */
  uint32_t reserved[2];
} grass_batch_config;

typedef struct grass_batch grass_batch;
int grass_batch_create(const grass_graph *g, grass_batch **out);
/* The same batched launch on an uncompressed CSR (grass_csr_*): the CSR side
 * of the compressed-vs-CSR comparison for batched jobs.  Every job's output
 * equals the compressed batch's on the graph the CSR was decoded from. */
int grass_batch_create_csr(const grass_csr *c, grass_batch **out);
int grass_batch_add(grass_batch *b, const grass_job *job);
int grass_batch_clear(grass_batch *b);
int grass_batch_set_config(grass_batch *b, const grass_batch_config *cfg);
int grass_batch_get_config(const grass_batch *b, grass_batch_config *cfg);
/* Runs every job once; d_total_edges (optional) receives the total number of
 * sampled edges (added to).  Asynchronous on the stream. */
int grass_batch_run(grass_batch *b, void *stream, unsigned long long *d_total_edges);
/* Times every configuration of the sweep on this batch (each run repeats
 * the whole batch), keeps the fastest and returns it with its time in ms. */
int grass_batch_autotune(grass_batch *b, void *stream, grass_batch_config *best,
                         float *best_ms);
/* Number of work items the current jobs split into (for inspection). */
int grass_batch_info(const grass_batch *b, uint64_t *jobs, uint64_t *work_items);
int grass_batch_destroy(grass_batch *b);

/* =========================================================================
 * Serving loop (no reference counterpart: the reference runs one app per
 * process, GT/src/main.cu:28-50).  The graph stays resident; requests are
 * submitted from any thread and a dispatcher thread groups them into batches
 * of the persistent kernel above.
 *
 * Admission: a request's device scratch (input, outputs, multi-RW state) is
 * reserved when its batch launches; launched batches never hold more than
 * scratch_budget bytes together, and requests wait (FIFO) until it fits.  A
 * request larger than the whole budget fails at submit with GRASS_E_BUDGET.
 *
 * Requests form two classes with their own queues and batches: RW and k-hop
 * requests, and multi-RW requests (chains of dependent steps), so a short
 * request never finishes with a long chain that shares its batch.
 *
 * Batching window: a batch of a class closes when a stream slot is free and
 * either the class's oldest waiting request is window_min_us old while no
 * batch of its class runs, window_max_us old while one does, the class's
 * waiting work reaches target_draws sampled edges, or max_batch_jobs of its
 * requests wait.
 *
 * Results are copied to pinned host memory owned by the server (or, with
 * results_on_device, stay in device memory) and stay valid until
 * grass_server_release.  Each request's result equals the standalone call
 * with the same parameters and seed.  Unreleased host results never stall
 * new batches: when they fill the staging arena, batches stage through a
 * pinned fallback pool (counted in staging_fallbacks).  Results kept on the
 * device count against scratch_budget until released, so a caller that holds
 * them must release some before waiting on requests that need the room.
 * ========================================================================= */
typedef struct {
  uint64_t scratch_budget;   /* device bytes for launched requests, allocated at create
                                (0: 8 GiB)                                            */
  uint64_t target_draws;     /* close a batch at this much waiting work (0: 2^20)     */
  uint64_t staging_bytes;    /* pinned host arena for inputs and results, made at
                                create (0: 1 GiB); a batch carries at most 1/8 of it
                                unless one request is larger.  Results hold their
                                part until released, and batches wait for room.      */
  uint32_t window_min_us;    /* 0: 200                                                 */
  uint32_t window_max_us;    /* 0: 1000                                                */
  uint32_t max_inflight;     /* batches in flight, one stream each (0: 16, at most 16);
                                multi-RW batches take at most half of them            */
  uint32_t max_batch_jobs;   /* requests per batch (0: 4096)                           */
  grass_batch_config batch;  /* kernel shape (zero fields: defaults)                   */
  uint32_t results_on_device;/* 1: results stay in device memory (grass_result.out are
                                device pointers) until released; they count against
                                scratch_budget meanwhile.  For callers that consume
                                samples on the GPU: no device-to-host copy.         */
  uint32_t reserved[3];
} grass_server_config;

typedef struct {
  uint32_t type;                    /* GRASS_JOB_*                                     */
  uint32_t count;                   /* walkers (RW), seeds (k-hop), samples (MRW)      */
  uint64_t seed;                    /* Philox key                                      */
  const uint32_t *input;            /* host: RW starts / k-hop seeds [count]; MRW roots
                                       [count][walkers] or NULL to draw them from seed
                                       as grass_mrw_roots does.  Copied at submit.     */
  uint32_t length, layout;          /* RW                                              */
  uint32_t hops;                    /* k-hop                                           */
  uint32_t fanouts[GRASS_MAX_HOPS];
  uint32_t walkers, steps, select;  /* MRW                                             */
} grass_request;

typedef struct {
  int status;                               /* GRASS_OK or the request's error          */
  uint32_t n_outputs;                       /* RW 1, k-hop hops, MRW 2 (src, dst)       */
  const uint32_t *out[GRASS_MAX_HOPS];      /* host pointers, owned by the server       */
  uint64_t out_words[GRASS_MAX_HOPS];
  uint64_t edges;                           /* sampled edges                            */
  double submit_us, launch_us, done_us;     /* since grass_server_create                */
  uint64_t batch;                           /* batch sequence number                    */
  uint32_t on_device;                       /* out[] are device pointers                */
  uint32_t reserved;
} grass_result;

typedef struct {
  uint64_t submitted, completed, rejected, failed, batches, edges;
  uint64_t waiting, running, scratch_in_use, scratch_peak;
  double busy_us;                           /* time with at least one batch in flight  */
  double issue_us;                          /* dispatcher time issuing batches         */
  double staging_alloc_us;                  /* of which pinned staging allocation      */
  double phase_us[6];                       /* issue time by step: pool allocation,
                                               staging fill, H2D enqueue, kernel launch,
                                               D2H enqueue, free + completion callback  */
  uint64_t staging_fallbacks;               /* batches staged through the pinned fallback
                                               pool because unreleased results held the
                                               staging arena                             */
} grass_server_stats;

typedef struct grass_server grass_server;
int grass_server_create(const grass_graph *g, const grass_server_config *cfg,
                        grass_server **out);
/* Queues a request; *ticket identifies it.  Never blocks on the GPU. */
int grass_server_submit(grass_server *s, const grass_request *r, uint64_t *ticket);
/* *done = 1 once the request finished (successfully or not). */
int grass_server_poll(grass_server *s, uint64_t ticket, int *done);
/* Waits up to timeout_ms; GRASS_E_TIMEOUT if the request is still running.
 * res (optional) receives the result; its status is the request's. */
int grass_server_wait(grass_server *s, uint64_t ticket, uint32_t timeout_ms, grass_result *res);
/* Frees a finished request's result memory. */
int grass_server_release(grass_server *s, uint64_t ticket);
int grass_server_stats_get(grass_server *s, grass_server_stats *st);
/* Fails the requests not yet launched with GRASS_E_TIMEOUT, waits up to
 * timeout_ms for the running batches, then stops the dispatcher thread and
 * frees the streams, arenas and results.  If batches are still running when
 * timeout_ms ends it returns GRASS_E_TIMEOUT and frees nothing (the
 * dispatcher and the batches' callbacks still use the server): the server
 * accepts no new requests and the caller calls grass_server_destroy again. */
int grass_server_destroy(grass_server *s, uint32_t timeout_ms);

/* Open-loop load generator for the serving loop: Poisson arrivals at `rate`
 * requests/s; each request's type, size and parameters are drawn as below
 * from the trace seed, and its Philox seed and start vertices from its own
 * index.  mode 0 drives a grass_server; mode 1 serves the same trace with one
 * standalone launch per request (grass_rw / grass_khop / grass_mrw, one
 * stream, inputs and outputs copied per request), the plain method. */
typedef struct {
  double rate;                  /* requests per second                               */
  uint32_t requests;            /* trace length                                       */
  uint32_t mode;                /* 0 server, 1 one job per launch                     */
  uint64_t seed;                /* trace seed                                         */
  uint32_t pct_rw, pct_khop;    /* percent of RW and k-hop requests; the rest are MRW */
  double size_mu, size_sigma;   /* RW walkers / k-hop seeds ~ lognormal(mu, sigma)    */
  uint32_t size_max;            /* clipped to [1, size_max]                           */
  uint32_t rw_len_min, rw_len_max;
  uint32_t n_fanouts;           /* k-hop fanout sets to choose from (at most 8)       */
  uint32_t fanouts[8][4];       /* zero-terminated                                    */
  uint32_t mrw_samples, mrw_walkers, mrw_steps, mrw_select;
  uint32_t timeout_ms;          /* bound on the wait for any one request              */
  grass_server_config server;
} grass_loadgen_config;

typedef struct {
  uint64_t completed, rejected, failed, batches;
  double p50_us, p99_us, p999_us, mean_us, max_us;
  double p50_type_us[3], p99_type_us[3];  /* per GRASS_JOB_* type                      */
  double queue_p50_us, queue_p99_us;      /* arrival to launch (server mode)             */
  double service_p50_us, service_p99_us;  /* launch to done (server mode)                */
  double issue_us, staging_alloc_us;      /* server: dispatcher time issuing batches     */
  double phase_us[6];                     /* server: issue time by step (see stats)       */
  double wall_s;                /* first arrival to last completion                   */
  double edges;                 /* sampled edges of completed requests                */
  double edges_per_s;           /* edges / wall_s                                     */
  double offered_rate, achieved_rate;
  uint64_t launches;            /* kernel launches of this run                        */
} grass_loadgen_report;

int grass_loadgen_run(const grass_graph *g, const grass_loadgen_config *c,
                      grass_loadgen_report *r);

/* =========================================================================
 * Uncompressed-CSR baseline with the same RNG streams (no reference
 * counterpart: the reference's NextDoor CSR loaders, GT/src/graph.hpp, are
 * never called).  Produces the same walks as the compressed sampler.
 * ========================================================================= */
int grass_csr_from_graph(const grass_graph *g, grass_csr **out);
int grass_csr_from_host(const uint64_t *rowptr, const uint32_t *cols, uint64_t n, int device,
                        grass_csr **out);
int grass_csr_close(grass_csr *c);
int grass_csr_info(const grass_csr *c, uint64_t *n, uint64_t *nnz, uint64_t *device_bytes);
int grass_csr_set_tuning(grass_csr *c, const grass_tuning *t);
int grass_csr_rw(const grass_csr *c, const grass_rw_params *p, const uint32_t *d_starts,
                 uint64_t W, uint32_t *d_paths, unsigned long long *d_edge_count, void *stream);
int grass_csr_khop(const grass_csr *c, const grass_khop_params *p, const uint32_t *d_seeds,
                   uint64_t S, uint32_t *const *d_hop_out, unsigned long long *d_edge_count,
                   void *stream);
int grass_csr_node2vec(const grass_csr *c, const grass_node2vec_params *p,
                       const uint32_t *d_starts, uint64_t W, uint32_t *d_paths,
                       unsigned long long *d_edge_count, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GRASS_B200_H */
