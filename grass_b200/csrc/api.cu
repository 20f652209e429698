// api.cu -- extern "C" entry points of the grass_b200 library (see
// include/grass.h for the contract and the reference interfaces replaced).
#include <stdio.h>
#include <string.h>
#include <sys/stat.h>

#include <algorithm>
#include <cmath>
#include <chrono>
#include <mutex>
#include <string>
#include <vector>

#include "graph.h"

namespace grass {

std::atomic<uint64_t> g_launches{0};
static thread_local std::string t_err;

int set_error(int code, const char *fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_err = buf;
  return code;
}

void clear_error() { t_err.clear(); }

int cuda_fail(cudaError_t e, const char *what) {
  return set_error(e == cudaErrorMemoryAllocation ? GRASS_E_OOM : GRASS_E_CUDA, "%s: %s", what,
                   cudaGetErrorString(e));
}

// Stream-ordered scratch for this library's kernels, from a memory pool of
// its own on each device.  The pool keeps up to 256 MiB of freed memory
// mapped across synchronisations: the default pool returns freed memory at
// every synchronisation, so the first allocation after one maps fresh memory,
// which measured 0.2-1.2 ms on a 60 KB request against a 0.1 ms compaction.
cudaError_t scratch_alloc(void **p, size_t bytes, cudaStream_t s) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, s);
  cudaMemPool_t pool;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&pools[dev], &props);
      if (e != cudaSuccess) {
        pools[dev] = nullptr;
        return e;
      }
      uint64_t keep = 256ull << 20;
      cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    }
    pool = pools[dev];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

void scratch_free(void *p, cudaStream_t s) { cudaFreeAsync(p, s); }

int sm_count(int device) {
  static int cache[64] = {0};
  if (device < 0 || device >= 64) return 148;
  if (!cache[device]) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || !v)
      v = 148;
    cache[device] = v;
  }
  return cache[device];
}

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// Field u of the .offset payload (MSB-first ubl-bit fields) read on the host.
uint64_t host_field(const uint8_t *pay, uint64_t pay_size, uint64_t u, uint32_t ubl) {
  uint64_t v = 0;
  const uint64_t bit0 = u * ubl;
  for (uint32_t k = 0; k < ubl; k++) {
    const uint64_t b = bit0 + k;
    const uint64_t byte = b >> 3;
    const uint32_t bitv = byte < pay_size ? (pay[byte] >> (7 - (b & 7))) & 1u : 0u;
    v = (v << 1) | bitv;
  }
  return v;
}

// Source of .graph bytes: a file or a memory image.
struct ByteSource {
  FILE *f = nullptr;
  const uint8_t *mem = nullptr;
  uint64_t size = 0, pos = 0;
  double read_s = 0;
  size_t read(uint8_t *dst, size_t want) {
    want = (size_t)std::min<uint64_t>(want, size - pos);
    double t0 = now_s();
    size_t got = want;
    if (f) got = fread(dst, 1, want, f);
    else memcpy(dst, mem + pos, want);
    read_s += now_s() - t0;
    pos += got;
    return got;
  }
};

struct Temps {
  std::vector<void *> dev;
  std::vector<void *> pinned;
  ~Temps() {
    for (void *p : dev) cudaFree(p);
    for (void *p : pinned) cudaFreeHost(p);
  }
};

int open_impl(ByteSource &src, const uint8_t *ob, uint64_t osize, int mode, int device,
              grass_graph **out) {
  if (mode != GRASS_MODE_GT && mode != GRASS_MODE_LE)
    return set_error(GRASS_E_ARG, "mode must be GRASS_MODE_GT or GRASS_MODE_LE");
  if (osize < 2) return set_error(GRASS_E_FORMAT, ".offset holds no length fields");
  const uint32_t ubl = ob[0];
  if (ubl < 1 || ubl > 64) return set_error(GRASS_E_FORMAT, "bad length-field width %u", ubl);
  const uint8_t *pay = ob + 1;
  const uint64_t pay_size = osize - 1;
  const uint64_t n_file = pay_size * 8 / ubl;
  // Trailing zero-length fields are byte padding (a real vertex encodes at
  // least one bit); the reference counts them as vertices.
  uint64_t n = n_file;
  while (n > 0 && host_field(pay, pay_size, n - 1, ubl) == 0) n--;
  if (n == 0) return set_error(GRASS_E_FORMAT, "graph has no vertices");
  if (n > 0xFFFFFFFEull) return set_error(GRASS_E_FORMAT, "more than 2^32-2 vertices");

  int ndev = 0;
  GRASS_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return set_error(GRASS_E_ARG, "no CUDA device %d", device);
  DeviceGuard dg(device);
  const double t0 = now_s();
  cudaStream_t st;
  GRASS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  struct StreamGuard {
    cudaStream_t s;
    ~StreamGuard() { cudaStreamDestroy(s); }
  } sg{st};

  auto *g = new (std::nothrow) grass_graph();
  if (!g) return set_error(GRASS_E_OOM, "host allocation failed");
  struct GraphGuard {
    grass_graph *g;
    ~GraphGuard() {
      if (g) {
        cudaFree(g->d_words);
        cudaFree(g->d_offsets);
        cudaFree(g->d_recs);
        cudaFree(g->d_err);
        delete g;
      }
    }
  } gg{g};
  g->device = device;
  g->mode = mode;
  const uint64_t gsize = src.size;
  g->n_words = (gsize + 3) / 4;
  // whole 32-byte sectors, at least one full zero sector past the stream
  // (sector loads may touch the sector after the one holding a field start)
  const uint64_t alloc_words = (g->n_words + kGuardWords + 7) / 8 * 8;
  GRASS_CUDA(cudaMalloc(&g->d_words, alloc_words * 4));
  GRASS_CUDA(cudaMalloc(&g->d_offsets, (n + 1) * sizeof(uint64_t)));
  GRASS_CUDA(cudaMalloc(&g->d_err, sizeof(unsigned int)));
  GRASS_CUDA(cudaMemsetAsync(g->d_err, 0, sizeof(unsigned int), st));
  // zero the tail (partial last word + guard words)
  const uint64_t tail_word = gsize / 4;
  GRASS_CUDA(cudaMemsetAsync(g->d_words + tail_word, 0, (alloc_words - tail_word) * 4, st));

  // Double-buffered pinned upload of the stream bytes.
  Temps tmp;
  const size_t chunk = 64ull << 20;
  uint8_t *pin[2] = {nullptr, nullptr};
  cudaEvent_t ev[2];
  for (int i = 0; i < 2; i++) {
    GRASS_CUDA(cudaMallocHost(&pin[i], chunk));
    tmp.pinned.push_back(pin[i]);
    GRASS_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
  }
  struct EvGuard {
    cudaEvent_t *e;
    ~EvGuard() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } eg{ev};
  bool used[2] = {false, false};
  uint64_t off = 0;
  int k = 0;
  while (off < gsize) {
    if (used[k]) GRASS_CUDA(cudaEventSynchronize(ev[k]));
    const size_t got = src.read(pin[k], chunk);
    if (got == 0) return set_error(GRASS_E_IO, "short read of .graph");
    GRASS_CUDA(cudaMemcpyAsync(reinterpret_cast<uint8_t *>(g->d_words) + off, pin[k], got,
                               cudaMemcpyHostToDevice, st));
    GRASS_CUDA(cudaEventRecord(ev[k], st));
    used[k] = true;
    off += got;
    k ^= 1;
  }
  launch_bswap(g->d_words, g->n_words, st);

  // .offset payload -> words -> lengths -> exclusive scan.
  const uint64_t opay_words = (pay_size + 3) / 4 + kGuardWords;
  uint32_t *d_opay = nullptr;
  GRASS_CUDA(cudaMalloc(&d_opay, opay_words * 4));
  tmp.dev.push_back(d_opay);
  GRASS_CUDA(cudaMemsetAsync(d_opay, 0, opay_words * 4, st));
  GRASS_CUDA(cudaMemcpyAsync(d_opay, pay, pay_size, cudaMemcpyHostToDevice, st));
  launch_bswap(d_opay, (pay_size + 3) / 4, st);
  uint64_t *d_scan = nullptr;
  GRASS_CUDA(cudaMalloc(&d_scan, (scan_tmp_words(n) + 1) * sizeof(uint64_t)));
  tmp.dev.push_back(d_scan);
  launch_unpack_scan(d_opay, n, ubl, g->d_offsets, d_scan, st);
  uint64_t total_bits = 0;
  GRASS_CUDA(cudaMemcpyAsync(&total_bits, g->d_offsets + n, sizeof(uint64_t),
                             cudaMemcpyDeviceToHost, st));
  GRASS_CUDA(cudaStreamSynchronize(st));
  if (total_bits > gsize * 8)
    return set_error(GRASS_E_FORMAT, ".offset lengths sum to %llu bits but .graph holds %llu",
                     (unsigned long long)total_bits, (unsigned long long)(gsize * 8));

  g->info.n = n;
  unsigned long long *d_stats = nullptr;
  GRASS_CUDA(cudaMalloc(&d_stats, 3 * sizeof(unsigned long long)));
  tmp.dev.push_back(d_stats);
  unsigned long long init[3] = {0, 0, ~0ull};
  GRASS_CUDA(cudaMemcpyAsync(d_stats, init, sizeof init, cudaMemcpyHostToDevice, st));
  launch_validate(g->view(), nullptr, d_stats, st);
  unsigned long long stats[3];
  GRASS_CUDA(cudaMemcpyAsync(stats, d_stats, sizeof stats, cudaMemcpyDeviceToHost, st));
  GRASS_CUDA(cudaStreamSynchronize(st));
  GRASS_CUDA(cudaGetLastError());
  if (stats[2] != ~0ull)
    return set_error(GRASS_E_FORMAT,
                     "vertex %llu: header does not match its length field (wrong mode or "
                     "corrupt file?)",
                     stats[2]);

  // Vertex records replace the bit-offset table for everything after load.
  GRASS_CUDA(cudaMalloc(&g->d_recs, n * sizeof(uint4)));
  launch_build_records(g->view(), g->d_recs, st);
  GRASS_CUDA(cudaStreamSynchronize(st));
  GRASS_CUDA(cudaGetLastError());
  cudaFree(g->d_offsets);
  g->d_offsets = nullptr;

  // The device layout: every vertex re-chunked into sector-sized slots
  // (device_common.cuh), built from the decoded neighbor lists; it replaces
  // the on-disk stream.
  uint64_t words_alloc = alloc_words;
  {
    Nvtx nv("device layout");
    const uint64_t E = stats[0];
    uint64_t *d_rp = nullptr, *d_P = nullptr;
    uint32_t *d_cl = nullptr, *d_meta = nullptr, *d_fp = nullptr;
    GRASS_CUDA(cudaMalloc(&d_rp, (n + 1) * sizeof(uint64_t)));
    tmp.dev.push_back(d_rp);
    GRASS_CUDA(cudaMalloc(&d_cl, std::max<uint64_t>(E, 1) * 4));
    tmp.dev.push_back(d_cl);
    GRASS_CUDA(cudaMalloc(&d_meta, n * 4));
    tmp.dev.push_back(d_meta);
    GRASS_CUDA(cudaMalloc(&d_fp, n * 4));
    tmp.dev.push_back(d_fp);
    GRASS_CUDA(cudaMalloc(&d_P, n * sizeof(uint64_t)));
    tmp.dev.push_back(d_P);
    launch_degrees64(g->view(), d_rp, st);
    launch_scan_u64_inplace(d_rp, n, d_scan, st);
    launch_disk_decode(mode, g->d_words, g->d_recs, (uint32_t)n, d_rp, d_cl, st);
    launch_slot_choose(mode, d_rp, d_cl, (uint32_t)n, d_meta, d_fp, st);
    std::vector<uint32_t> meta(n);
    std::vector<uint64_t> rp(n + 1), P(n, 0);
    GRASS_CUDA(cudaMemcpyAsync(meta.data(), d_meta, n * 4, cudaMemcpyDeviceToHost, st));
    GRASS_CUDA(cudaMemcpyAsync(rp.data(), d_rp, (n + 1) * 8, cudaMemcpyDeviceToHost, st));
    GRASS_CUDA(cudaStreamSynchronize(st));
    GRASS_CUDA(cudaGetLastError());
    // First fit in vertex order: a vertex whose slots fit in one sector goes
    // at the current bit if it does not cross the sector end; a larger one
    // starts on the next sector.  Slots: GT ceil(d / T), LE ceil((d - 1) / T)
    // (an LE vertex of degree 1 keeps its neighbor in the record).
    const bool gt = mode == GRASS_MODE_GT;
    uint64_t pos = 0;
    for (uint64_t v = 0; v < n; v++) {
      const uint64_t d = rp[v + 1] - rp[v];
      if (d < (gt ? 1u : 2u)) continue;
      const uint32_t m = meta[v];
      const uint64_t T = m & 0xFFu, b = (m >> 8) & 0xFFu, K = (m >> 16) & 0xFFu, a = m >> 24;
      const uint64_t cb = gt ? a + (T - 1) * b : 2 * a + (T - 1) * (b + 1);
      const uint64_t C = gt ? (d - 1) / T + 1 : (d - 2) / T + 1;
      if (C <= K) {
        if ((pos & 255) + C * cb > 256) pos = (pos + 255) & ~255ull;
      } else {
        pos = (pos + 255) & ~255ull;
      }
      P[v] = pos;
      pos += (C / K) * 256 + (C % K) * cb;
    }
    if (pos >= (1ull << 40))
      return set_error(GRASS_E_FORMAT, "device layout needs %llu bits (limit 2^40)",
                       (unsigned long long)pos);
    const uint64_t nw = (pos + 31) / 32;
    words_alloc = (nw + kGuardWords + 7) / 8 * 8;
    uint32_t *d_slots = nullptr;
    GRASS_CUDA(cudaMalloc(&d_slots, words_alloc * 4));
    tmp.dev.push_back(d_slots);
    GRASS_CUDA(cudaMemsetAsync(d_slots, 0, words_alloc * 4, st));
    GRASS_CUDA(cudaMemcpyAsync(d_P, P.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
    launch_slot_write(mode, d_rp, d_cl, (uint32_t)n, d_meta, d_fp, d_P, d_slots, g->d_recs, st);
    GRASS_CUDA(cudaStreamSynchronize(st));
    GRASS_CUDA(cudaGetLastError());
    tmp.dev.back() = g->d_words;  // the on-disk stream is freed with tmp
    g->d_words = d_slots;
    g->n_words = nw;
  }

  g->info.n_file = n_file;
  g->info.num_edges = stats[0];
  g->info.max_degree = (uint32_t)stats[1];
  g->info.ubl = ubl;
  g->info.mode = mode;
  g->info.device = device;
  g->info.graph_file_bytes = gsize;
  g->info.offset_file_bytes = osize;
  g->info.device_bytes = words_alloc * 4 + n * sizeof(uint4);
  g->info.read_seconds = src.read_s;
  g->info.upload_seconds = now_s() - t0;
  *out = g;
  gg.g = nullptr;
  return GRASS_OK;
}

bool read_whole(const std::string &path, std::vector<uint8_t> &buf) {
  FILE *f = fopen(path.c_str(), "rb");
  if (!f) return false;
  fseek(f, 0, SEEK_END);
  long s = ftell(f);
  fseek(f, 0, SEEK_SET);
  buf.resize(s > 0 ? (size_t)s : 0);
  bool ok = s >= 0 && (s == 0 || fread(buf.data(), 1, (size_t)s, f) == (size_t)s);
  fclose(f);
  return ok;
}

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// CSR row pointers are read a 32-byte sector at a time (csr_row): whole
// sectors plus one spare.
size_t csr_rowptr_bytes(uint64_t n) { return ((n + 1 + 3) / 4 * 4 + 4) * sizeof(uint64_t); }

int check_launch() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? GRASS_OK : cuda_fail(e, "kernel launch");
}

int check_graph(const grass_graph *g) {
  if (!g) return set_error(GRASS_E_ARG, "null graph");
  return GRASS_OK;
}

int check_khop(const grass_khop_params *p, uint64_t *width_out) {
  if (!p || p->hops == 0 || p->hops > GRASS_MAX_HOPS)
    return set_error(GRASS_E_ARG, "k-hop: hops must be in [1, %d]", GRASS_MAX_HOPS);
  uint64_t w = 1;
  for (uint32_t h = 0; h < p->hops; h++) {
    if (p->fanouts[h] == 0) return set_error(GRASS_E_ARG, "k-hop: fanout %u is zero", h);
    w *= p->fanouts[h];
    if (w > (1ull << 32)) return set_error(GRASS_E_ARG, "k-hop: fanout product too large");
    width_out[h] = w;
  }
  return GRASS_OK;
}

// Device buffer owned for the duration of a _host call.
struct DevBuf {
  void *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};

int read_err_flag(const grass_graph *g, cudaStream_t st) {
  unsigned int e = 0;
  GRASS_CUDA(cudaMemcpyAsync(&e, g->d_err, sizeof e, cudaMemcpyDeviceToHost, st));
  GRASS_CUDA(cudaStreamSynchronize(st));
  if (e) {
    cudaMemsetAsync(g->d_err, 0, sizeof(unsigned int), st);
    cudaStreamSynchronize(st);
    if (e & 2u)
      return set_error(GRASS_E_TIMEOUT, "a decode warp's staged stream copy did not complete");
    return set_error(GRASS_E_DATA, "a decoded vertex id was out of range (corrupt payload)");
  }
  return GRASS_OK;
}

}  // namespace
}  // namespace grass

using namespace grass;

extern "C" {

const char *grass_last_error(void) { return grass::t_err.c_str(); }
uint64_t grass_launch_count(void) { return grass::g_launches.load(); }
const char *grass_version(void) { return "grass_b200 0.1 (sm_100a)"; }

int grass_open(const char *prefix, int mode, int device, grass_graph **out) {
  grass::Nvtx nvtx_("grass_open");
  clear_error();
  if (!prefix || !out) return set_error(GRASS_E_ARG, "null argument");
  *out = nullptr;
  const std::string p(prefix);
  std::vector<uint8_t> ob;
  FILE *gf = fopen((p + ".graph").c_str(), "rb");
  if (!gf) return set_error(GRASS_E_IO, "Open graph file failed: %s.graph", prefix);
  if (!read_whole(p + ".offset", ob)) {
    fclose(gf);
    return set_error(GRASS_E_IO, "Open offset file failed: %s.offset", prefix);
  }
  fseek(gf, 0, SEEK_END);
  ByteSource src;
  src.f = gf;
  src.size = (uint64_t)ftell(gf);
  fseek(gf, 0, SEEK_SET);
  int rc = open_impl(src, ob.data(), ob.size(), mode, device, out);
  fclose(gf);
  return rc;
}

int grass_open_mem(const void *graph_bytes, uint64_t graph_size, const void *offset_bytes,
                   uint64_t offset_size, int mode, int device, grass_graph **out) {
  grass::Nvtx nvtx_("grass_open_mem");
  clear_error();
  if (!out || (!graph_bytes && graph_size) || !offset_bytes)
    return set_error(GRASS_E_ARG, "null argument");
  *out = nullptr;
  ByteSource src;
  src.mem = static_cast<const uint8_t *>(graph_bytes);
  src.size = graph_size;
  return open_impl(src, static_cast<const uint8_t *>(offset_bytes), offset_size, mode, device,
                   out);
}

int grass_close(grass_graph *g) {
  if (!g) return GRASS_OK;
  DeviceGuard dg(g->device);
  delete g->pipe;
  cudaFree(g->d_words);
  cudaFree(g->d_offsets);
  cudaFree(g->d_recs);
  cudaFree(g->d_err);
  cudaFree(g->d_plan_big);
  cudaFree(g->d_plan_small);
  cudaFree(g->d_plan_flat);
  delete g;
  return GRASS_OK;
}

int grass_check_device_error(grass_graph *g, void *stream) {
  clear_error();
  if (!g) return set_error(GRASS_E_ARG, "null graph");
  DeviceGuard dg(g->device);
  return read_err_flag(g, as_stream(stream));
}

int grass_get_info(const grass_graph *g, grass_graph_info *info) {
  if (!g || !info) return set_error(GRASS_E_ARG, "null argument");
  *info = g->info;
  return GRASS_OK;
}

int grass_device_view(const grass_graph *g, const uint32_t **words, uint64_t *n_words,
                      const void **records) {
  if (!g) return set_error(GRASS_E_ARG, "null graph");
  if (words) *words = g->d_words;
  if (n_words) *n_words = g->n_words;
  if (records) *records = g->d_recs;
  return GRASS_OK;
}

int grass_set_tuning(grass_graph *g, const grass_tuning *t) {
  if (!g || !t) return set_error(GRASS_E_ARG, "null argument");
  if (t->rw_depth && t->rw_depth != 1 && t->rw_depth != 2 && t->rw_depth != 4)
    return set_error(GRASS_E_ARG, "rw_depth must be 1, 2 or 4");
  if (t->rw_threads && (t->rw_threads % 32 || t->rw_threads > 512))
    return set_error(GRASS_E_ARG, "rw_threads must be a multiple of 32 up to 512");
  if (t->decode_stage_depth > 4 || t->decode_stage_depth == 3)
    return set_error(GRASS_E_ARG, "decode_stage_depth must be 0 (default), 1, 2 or 4");
  DeviceGuard dg(g->device);
  if (int rc = apply_tuning(g->device, *t, g->d_recs, g->info.n * sizeof(uint4), g->l2win))
    return rc;
  g->tuning = *t;
  return GRASS_OK;
}

int grass_get_tuning(const grass_graph *g, grass_tuning *t) {
  if (!g || !t) return set_error(GRASS_E_ARG, "null argument");
  *t = resolve_tuning(g->tuning, g->mode);
  return GRASS_OK;
}

int grass_degrees(const grass_graph *g, uint32_t *d_deg, void *stream) {
  grass::Nvtx nvtx_("grass_degrees");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  if (!d_deg) return set_error(GRASS_E_ARG, "null output");
  DeviceGuard dg(g->device);
  launch_degrees(g->view(), d_deg, as_stream(stream));
  return check_launch();
}

int grass_decode_all(const grass_graph *g, uint64_t *d_rowptr, uint32_t *d_cols, void *stream) {
  grass::Nvtx nvtx_("grass_decode_all");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  if (!d_rowptr || (!d_cols && g->info.num_edges)) return set_error(GRASS_E_ARG, "null output");
  DeviceGuard dg(g->device);
  cudaStream_t st = as_stream(stream);
  const uint64_t n = g->info.n;
  // degrees as u64 straight into rowptr, scanned in place, then decode;
  // the only scratch is one u64 per 4096-vertex tile.
  uint64_t *scan_tmp = nullptr;
  GRASS_CUDA(scratch_alloc(reinterpret_cast<void **>(&scan_tmp),
                           (scan_tmp_words(n) + 1) * sizeof(uint64_t), st));
  launch_degrees64(g->view(), d_rowptr, st);
  launch_scan_u64_inplace(d_rowptr, n, scan_tmp, st);
  int rc = launch_decode_planned(g, d_rowptr, d_cols, g->d_err, st);
  scratch_free(scan_tmp, st);
  return rc ? rc : check_launch();
}

int grass_uniform_starts(uint64_t n, uint64_t count, uint64_t seed, uint32_t *d_out,
                         void *stream) {
  clear_error();
  if (!n || n > 0xFFFFFFFFull || (count && !d_out)) return set_error(GRASS_E_ARG, "bad arguments");
  launch_uniform_starts(n, count, seed, d_out, as_stream(stream));
  return check_launch();
}

int grass_mrw_roots(uint64_t n, uint64_t S, uint32_t R, uint64_t seed, uint32_t *d_roots,
                    void *stream) {
  clear_error();
  if (!n || n > 0xFFFFFFFFull || (S && R && !d_roots)) return set_error(GRASS_E_ARG, "bad arguments");
  launch_uniform_starts(n, S * (uint64_t)R, seed, d_roots, as_stream(stream), true);
  return check_launch();
}

namespace {
int run_compact(const CompactSeg *segs, uint32_t nseg, uint32_t *d_src, uint32_t *d_dst,
                uint64_t capacity, unsigned long long *d_count, void *stream) {
  if (!d_count) return set_error(GRASS_E_ARG, "compaction: null count");
  if (capacity && (!d_src || !d_dst)) return set_error(GRASS_E_ARG, "compaction: null output");
  if (int rc = launch_compact(segs, nseg, d_src, d_dst, capacity, d_count, as_stream(stream)))
    return rc;
  return check_launch();
}
}  // namespace

int grass_khop_edges(const grass_khop_params *p, const uint32_t *d_seeds, uint64_t S,
                     const uint32_t *const *d_hop_out, uint32_t *d_src, uint32_t *d_dst,
                     uint64_t capacity, unsigned long long *d_count, void *stream) {
  grass::Nvtx nvtx_("grass_khop_edges");
  clear_error();
  uint64_t width[GRASS_MAX_HOPS];
  if (int rc = check_khop(p, width)) return rc;
  if (S > (1ull << 32)) return set_error(GRASS_E_ARG, "k-hop edges: more than 2^32 seeds");
  if (S && (!d_seeds || !d_hop_out)) return set_error(GRASS_E_ARG, "k-hop edges: null buffers");
  CompactSeg segs[GRASS_MAX_HOPS];
  for (uint32_t h = 0; h < p->hops; h++) {
    if (S && !d_hop_out[h]) return set_error(GRASS_E_ARG, "k-hop edges: null output for hop %u", h);
    segs[h] = CompactSeg{h ? d_hop_out[h - 1] : d_seeds, S ? d_hop_out[h] : nullptr,
                         S * width[h], 0, p->fanouts[h], kCompactFan};
  }
  return run_compact(segs, p->hops, d_src, d_dst, capacity, d_count, stream);
}

int grass_rw_edges(const grass_rw_params *p, const uint32_t *d_paths, uint64_t W,
                   uint32_t *d_src, uint32_t *d_dst, uint64_t capacity,
                   unsigned long long *d_count, void *stream) {
  grass::Nvtx nvtx_("grass_rw_edges");
  clear_error();
  if (!p || p->layout > 1 || (W && !d_paths))
    return set_error(GRASS_E_ARG, "walk edges: bad arguments");
  if (W > (1ull << 40)) return set_error(GRASS_E_ARG, "walk edges: too many walks");
  const uint64_t n = W * p->length;
  CompactSeg sg;
  if (p->layout == GRASS_LAYOUT_WALK_MAJOR)
    sg = CompactSeg{d_paths, d_paths, n, 0, p->length, kCompactPath};
  else  // step-major: column s + 1 starts W entries after column s
    sg = CompactSeg{d_paths, n ? d_paths + W : nullptr, n, 0, 1, kCompactFan};
  return run_compact(&sg, 1, d_src, d_dst, capacity, d_count, stream);
}

int grass_mrw_edges(const grass_mrw_params *p, uint64_t S, const uint32_t *d_step_src,
                    const uint32_t *d_step_dst, uint32_t *d_src, uint32_t *d_dst,
                    uint64_t capacity, unsigned long long *d_count, void *stream) {
  grass::Nvtx nvtx_("grass_mrw_edges");
  clear_error();
  if (!p || (S && p->steps && (!d_step_src || !d_step_dst)))
    return set_error(GRASS_E_ARG, "multi-RW edges: bad arguments");
  if (S > (1ull << 40)) return set_error(GRASS_E_ARG, "multi-RW edges: too many samples");
  CompactSeg sg{d_step_src, d_step_dst, S * p->steps, 0, 1, kCompactFan};
  return run_compact(&sg, 1, d_src, d_dst, capacity, d_count, stream);
}

int grass_rw(const grass_graph *g, const grass_rw_params *p, const uint32_t *d_starts,
             uint64_t W, uint32_t *d_paths, unsigned long long *d_edge_count, void *stream) {
  grass::Nvtx nvtx_("grass_rw");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  if (!p || p->layout > 1 || (W && (!d_starts || !d_paths)))
    return set_error(GRASS_E_ARG, "random walk: bad arguments");
  DeviceGuard dg(g->device);
  launch_rw(g->view(), *p, d_starts, W, d_paths, d_edge_count, g->d_err, as_stream(stream),
            g->tuning, g->l2win);
  return check_launch();
}

// node2vec acceptance thresholds: floor(alpha / alpha_max * 2^32) for alpha
// = 1/p (return), 1 (a neighbor of the previous vertex), 1/q (farther); the
// largest is exactly 2^32 (always accepted).  The oracle computes the same.
static int node2vec_args(const grass_node2vec_params *p, grass_node2vec_params &r,
                         uint64_t t[3]) {
  if (!p || p->layout > 1 || !(p->p > 0.0) || !(p->q > 0.0) || !std::isfinite(p->p) ||
      !std::isfinite(p->q) || p->max_tries > 65536u)
    return set_error(GRASS_E_ARG, "node2vec: bad parameters");
  r = *p;
  if (!r.max_tries) r.max_tries = 64;
  const double a[3] = {1.0 / r.p, 1.0, 1.0 / r.q};
  const double amax = std::max(a[0], std::max(a[1], a[2]));
  for (int k = 0; k < 3; k++) t[k] = (uint64_t)(a[k] / amax * 4294967296.0);
  return GRASS_OK;
}

int grass_node2vec(const grass_graph *g, const grass_node2vec_params *p,
                   const uint32_t *d_starts, uint64_t W, uint32_t *d_paths,
                   unsigned long long *d_edge_count, void *stream) {
  grass::Nvtx nvtx_("grass_node2vec");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  grass_node2vec_params r;
  uint64_t t[3];
  if (int rc = node2vec_args(p, r, t)) return rc;
  if (W && (!d_starts || !d_paths)) return set_error(GRASS_E_ARG, "node2vec: null buffers");
  DeviceGuard dg(g->device);
  launch_node2vec(g->view(), r, t, d_starts, W, d_paths, d_edge_count, g->d_err,
                  as_stream(stream));
  return check_launch();
}

int grass_rw_account(const grass_graph *g, const grass_rw_params *p, const uint32_t *d_starts,
                     uint64_t W, unsigned long long *d_out, void *stream) {
  clear_error();
  if (int rc = check_graph(g)) return rc;
  if (!p || !d_out || (W && !d_starts)) return set_error(GRASS_E_ARG, "bad arguments");
  DeviceGuard dg(g->device);
  launch_rw_account(g->view(), *p, d_starts, W, d_out, as_stream(stream));
  return check_launch();
}

int grass_random_read_probe(const uint32_t *d_buf, uint64_t n_words, uint64_t reads,
                            uint64_t seed, unsigned long long *d_sink, uint64_t *issued,
                            void *stream) {
  clear_error();
  if (!d_buf || !d_sink || !n_words || (n_words & (n_words - 1)))
    return set_error(GRASS_E_ARG, "random-read probe: n_words must be a power of two");
  const uint64_t k = launch_random_read(d_buf, n_words, reads, seed, d_sink, as_stream(stream));
  if (issued) *issued = k;
  return check_launch();
}

int grass_rw_host(const grass_graph *g, const grass_rw_params *p, const uint32_t *h_starts,
                  uint64_t W, uint32_t *h_paths, uint64_t *edges_out) {
  grass::Nvtx nvtx_("grass_rw_host");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  if (!p || p->layout > 1 || (W && (!h_starts || !h_paths)))
    return set_error(GRASS_E_ARG, "random walk: bad arguments");
  DeviceGuard dg(g->device);
  auto *gm = const_cast<grass_graph *>(g);
  if (!gm->pipe) {
    static std::mutex create_mu;
    std::lock_guard<std::mutex> lk(create_mu);
    if (!gm->pipe) gm->pipe = new (std::nothrow) HostPipe();
    if (!gm->pipe) return set_error(GRASS_E_OOM, "host allocation failed");
  }
  HostPipe &hp = *gm->pipe;
  std::lock_guard<std::mutex> lk(hp.mu);
  if (!hp.st[0]) {
    for (int i = 0; i < 2; i++)
      GRASS_CUDA(cudaStreamCreateWithFlags(&hp.st[i], cudaStreamNonBlocking));
    GRASS_CUDA(cudaEventCreateWithFlags(&hp.ev, cudaEventDisableTiming));
    GRASS_CUDA(cudaMalloc(&hp.d_edges, sizeof(unsigned long long)));
  }
  // Chunks of walkers alternate between two streams: while one chunk's paths
  // are copied out, the next chunk is copied in and walked.  Walker ids stay
  // global (w0 = chunk base), so the walks equal one launch over all W.
  const uint64_t L1 = (uint64_t)p->length + 1;
  const uint64_t chunk = std::min<uint64_t>(std::max<uint64_t>(W, 1), 1u << 17);
  if (hp.cap_starts < chunk || hp.cap_paths < chunk * L1) {
    for (int i = 0; i < 2; i++) {
      cudaFree(hp.d_starts[i]);
      cudaFree(hp.d_paths[i]);
      hp.d_starts[i] = nullptr;
      hp.d_paths[i] = nullptr;
    }
    hp.cap_starts = hp.cap_paths = 0;
    for (int i = 0; i < 2; i++) {
      GRASS_CUDA(cudaMalloc(&hp.d_starts[i], chunk * 4));
      GRASS_CUDA(cudaMalloc(&hp.d_paths[i], chunk * L1 * 4));
    }
    hp.cap_starts = chunk;
    hp.cap_paths = chunk * L1;
  }
  GRASS_CUDA(cudaMemsetAsync(hp.d_edges, 0, sizeof(unsigned long long), hp.st[0]));
  GRASS_CUDA(cudaEventRecord(hp.ev, hp.st[0]));
  GRASS_CUDA(cudaStreamWaitEvent(hp.st[1], hp.ev, 0));
  for (uint64_t base = 0, c = 0; base < W; base += chunk, c++) {
    const int k = (int)(c & 1);
    cudaStream_t s = hp.st[k];
    const uint64_t nc = std::min(chunk, W - base);
    GRASS_CUDA(cudaMemcpyAsync(hp.d_starts[k], h_starts + base, nc * 4, cudaMemcpyHostToDevice, s));
    launch_rw(g->view(), *p, hp.d_starts[k], nc, hp.d_paths[k], hp.d_edges, g->d_err, s,
              g->tuning, g->l2win, base);
    if (int rc = check_launch()) return rc;
    if (p->layout == GRASS_LAYOUT_WALK_MAJOR)
      GRASS_CUDA(cudaMemcpyAsync(h_paths + base * L1, hp.d_paths[k], nc * L1 * 4,
                                 cudaMemcpyDeviceToHost, s));
    else
      GRASS_CUDA(cudaMemcpy2DAsync(h_paths + base, W * 4, hp.d_paths[k], nc * 4, nc * 4, L1,
                                   cudaMemcpyDeviceToHost, s));
  }
  GRASS_CUDA(cudaEventRecord(hp.ev, hp.st[1]));
  GRASS_CUDA(cudaStreamWaitEvent(hp.st[0], hp.ev, 0));
  unsigned long long e = 0;
  GRASS_CUDA(cudaMemcpyAsync(&e, hp.d_edges, sizeof e, cudaMemcpyDeviceToHost, hp.st[0]));
  if (int rc = read_err_flag(g, hp.st[0])) return rc;
  if (edges_out) *edges_out = e;
  return GRASS_OK;
}

int grass_khop(const grass_graph *g, const grass_khop_params *p, const uint32_t *d_seeds,
               uint64_t S, uint32_t *const *d_hop_out, unsigned long long *d_edge_count,
               void *stream) {
  grass::Nvtx nvtx_("grass_khop");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  uint64_t width[GRASS_MAX_HOPS];
  if (int rc = check_khop(p, width)) return rc;
  if (S && (!d_seeds || !d_hop_out)) return set_error(GRASS_E_ARG, "k-hop: null buffers");
  for (uint32_t h = 0; S && h < p->hops; h++)
    if (!d_hop_out[h]) return set_error(GRASS_E_ARG, "k-hop: null output for hop %u", h);
  DeviceGuard dg(g->device);
  launch_khop(g->view(), *p, d_seeds, S, d_hop_out, d_edge_count, g->d_err, as_stream(stream));
  return check_launch();
}

int grass_khop_host(const grass_graph *g, const grass_khop_params *p, const uint32_t *h_seeds,
                    uint64_t S, uint32_t *const *h_hop_out, uint64_t *edges_out) {
  grass::Nvtx nvtx_("grass_khop_host");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  uint64_t width[GRASS_MAX_HOPS];
  if (int rc = check_khop(p, width)) return rc;
  if (S && (!h_seeds || !h_hop_out)) return set_error(GRASS_E_ARG, "k-hop: null buffers");
  DeviceGuard dg(g->device);
  cudaStream_t st = 0;
  DevBuf ds, de, dh[GRASS_MAX_HOPS];
  uint32_t *outs[GRASS_MAX_HOPS] = {nullptr};
  GRASS_CUDA(cudaMalloc(&ds.p, std::max<uint64_t>(S, 1) * 4));
  GRASS_CUDA(cudaMalloc(&de.p, 8));
  for (uint32_t h = 0; h < p->hops; h++) {
    GRASS_CUDA(cudaMalloc(&dh[h].p, std::max<uint64_t>(S * width[h], 1) * 4));
    outs[h] = (uint32_t *)dh[h].p;
  }
  GRASS_CUDA(cudaMemsetAsync(de.p, 0, 8, st));
  GRASS_CUDA(cudaMemcpyAsync(ds.p, h_seeds, S * 4, cudaMemcpyHostToDevice, st));
  launch_khop(g->view(), *p, (uint32_t *)ds.p, S, outs, (unsigned long long *)de.p, g->d_err, st);
  if (int rc = check_launch()) return rc;
  for (uint32_t h = 0; h < p->hops; h++)
    GRASS_CUDA(cudaMemcpyAsync(h_hop_out[h], outs[h], S * width[h] * 4, cudaMemcpyDeviceToHost, st));
  unsigned long long e = 0;
  GRASS_CUDA(cudaMemcpyAsync(&e, de.p, 8, cudaMemcpyDeviceToHost, st));
  if (int rc = read_err_flag(g, st)) return rc;
  if (edges_out) *edges_out = e;
  return GRASS_OK;
}

int grass_mrw(const grass_graph *g, const grass_mrw_params *p, uint32_t *d_roots, uint64_t S,
              uint32_t *d_src, uint32_t *d_dst, unsigned long long *d_edge_count, void *stream) {
  grass::Nvtx nvtx_("grass_mrw");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  if (!p || p->walkers == 0 || p->select > 2 || (S && (!d_roots || !d_src || !d_dst)) ||
      (p->select == GRASS_SELECT_DEGREE_CT && S > 0xFFFFFFFFull))
    return set_error(GRASS_E_ARG, "multi-RW: bad arguments");
  DeviceGuard dg(g->device);
  if (int rc = launch_mrw(g->view(), *p, d_roots, S, d_src, d_dst, d_edge_count, g->d_err,
                          as_stream(stream)))
    return rc;
  return check_launch();
}

int grass_mrw_host(const grass_graph *g, const grass_mrw_params *p, uint32_t *h_roots,
                   uint64_t S, uint32_t *h_src, uint32_t *h_dst, uint64_t *edges_out) {
  grass::Nvtx nvtx_("grass_mrw_host");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  if (!p || p->walkers == 0 || p->select > 2 || (S && (!h_roots || !h_src || !h_dst)) ||
      (p->select == GRASS_SELECT_DEGREE_CT && S > 0xFFFFFFFFull))
    return set_error(GRASS_E_ARG, "multi-RW: bad arguments");
  DeviceGuard dg(g->device);
  cudaStream_t st = 0;
  const uint64_t nr = S * p->walkers, ne = S * (uint64_t)p->steps;
  DevBuf dr, dsrc, ddst, de;
  GRASS_CUDA(cudaMalloc(&dr.p, std::max<uint64_t>(nr, 1) * 4));
  GRASS_CUDA(cudaMalloc(&dsrc.p, std::max<uint64_t>(ne, 1) * 4));
  GRASS_CUDA(cudaMalloc(&ddst.p, std::max<uint64_t>(ne, 1) * 4));
  GRASS_CUDA(cudaMalloc(&de.p, 8));
  GRASS_CUDA(cudaMemsetAsync(de.p, 0, 8, st));
  GRASS_CUDA(cudaMemcpyAsync(dr.p, h_roots, nr * 4, cudaMemcpyHostToDevice, st));
  if (int rc = launch_mrw(g->view(), *p, (uint32_t *)dr.p, S, (uint32_t *)dsrc.p,
                          (uint32_t *)ddst.p, (unsigned long long *)de.p, g->d_err, st))
    return rc;
  if (int rc = check_launch()) return rc;
  GRASS_CUDA(cudaMemcpyAsync(h_roots, dr.p, nr * 4, cudaMemcpyDeviceToHost, st));
  GRASS_CUDA(cudaMemcpyAsync(h_src, dsrc.p, ne * 4, cudaMemcpyDeviceToHost, st));
  GRASS_CUDA(cudaMemcpyAsync(h_dst, ddst.p, ne * 4, cudaMemcpyDeviceToHost, st));
  unsigned long long e = 0;
  GRASS_CUDA(cudaMemcpyAsync(&e, de.p, 8, cudaMemcpyDeviceToHost, st));
  if (int rc = read_err_flag(g, st)) return rc;
  if (edges_out) *edges_out = e;
  return GRASS_OK;
}

// ---- CSR baseline ----

int grass_csr_from_graph(const grass_graph *g, grass_csr **out) {
  grass::Nvtx nvtx_("grass_csr_from_graph");
  clear_error();
  if (int rc = check_graph(g)) return rc;
  if (!out) return set_error(GRASS_E_ARG, "null output");
  *out = nullptr;
  DeviceGuard dg(g->device);
  auto *c = new (std::nothrow) grass_csr();
  if (!c) return set_error(GRASS_E_OOM, "host allocation failed");
  c->device = g->device;
  c->n = g->info.n;
  c->nnz = g->info.num_edges;
  cudaError_t e1 = cudaMalloc(&c->d_rowptr, csr_rowptr_bytes(c->n));
  cudaError_t e2 = cudaMalloc(&c->d_cols, std::max<uint64_t>(c->nnz, 1) * 4);
  if (e1 != cudaSuccess || e2 != cudaSuccess) {
    grass_csr_close(c);
    return set_error(GRASS_E_OOM, "CSR allocation failed");
  }
  int rc = grass_decode_all(g, c->d_rowptr, c->d_cols, nullptr);
  if (rc == GRASS_OK) rc = read_err_flag(g, 0);
  if (rc) {
    grass_csr_close(c);
    return rc;
  }
  *out = c;
  return GRASS_OK;
}

int grass_csr_from_host(const uint64_t *rowptr, const uint32_t *cols, uint64_t n, int device,
                        grass_csr **out) {
  clear_error();
  if (!rowptr || !out || n == 0 || n > 0xFFFFFFFEull) return set_error(GRASS_E_ARG, "bad arguments");
  *out = nullptr;
  DeviceGuard dg(device);
  auto *c = new (std::nothrow) grass_csr();
  if (!c) return set_error(GRASS_E_OOM, "host allocation failed");
  c->device = device;
  c->n = n;
  c->nnz = rowptr[n];
  if (c->nnz && !cols) {
    delete c;
    return set_error(GRASS_E_ARG, "null cols");
  }
  cudaError_t e1 = cudaMalloc(&c->d_rowptr, csr_rowptr_bytes(n));
  cudaError_t e2 = cudaMalloc(&c->d_cols, std::max<uint64_t>(c->nnz, 1) * 4);
  if (e1 != cudaSuccess || e2 != cudaSuccess) {
    grass_csr_close(c);
    return set_error(GRASS_E_OOM, "CSR allocation failed");
  }
  cudaError_t e3 = cudaMemcpy(c->d_rowptr, rowptr, (n + 1) * 8, cudaMemcpyHostToDevice);
  cudaError_t e4 = c->nnz ? cudaMemcpy(c->d_cols, cols, c->nnz * 4, cudaMemcpyHostToDevice)
                          : cudaSuccess;
  if (e3 != cudaSuccess || e4 != cudaSuccess) {
    grass_csr_close(c);
    return cuda_fail(e3 != cudaSuccess ? e3 : e4, "CSR upload");
  }
  *out = c;
  return GRASS_OK;
}

int grass_csr_close(grass_csr *c) {
  if (!c) return GRASS_OK;
  DeviceGuard dg(c->device);
  cudaFree(c->d_rowptr);
  cudaFree(c->d_cols);
  delete c;
  return GRASS_OK;
}

int grass_csr_info(const grass_csr *c, uint64_t *n, uint64_t *nnz, uint64_t *device_bytes) {
  if (!c) return set_error(GRASS_E_ARG, "null csr");
  if (n) *n = c->n;
  if (nnz) *nnz = c->nnz;
  if (device_bytes) *device_bytes = (c->n + 1) * 8 + c->nnz * 4;
  return GRASS_OK;
}

int grass_csr_set_tuning(grass_csr *c, const grass_tuning *t) {
  if (!c || !t) return set_error(GRASS_E_ARG, "null argument");
  DeviceGuard dg(c->device);
  if (int rc = apply_tuning(c->device, *t, c->d_rowptr, (c->n + 1) * sizeof(uint64_t), c->l2win))
    return rc;
  c->tuning = *t;
  return GRASS_OK;
}

int grass_csr_rw(const grass_csr *c, const grass_rw_params *p, const uint32_t *d_starts,
                 uint64_t W, uint32_t *d_paths, unsigned long long *d_edge_count, void *stream) {
  grass::Nvtx nvtx_("grass_csr_rw");
  clear_error();
  if (!c || !p || p->layout > 1 || (W && (!d_starts || !d_paths)))
    return set_error(GRASS_E_ARG, "CSR random walk: bad arguments");
  DeviceGuard dg(c->device);
  launch_rw_csr(c->view(), *p, d_starts, W, d_paths, d_edge_count, as_stream(stream),
                c->tuning, c->l2win);
  return check_launch();
}

int grass_csr_khop(const grass_csr *c, const grass_khop_params *p, const uint32_t *d_seeds,
                   uint64_t S, uint32_t *const *d_hop_out, unsigned long long *d_edge_count,
                   void *stream) {
  grass::Nvtx nvtx_("grass_csr_khop");
  clear_error();
  if (!c) return set_error(GRASS_E_ARG, "null csr");
  uint64_t width[GRASS_MAX_HOPS];
  if (int rc = check_khop(p, width)) return rc;
  if (S && (!d_seeds || !d_hop_out)) return set_error(GRASS_E_ARG, "k-hop: null buffers");
  DeviceGuard dg(c->device);
  launch_khop_csr(c->view(), *p, d_seeds, S, d_hop_out, d_edge_count, as_stream(stream));
  return check_launch();
}

int grass_csr_node2vec(const grass_csr *c, const grass_node2vec_params *p,
                       const uint32_t *d_starts, uint64_t W, uint32_t *d_paths,
                       unsigned long long *d_edge_count, void *stream) {
  grass::Nvtx nvtx_("grass_csr_node2vec");
  clear_error();
  if (!c) return set_error(GRASS_E_ARG, "null csr");
  grass_node2vec_params r;
  uint64_t t[3];
  if (int rc = node2vec_args(p, r, t)) return rc;
  if (W && (!d_starts || !d_paths)) return set_error(GRASS_E_ARG, "node2vec: null buffers");
  DeviceGuard dg(c->device);
  grass::DevGraph v{};
  v.n = (uint32_t)c->n;
  v.mode = grass::GRASS_MODE_CSR_INTERNAL;
  v.rowptr = c->d_rowptr;
  v.cols = c->d_cols;
  launch_node2vec(v, r, t, d_starts, W, d_paths, d_edge_count, nullptr, as_stream(stream));
  return check_launch();
}

}  // extern "C"
