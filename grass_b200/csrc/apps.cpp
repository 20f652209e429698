// apps.cpp -- drop-in replacements for the reference's sampling binaries.
//
// One source, four binaries chosen by argv[0]: rw (DeepWalkApp), khop and its
// alias ks (KHopApp), mrw (MultiRWApp).  The reference's options are kept
// (appMain, GT/src/main.cu:5-41, parsed there by AnyOption):
//   -h --help          usage
//   -g --graph-file    <cgc_path>: reads <cgc_path>.graph and <cgc_path>.offset
//   -n --nruns         number of runs (default 1)
// With no options, or without -g, the usage is printed and the exit code is 0,
// as in the reference.  The reference's default workloads are the defaults
// here: rw = one walker per vertex starting at i % n, 80 steps
// (GT/src/apps/randomwalk/randomWalks.cu:4-24); khop = one seed per vertex,
// fanouts 10 then 25 (GT/src/apps/khop/khop.cu:3-8); mrw = one sample per
// vertex, 80 roots, 100 steps, uniform walker choice
// (GT/src/apps/multiRW/multiRW.cu:3-16, 93-111).  The timing lines of
// nextdoor() (GT/src/grass.cu:2127-2130) are printed.
//
// Additions: --mode gt|le|auto, --device, --seed, --walkers, --length,
// --starts identity|uniform, --fanouts a,b,..., --seeds, --samples, --roots,
// --steps, --select uniform|degree, --output FILE (raw u32 samples of the
// last run), --json.  Deviations: errors exit non-zero (the reference exits 0
// after "Open graph file failed!"); draws use Philox4x32-10, not cuRAND.
#include <cuda_runtime.h>
#include <libgen.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <string>
#include <vector>

#include "../../include/grass.h"

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

void usage() {
  printf("usage: \n\n");
  printf("-h --help              Prints this help\n");
  printf("-g --graph-file        File containing graph\n");
  printf("-n --nruns             Number of runs\n");
  printf("\n(grass_b200 additions)\n");
  printf("   --mode gt|le|auto   compressed format (default auto)\n");
  printf("   --device D          CUDA device (default 0)\n");
  printf("   --seed S            Philox seed (default 7)\n");
  printf("rw:   --walkers W --length L --starts identity|uniform\n");
  printf("khop: --seeds S --fanouts a,b[,c...] --starts identity|uniform\n");
  printf("mrw:  --samples S --roots R --steps T --select uniform|degree\n");
  printf("   --output FILE       raw uint32 samples of the last run\n");
  printf("   --json              print a JSON summary line\n");
}

struct Opts {
  bool help = false, json = false, any = false;
  std::string graph, mode = "auto", starts = "identity", select = "uniform", output;
  long nruns = 1;
  int device = 0;
  unsigned long long seed = 7;
  long long walkers = -1, seeds = -1, samples = -1;
  long length = 80, roots = 80, steps = 100;
  std::vector<uint32_t> fanouts;
};

bool take(int argc, char **argv, int &i, const char *shortf, const char *longf,
          std::string &val) {
  const char *a = argv[i];
  const size_t ll = strlen(longf);
  if (longf[0] && strncmp(a, "--", 2) == 0 && strncmp(a + 2, longf, ll) == 0) {
    if (a[2 + ll] == '=') {
      val = a + 3 + ll;
      return true;
    }
    if (a[2 + ll] == 0 && i + 1 < argc) {
      val = argv[++i];
      return true;
    }
  }
  if (shortf[0] && a[0] == '-' && a[1] == shortf[0] && a[1] != '-') {
    if (a[2]) {
      val = a + 2;
      return true;
    }
    if (i + 1 < argc) {
      val = argv[++i];
      return true;
    }
  }
  return false;
}

int parse(int argc, char **argv, Opts &o) {
  for (int i = 1; i < argc; i++) {
    std::string v;
    const char *a = argv[i];
    o.any = true;
    if (!strcmp(a, "-h") || !strcmp(a, "--help")) o.help = true;
    else if (!strcmp(a, "--json")) o.json = true;
    else if (take(argc, argv, i, "g", "graph-file", v)) o.graph = v;
    else if (take(argc, argv, i, "n", "nruns", v)) o.nruns = atol(v.c_str());
    else if (take(argc, argv, i, "", "mode", v)) o.mode = v;
    else if (take(argc, argv, i, "", "device", v)) o.device = atoi(v.c_str());
    else if (take(argc, argv, i, "", "seed", v)) o.seed = strtoull(v.c_str(), nullptr, 0);
    else if (take(argc, argv, i, "", "walkers", v)) o.walkers = atoll(v.c_str());
    else if (take(argc, argv, i, "", "length", v)) o.length = atol(v.c_str());
    else if (take(argc, argv, i, "", "starts", v)) o.starts = v;
    else if (take(argc, argv, i, "", "seeds", v)) o.seeds = atoll(v.c_str());
    else if (take(argc, argv, i, "", "samples", v)) o.samples = atoll(v.c_str());
    else if (take(argc, argv, i, "", "roots", v)) o.roots = atol(v.c_str());
    else if (take(argc, argv, i, "", "steps", v)) o.steps = atol(v.c_str());
    else if (take(argc, argv, i, "", "select", v)) o.select = v;
    else if (take(argc, argv, i, "", "output", v)) o.output = v;
    else if (take(argc, argv, i, "", "fanouts", v)) {
      o.fanouts.clear();
      for (char *t = strtok(&v[0], ","); t; t = strtok(nullptr, ",")) o.fanouts.push_back(atoi(t));
    } else {
      fprintf(stderr, "unknown option %s\n", a);
      return 1;
    }
  }
  return 0;
}

int fail(const char *what) {
  fprintf(stderr, "%s: %s\n", what, grass_last_error());
  return 1;
}

#define CK(call)                                                              \
  do {                                                                        \
    cudaError_t e_ = (call);                                                  \
    if (e_ != cudaSuccess) {                                                  \
      fprintf(stderr, "Cuda Error: %s %s\n", cudaGetErrorString(e_), #call); \
      return 1;                                                               \
    }                                                                         \
  } while (0)

}  // namespace

int main(int argc, char **argv) {
  std::string app = basename(argv[0]);
  if (app == "ks") app = "khop";
  if (app != "rw" && app != "khop" && app != "mrw") app = "rw";
  Opts o;
  if (parse(argc, argv, o)) {
    usage();
    return 2;
  }
  if (!o.any || o.help || o.graph.empty()) {  // GT/src/main.cu:20-34
    usage();
    return 0;
  }
  if (o.nruns < 1) o.nruns = 1;

  const double e2e0 = now_s();
  grass_graph *g = nullptr;
  int rc;
  if (o.mode == "gt" || o.mode == "GT") rc = grass_open(o.graph.c_str(), GRASS_MODE_GT, o.device, &g);
  else if (o.mode == "le" || o.mode == "LE") rc = grass_open(o.graph.c_str(), GRASS_MODE_LE, o.device, &g);
  else {
    rc = grass_open(o.graph.c_str(), GRASS_MODE_GT, o.device, &g);
    if (rc == GRASS_E_FORMAT) rc = grass_open(o.graph.c_str(), GRASS_MODE_LE, o.device, &g);
  }
  if (rc) return fail(rc == GRASS_E_IO ? "Open graph file failed!" : "load");
  grass_graph_info info;
  grass_get_info(g, &info);
  const double t_transfer = now_s() - e2e0;
  printf("Graph loaded. Graph has %llu vertices.\n", (unsigned long long)info.n);
  printf("Format: %s, %llu edges, %llu device bytes (uncompressed CSR would be %llu)\n",
         info.mode == GRASS_MODE_GT ? "GT" : "LE", (unsigned long long)info.num_edges,
         (unsigned long long)info.device_bytes,
         (unsigned long long)((info.n + 1) * 8 + info.num_edges * 4));
  CK(cudaSetDevice(o.device));
  const uint64_t n = info.n;

  // starts / seeds: i % n (the reference's initialSample) or uniform Philox draws
  auto make_starts = [&](uint64_t count, uint32_t *d_out) -> int {
    if (o.starts == "uniform") return grass_uniform_starts(n, count, o.seed, d_out, nullptr);
    std::vector<uint32_t> h(count);
    for (uint64_t i = 0; i < count; i++) h[i] = (uint32_t)(i % n);
    return cudaMemcpy(d_out, h.data(), count * 4, cudaMemcpyHostToDevice) == cudaSuccess
               ? GRASS_OK
               : GRASS_E_CUDA;
  };

  unsigned long long *d_edges = nullptr;
  CK(cudaMalloc(&d_edges, 8));
  std::vector<void *> bufs;
  std::vector<std::pair<void *, uint64_t>> outputs;
  double t_run = 0;
  if (app == "rw") {
    const uint64_t W = o.walkers > 0 ? (uint64_t)o.walkers : n;
    uint32_t *d_starts, *d_paths;
    CK(cudaMalloc(&d_starts, W * 4));
    CK(cudaMalloc(&d_paths, W * (o.length + 1) * 4));
    bufs = {d_starts, d_paths};
    if (make_starts(W, d_starts)) return fail("starts");
    grass_rw_params p{(uint32_t)o.length, GRASS_LAYOUT_WALK_MAJOR, o.seed};
    CK(cudaDeviceSynchronize());
    CK(cudaMemset(d_edges, 0, 8));
    const double t0 = now_s();
    for (long r = 0; r < o.nruns; r++)
      if (grass_rw(g, &p, d_starts, W, d_paths, d_edges, nullptr)) return fail("rw");
    CK(cudaDeviceSynchronize());
    t_run = now_s() - t0;
    outputs.push_back({d_paths, W * (o.length + 1)});
  } else if (app == "khop") {
    const uint64_t S = o.seeds > 0 ? (uint64_t)o.seeds : n;
    grass_khop_params p{};
    if (o.fanouts.empty()) o.fanouts = {10, 25};
    if (o.fanouts.size() > GRASS_MAX_HOPS) return fail("too many hops");
    p.hops = (uint32_t)o.fanouts.size();
    uint64_t w = 1;
    uint32_t *outs[GRASS_MAX_HOPS];
    uint32_t *d_seeds;
    CK(cudaMalloc(&d_seeds, S * 4));
    bufs.push_back(d_seeds);
    for (uint32_t h = 0; h < p.hops; h++) {
      p.fanouts[h] = o.fanouts[h];
      w *= o.fanouts[h];
      CK(cudaMalloc(&outs[h], S * w * 4));
      bufs.push_back(outs[h]);
      outputs.push_back({outs[h], S * w});
    }
    p.seed = o.seed;
    if (make_starts(S, d_seeds)) return fail("seeds");
    CK(cudaDeviceSynchronize());
    CK(cudaMemset(d_edges, 0, 8));
    const double t0 = now_s();
    for (long r = 0; r < o.nruns; r++)
      if (grass_khop(g, &p, d_seeds, S, outs, d_edges, nullptr)) return fail("khop");
    CK(cudaDeviceSynchronize());
    t_run = now_s() - t0;
  } else {
    const uint64_t S = o.samples > 0 ? (uint64_t)o.samples : n;
    grass_mrw_params p{(uint32_t)o.roots, (uint32_t)o.steps,
                       o.select == "degree" ? (uint32_t)GRASS_SELECT_DEGREE
                                            : (uint32_t)GRASS_SELECT_UNIFORM,
                       0, o.seed};
    uint32_t *d_roots, *d_init, *d_src, *d_dst;
    const uint64_t nr = S * (uint64_t)o.roots, ne = S * (uint64_t)o.steps;
    CK(cudaMalloc(&d_roots, nr * 4));
    CK(cudaMalloc(&d_init, nr * 4));
    CK(cudaMalloc(&d_src, ne * 4));
    CK(cudaMalloc(&d_dst, ne * 4));
    bufs = {d_roots, d_init, d_src, d_dst};
    if (grass_mrw_roots(n, S, (uint32_t)o.roots, o.seed, d_init, nullptr)) return fail("roots");
    CK(cudaDeviceSynchronize());
    CK(cudaMemset(d_edges, 0, 8));
    const double t0 = now_s();
    for (long r = 0; r < o.nruns; r++) {
      CK(cudaMemcpyAsync(d_roots, d_init, nr * 4, cudaMemcpyDeviceToDevice));
      if (grass_mrw(g, &p, d_roots, S, d_src, d_dst, d_edges, nullptr)) return fail("mrw");
    }
    CK(cudaDeviceSynchronize());
    t_run = now_s() - t0;
    outputs.push_back({d_src, ne});
    outputs.push_back({d_dst, ne});
  }
  unsigned long long edges = 0;
  CK(cudaMemcpy(&edges, d_edges, 8, cudaMemcpyDeviceToHost));
  if (!o.output.empty()) {
    FILE *f = fopen(o.output.c_str(), "wb");
    if (!f) return fail("cannot open --output");
    for (auto &ob : outputs) {
      std::vector<uint32_t> h(ob.second);
      CK(cudaMemcpy(h.data(), ob.first, ob.second * 4, cudaMemcpyDeviceToHost));
      fwrite(h.data(), 4, h.size(), f);
    }
    fclose(f);
  }
  const double t_e2e = now_s() - e2e0;
  printf("EndToEndTime: %f\n", t_e2e);
  printf("transferEndToEndTime: %f\n", t_transfer + t_run);
  printf("transferDataTime: %f\n", t_transfer);
  printf("runSamplingTime: %f\n", t_run);
  printf("SampledEdges: %llu\n", edges);
  printf("SampledEdgesPerSecond: %.6e\n", t_run > 0 ? edges / t_run : 0.0);
  if (o.json)
    printf("{\"app\": \"%s\", \"n\": %llu, \"edges\": %llu, \"runs\": %ld, \"run_s\": %f, "
           "\"edges_per_s\": %.6e}\n",
           app.c_str(), (unsigned long long)n, edges, o.nruns, t_run,
           t_run > 0 ? edges / t_run : 0.0);
  for (void *b : bufs) cudaFree(b);
  cudaFree(d_edges);
  grass_close(g);
  return 0;
}
