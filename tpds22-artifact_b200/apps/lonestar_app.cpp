// Lonestar application harness on libgsrb: bfs / sssp / pr over a Galois .gr
// file, with the command line, the block-factor prompt and the output format
// of the reference's skel harness, so that scripts written for the reference's
// binaries run unchanged.
//
//   reference harness   LONESTAR/skelapp/skel.cu.prehip:45 (load, run, output),
//                       :88-130 (options -q -g -o and the app's own options)
//   bfs options/output  LONESTAR/apps/bfs/support.cu:5-45   (-l -s; "%d %d" / "%d INF")
//   sssp options        LONESTAR/apps/sssp/support.cu:6-50  (-l -d delta -s)
//   pr options/output   LONESTAR/apps/pr/support.cu:16-98   (-n -t -x; "sum: %f (%d)")
//   block factor        LONESTAR/apps/bfs/kernel_gsrb.cu:716-719 (" Enter Block factor",
//                       read from stdin: CTAs per SM)
//   "Kernel time (ms)"  LONESTAR/apps/bfs/kernel_gsrb.cu:701
//
// One source builds every app (GSRB_APP = 1 bfs, 2 sssp, 3 pr).  The barrier
// follows the program name, as the reference's three builds do: *_gsrb runs the
// native grid barrier (library default), *_gcpusrb the flat CPU-style
// sense-reversing barrier, *_ccg cooperative groups; -b <variant> overrides.
// Extra options: -m <push|heuristic|learned|pull|topo> (BFS schedule),
// -P <file> (policy weights, raw float32); PR runs the reference's
// push-residual algorithm until no residual exceeds epsilon = 1e-6 (-x caps
// the rounds, as in the reference), or with -u the pull form for -x
// iterations (default 50).
// -l: BFS expands large push levels with the load balancer (GSRB_BFS_FLAG_LB,
// the reference's thread-block load balancer); SSSP accepts -l and expands as
// usual (hub vertices are always split across CTAs).
#include <getopt.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <iostream>
#include <string>
#include <vector>

#include "gsrb.h"

#ifndef GSRB_APP
#define GSRB_APP 1
#endif

namespace {

int g_quiet = 0, g_device = 0, g_start = 0, g_delta = 10000, g_iters = -1, g_no_rank = 0, g_top = 0, g_pull = 0;
int g_lb = 0;
int g_variant = -1, g_mode = GSRB_BFS_HEURISTIC;
const char* g_output = nullptr;
const char* g_policy = nullptr;

#if GSRB_APP == 1
const char* kAppOpts = "ls:m:P:";
const char* kAppUsage = "[-l] [-s startNode] [-m push|heuristic|learned|pull|topo] [-P policy.f32]";
#elif GSRB_APP == 2
const char* kAppOpts = "ls:d:";
const char* kAppUsage = "[-l] [-d delta] [-s startNode]";
#else
const char* kAppOpts = "nt:x:u";
const char* kAppUsage = "[-n] [-t top_ranks] [-x max_iterations] [-u (pull form)]";
#endif

void usage(const char* argv0) {
  fprintf(stderr, "usage: %s [-q] [-g gpunum] [-o output-file] [-b variant] %s graph-file\n", argv0, kAppUsage);
}

[[noreturn]] void die(const char* what, gsrb_status_t st) {
  fprintf(stderr, "%s: %s (%d)\n", what, gsrb_status_string(st), (int)st);
  exit(EXIT_FAILURE);
}

#define CHECK(call)                       \
  do {                                    \
    gsrb_status_t _s = (call);            \
    if (_s != GSRB_OK) die(#call, _s);    \
  } while (0)

int parse_mode(const char* s) {
  const char* names[] = {"push", "heuristic", "learned", "pull", "topo"};
  for (int i = 0; i < 5; ++i)
    if (!strcmp(s, names[i])) return i;
  fprintf(stderr, "unknown BFS mode '%s'\n", s);
  exit(EXIT_FAILURE);
}

int variant_from_name(const char* argv0) {
  std::string n(argv0);
  if (n.size() >= 8 && n.compare(n.size() - 8, 8, "_gcpusrb") == 0) return GSRB_BAR_FLAT;
  if (n.size() >= 4 && n.compare(n.size() - 4, 4, "_ccg") == 0) return GSRB_BAR_CCG;
  return -1;  // *_gsrb and anything else: the library's default barrier
}

void parse_args(int argc, char** argv) {
  std::string opts = std::string("g:qo:b:") + kAppOpts;
  int c;
  while ((c = getopt(argc, argv, opts.c_str())) != -1) {
    switch (c) {
      case 'q': g_quiet = 1; break;
      case 'o': g_output = optarg; break;
      case 'g': {
        char* end;
        g_device = (int)strtol(optarg, &end, 10);
        if (*end) {
          fprintf(stderr, "Invalid GPU device '%s'. An integer must be specified.\n", optarg);
          exit(EXIT_FAILURE);
        }
        break;
      }
      case 'b': g_variant = atoi(optarg); break;
      case 'l': g_lb = 1; break;
      case 's':
        g_start = atoi(optarg);
        if (g_start < 0) { usage(argv[0]); exit(EXIT_FAILURE); }
        break;
      case 'd':
        g_delta = atoi(optarg);
        if (g_delta <= 0) { usage(argv[0]); exit(EXIT_FAILURE); }
        break;
      case 'm': g_mode = parse_mode(optarg); break;
      case 'P': g_policy = optarg; break;
      case 'n': g_no_rank = 1; break;
      case 't': g_top = atoi(optarg); break;
      case 'x': g_iters = atoi(optarg); break;
      case 'u': g_pull = 1; break;
      default: usage(argv[0]); exit(EXIT_FAILURE);
    }
  }
  if (optind >= argc) {
    usage(argv[0]);
    exit(EXIT_FAILURE);
  }
}

FILE* open_output() {
  if (!g_output) return nullptr;
  if (!strcmp(g_output, "-")) return stdout;
  FILE* f = fopen(g_output, "w");
  if (!f) {
    perror(g_output);
    exit(EXIT_FAILURE);
  }
  return f;
}

void write_levels(const std::vector<int32_t>& v) {
  FILE* f = open_output();
  if (!f) return;
  for (size_t i = 0; i < v.size(); ++i) {
    if (v[i] == INT32_MAX)
      fprintf(f, "%d INF\n", (int)i);
    else
      fprintf(f, "%d %d\n", (int)i, v[i]);
  }
  if (f != stdout) fclose(f);
}

void write_ranks(const std::vector<float>& r) {
  float sum = 0;
  for (float x : r) sum += x;
  fprintf(stdout, "sum: %f (%d)\n", sum, (int)r.size());
  FILE* f = open_output();
  if (!f) return;
  size_t n = r.size();
  if (g_top > 0 && (size_t)g_top < n) n = (size_t)g_top;
  for (size_t i = 0; i < n; ++i) {
    if (g_no_rank)
      fprintf(f, "%d\n", (int)i);
    else
      fprintf(f, "%d %f\n", (int)i, r[i]);
  }
  if (f != stdout) fclose(f);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc == 1) {
    usage(argv[0]);
    return 1;
  }
  parse_args(argc, argv);
  const char* input = argv[optind];

  gsrb_ctx_t ctx;
  CHECK(gsrb_ctx_create(g_device, &ctx));
  int32_t sms = 0, dev = 0;
  int64_t l2 = 0;
  CHECK(gsrb_ctx_info(ctx, &sms, &l2, &dev));
  printf("Using GPU: device %d (%d SMs, %lld MB L2)\n", dev, sms, (long long)(l2 >> 20));

  gsrb_host_csr_t hg;
  memset(&hg, 0, sizeof(hg));
  auto t0 = std::chrono::steady_clock::now();
  CHECK(gsrb_gr_read(input, &hg));
  fprintf(stderr, "Read %u nodes, %llu edges from %s\n", hg.nnodes, (unsigned long long)hg.nedges, input);
  if (GSRB_APP != 3 && (uint32_t)g_start >= hg.nnodes) {
    fprintf(stderr, "start node %d out of range (%u nodes)\n", g_start, hg.nnodes);
    return EXIT_FAILURE;
  }
  if (GSRB_APP == 2 && !hg.edge_data) {
    fprintf(stderr, "sssp needs a weighted .gr file\n");
    return EXIT_FAILURE;
  }

  gsrb_graph_t g;
  CHECK(gsrb_graph_upload(ctx, &hg, &g));

  if (g_policy) {
    size_t count = gsrb_mlp_param_count();
    std::vector<float> w(count);
    FILE* f = fopen(g_policy, "rb");
    if (!f || fread(w.data(), sizeof(float), count, f) != count) {
      fprintf(stderr, "cannot read %zu float32 weights from %s\n", count, g_policy);
      return EXIT_FAILURE;
    }
    fclose(f);
    CHECK(gsrb_graph_set_policy(g, w.data(), count));
  }

  // The reference asks for the block factor (CTAs per SM) on stdin.
  std::cout << " Enter Block factor" << std::endl;
  int block_factor = 0;
  if (!(std::cin >> block_factor) || block_factor < 0) block_factor = 0;

  gsrb_cfg_t cfg;
  gsrb_cfg_default(&cfg);
  int v = g_variant >= 0 ? g_variant : variant_from_name(argv[0]);
  if (v >= 0) cfg.variant = v;
  if (block_factor > 0) cfg.ctas_per_sm = block_factor;
  fprintf(stderr, "OPTIONS: variant %d, CTAs/SM %d, threads %d\n", cfg.variant, cfg.ctas_per_sm, cfg.threads);

  gsrb_traversal_stats_t st;
  memset(&st, 0, sizeof(st));
  gsrb_status_t rc;
  uint32_t n = hg.nnodes;
  if (GSRB_APP == 3) {
    float* d = nullptr;
    CHECK(gsrb_malloc((void**)&d, sizeof(float) * (n ? n : 1)));
    if (g_pull) {
      rc = gsrb_pagerank(ctx, g, 0.85f, g_iters >= 0 ? g_iters : 50, d, &cfg, &st);
      if (rc != GSRB_OK) die("gsrb_pagerank", rc);
    } else {
      // ALPHA = 0.85, EPSILON = 1e-6 (apps/pr/kernel_gsrb.cu:291-292); MAX_ITERATIONS
      // defaults to INT_MAX (apps/pr/support.cu:26)
      rc = gsrb_pagerank_residual(ctx, g, 0.85f, 1e-6f, g_iters >= 0 ? g_iters : INT32_MAX, d, &cfg, &st);
      if (rc != GSRB_OK) die("gsrb_pagerank_residual", rc);
    }
    printf("Kernel time (ms) %f\n", st.kernel_ms);
    printf("PR took %u iterations\n", st.levels);
    std::vector<float> r(n);
    CHECK(gsrb_memcpy_d2h(ctx, r.data(), d, sizeof(float) * n));
    CHECK(gsrb_ctx_synchronize(ctx));
    if (!g_quiet) write_ranks(r);
    gsrb_free(d);
  } else {
    int32_t* d = nullptr;
    CHECK(gsrb_malloc((void**)&d, sizeof(int32_t) * (n ? n : 1)));
    if (GSRB_APP == 1) {
      rc = gsrb_bfs(ctx, g, (uint32_t)g_start, d, g_mode | (g_lb ? GSRB_BFS_FLAG_LB : 0), &cfg, &st);
      if (rc != GSRB_OK) die("gsrb_bfs", rc);
      printf("Kernel time (ms) %f\n", st.kernel_ms);
      printf("levels: %u\n", st.levels);
    } else {
      printf("delta: %d\n", g_delta);
      rc = gsrb_sssp(ctx, g, (uint32_t)g_start, d, g_delta, &cfg, &st);
      if (rc != GSRB_OK) die("gsrb_sssp", rc);
      printf("Kernel time (ms) is  %f\n", st.kernel_ms);
      printf("iterations: %u\n", st.levels);
    }
    std::vector<int32_t> out(n);
    CHECK(gsrb_memcpy_d2h(ctx, out.data(), d, sizeof(int32_t) * n));
    CHECK(gsrb_ctx_synchronize(ctx));
    if (!g_quiet) write_levels(out);
    gsrb_free(d);
  }
  double total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  fprintf(stderr, "gg_main total (ms, incl. read and upload): %.3f\n", total);
  gsrb_graph_free(g);
  gsrb_host_csr_free(&hg);
  gsrb_ctx_destroy(ctx);
  return 0;
}
