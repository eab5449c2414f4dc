// gg_main for the reference's own Lonestar harness: BFS, SSSP and PageRank on
// libgsrb, linked with the reference's unchanged skel.cu (argument parsing,
// .gr loading, copy to the GPU, output), apps/<app>/support.cu (app options
// and output format) and rt/src/csr_graph.cu (CSRGraph).  This file takes the
// place of apps/<app>/kernel_gsrb.cu and nothing else; GSRB_APP selects the
// app (1 bfs, 2 sssp, 3 pr).
//
//   gg_main(CSRGraphTy& hg, CSRGraphTy& gg)   LONESTAR/skelapp/skel.cu.prehip:12 (declared),
//                                             :61 (called); app definitions
//                                             apps/bfs/kernel_gsrb.cu:712-730,
//                                             apps/sssp/kernel_gsrb.cu:791-820,
//                                             apps/pr/kernel_gsrb.cu:683-715
//   block factor prompt, stdin                apps/bfs/kernel_gsrb.cu:716-719
//   globals the support files expect          INF, enable_lb (bfs/kernel_gsrb.cu:291-295),
//                                             DELTA (sssp/support.cu:10), P_CURR/P_NEXT,
//                                             ALPHA/EPSILON (pr/kernel_gsrb.cu:288-292)
//   printed lines                             "Kernel time (ms)" (bfs :701),
//                                             "Kernel time (ms) is " (sssp :778),
//                                             "delta:", "iterations:" (sssp :813,819),
//                                             "PR took %d iterations" (pr :712)
//
// The graph stays where skel put it: gg's device arrays are wrapped, not
// copied (gsrb_graph_wrap), and BFS levels / SSSP distances are written
// straight into gg.node_data, which skel copies back and prints.  PageRank
// leaves its ranks in P_CURR (host), which pr/support.cu's output() prints.
// Errors from the library are printed and end the program with exit(1), as
// the reference's check_cuda does.
#include "gg.h"

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <iostream>

#include "gsrb.h"

#ifndef GSRB_APP
#define GSRB_APP 1
#endif

const char* GGC_OPTIONS = "libgsrb persistent traversal (sm_100a), grid barrier chosen by the library";
bool enable_lb = false;

#if GSRB_APP == 1 || GSRB_APP == 2
extern const int INF = INT_MAX;
extern int start_node;
#endif
#if GSRB_APP == 2
extern int DELTA;
#endif
#if GSRB_APP == 3
float* P_CURR = nullptr;
float* P_NEXT = nullptr;
extern const float ALPHA = 0.85f;
extern const float EPSILON = 0.000001f;
extern int MAX_ITERATIONS;
#endif

namespace {

void must(gsrb_status_t st, const char* what) {
  if (st != GSRB_OK) {
    fprintf(stderr, "%s: %s (%d)\n", what, gsrb_status_string(st), (int)st);
    exit(1);
  }
}

}  // namespace

void gg_main(CSRGraphTy& hg, CSRGraphTy& gg) {
  std::cout << " Enter Block factor" << std::endl;
  int block_factor = 0;
  if (!(std::cin >> block_factor) || block_factor < 0) block_factor = 0;

  int dev = 0;
  check_cuda(cudaGetDevice(&dev));
  gsrb_ctx_t ctx;
  must(gsrb_ctx_create(dev, &ctx), "gsrb_ctx_create");
  gsrb_graph_t g;
  must(gsrb_graph_wrap(ctx, gg.nnodes, gg.nedges, gg.row_start, gg.edge_dst, gg.edge_data, &g), "gsrb_graph_wrap");

  gsrb_cfg_t cfg;
  gsrb_cfg_default(&cfg);
  if (block_factor > 0) cfg.ctas_per_sm = block_factor;
  gsrb_traversal_stats_t st = {};

#if GSRB_APP == 1
  if ((unsigned)start_node >= gg.nnodes) {
    fprintf(stderr, "start node %d out of range (%u nodes)\n", start_node, gg.nnodes);
    exit(1);
  }
  must(gsrb_bfs(ctx, g, (uint32_t)start_node, gg.node_data,
                GSRB_BFS_HEURISTIC | (enable_lb ? GSRB_BFS_FLAG_LB : 0), &cfg, &st),
       "gsrb_bfs");
  std::cout << "Kernel time (ms) " << st.kernel_ms << std::endl;
#elif GSRB_APP == 2
  if ((unsigned)start_node >= gg.nnodes) {
    fprintf(stderr, "start node %d out of range (%u nodes)\n", start_node, gg.nnodes);
    exit(1);
  }
  printf("delta: %d\n", DELTA);
  must(gsrb_sssp(ctx, g, (uint32_t)start_node, gg.node_data, DELTA, &cfg, &st), "gsrb_sssp");
  std::cout << "Kernel time (ms) is  " << st.kernel_ms << std::endl;
  printf("iterations: %u\n", st.levels);
#else
  float* d_rank = nullptr;
  must(gsrb_malloc((void**)&d_rank, sizeof(float) * (gg.nnodes ? gg.nnodes : 1)), "gsrb_malloc");
  must(gsrb_pagerank_residual(ctx, g, ALPHA, EPSILON, MAX_ITERATIONS, d_rank, &cfg, &st), "gsrb_pagerank_residual");
  std::cout << "Kernel Time (ms) " << st.kernel_ms << std::endl;
  P_CURR = (float*)calloc(hg.nnodes ? hg.nnodes : 1, sizeof(float));
  if (!P_CURR) {
    fprintf(stderr, "Failed to allocate memory\n");
    exit(1);
  }
  must(gsrb_memcpy_d2h(ctx, P_CURR, d_rank, sizeof(float) * hg.nnodes), "gsrb_memcpy_d2h");
  P_NEXT = P_CURR;
  printf("PR took %u iterations\n", st.levels);
#endif
  must(gsrb_ctx_synchronize(ctx), "gsrb_ctx_synchronize");
#if GSRB_APP == 3
  gsrb_free(d_rank);
#endif
  must(gsrb_graph_free(g), "gsrb_graph_free");
  must(gsrb_ctx_destroy(ctx), "gsrb_ctx_destroy");
}
