/* oracle.h -- CPU restatement of the reference algorithms on the hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: the parity tests,
 * the smoke test and the CPU-baseline leg of bench.py call it; the product
 * (libgsrb.so and everything under tpds22-artifact_b200/) never links, loads
 * or calls it, and has no CPU fallback.
 *
 * Each function cites the reference file:line whose behaviour it restates.
 * Pins: the scan oracle is checked against the reference's own cpu_sum_scan
 * compiled from scan/main.cu (oracle/ref_build.sh -> oracle/_ref/), the reduce
 * and scan oracles against the reference's all-ones golden cases
 * (Reduce/test_reduce.cu:14-17, scan/main.cu:37-41), the Heterosync replay
 * against the reference's golden loop (Heterosync/main.cu:2987-3166).  The
 * graph oracles (BFS, Dijkstra, PageRank) have no CPU counterpart in the
 * reference; they are pinned against the outputs of the reference's own
 * Lonestar programs (bfs/sssp/pr_ccg built for sm_100a) on six seeded graphs,
 * frozen in tests/golden/ref_lonestar_golden.npz by
 * tests/golden/make_ref_lonestar.py, and by hand-computed fixtures.
 */
#ifndef GSRB_ORACLE_H_
#define GSRB_ORACLE_H_
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Serial int64 sum (Reduce: reduce() returns the sum of arr, Reduce/reduce.cuh:42-47). */
int64_t orc_sum_i32(const int32_t* in, size_t n);
/* The same sum on `threads` host threads (CPU baseline, all cores). */
int64_t orc_sum_i32_mt(const int32_t* in, size_t n, int threads);

/* Exclusive prefix sum with uint32 wraparound: cpu_sum_scan, scan/main.cu:11-21. */
void orc_scan_u32(const uint32_t* in, uint32_t* out, size_t n);
/* Two-pass blocked exclusive scan on `threads` host threads (CPU baseline). */
void orc_scan_u32_mt(const uint32_t* in, uint32_t* out, size_t n, int threads);
/* FP64 exclusive prefix of FP32 input (oracle for the FP32 scan). */
void orc_scan_f32_f64(const float* in, double* out, size_t n);
/* max_i |gpu_i - ref_i| / max(|ref_i|, floor); the FP32 scan tolerance check. */
double orc_max_rel_err_f32_f64(const float* gpu, const double* ref, size_t n, double floor_);

/* BFS levels: level[src] = 0, unreachable = INT32_MAX, level L for vertices first
 * reached in round L (LONESTAR/apps/bfs/kernel_gsrb.cu:299-311, :473-479, :724). */
void orc_bfs(uint32_t n, const uint32_t* row, const uint32_t* dst, uint32_t src, int32_t* level);
/* Dijkstra with a binary heap; INT32_MAX = unreachable (LONESTAR/apps/sssp/kernel_gsrb.cu:297-309). */
void orc_dijkstra(uint32_t n, const uint32_t* row, const uint32_t* dst, const int32_t* w, uint32_t src,
                  int32_t* dist);
/* Pull PageRank in FP64: x0 = 1 - alpha (LONESTAR/apps/pr/kernel_gsrb.cu:311),
 * x <- (1 - alpha) + alpha * sum_{u in N(v)} x_u / deg(u), `iters` times;
 * vertices without edges contribute nothing. */
void orc_pagerank_pull(uint32_t n, const uint32_t* row, const uint32_t* dst, double alpha, int iters,
                       double* x);
/* The same fixed point in scatter form over out-edges, for any graph (the
 * fixed point of the reference's push-residual PageRank,
 * LONESTAR/apps/pr/kernel_gsrb.cu:298-336); equals orc_pagerank_pull on a
 * symmetric graph. */
void orc_pagerank_push(uint32_t n, const uint32_t* row, const uint32_t* dst, double alpha, int iters,
                       double* x);
/* The same BFS and pull PageRank on `threads` host threads (CPU baseline, all
 * cores): level-synchronous BFS with compare-and-swap claims, PageRank split
 * over vertex chunks.  Results equal orc_bfs / orc_pagerank_pull. */
void orc_bfs_mt(uint32_t n, const uint32_t* row, const uint32_t* dst, uint32_t src, int32_t* level, int threads);
void orc_pagerank_pull_mt(uint32_t n, const uint32_t* row, const uint32_t* dst, double alpha, int iters,
                          double* x, int threads);
/* sum_v |a_v/sum(a) - b_v/sum(b)| with `a` FP32 and `b` FP64. */
double orc_normalized_l1(const float* a, const double* b, uint32_t n);
/* Directed CSR edges out of reached vertices (value != INT32_MAX): the TEPS numerator. */
uint64_t orc_traversed_edges(uint32_t n, const uint32_t* row, const int32_t* value);

/* Independent `.gr` v1 reader (LONESTAR/rt/src/csr_graph.cu:152-237) used to
 * cross-check the product's writer.  Returns 0 on success; buffers are malloc'd. */
int orc_gr_read(const char* path, uint32_t* n, uint64_t* m, uint32_t** row, uint32_t** dst, int32_t** w);
void orc_free(void* p);

/* Heterosync golden replay (Heterosync/main.cu:41-59, :2987-3166): applies the
 * critical-section accesses of `numIters` iterations x `numRepeats` launches of
 * microbenchmark `syncPrim` (the reference's numbering, :2478-2535) to
 * `storage` (initialised by the caller to storage[i] = i). */
void orc_heterosync_golden(int syncPrim, int numLdSt, int numTBs, int numIters, int numRepeats,
                           int numSM, int threadsPerBlock, float* storage, int numStorageLocs);
/* Storage size the reference harness allocates for a microbenchmark (:2561-2583). */
int orc_heterosync_storage_locs(int syncPrim, int numLdSt, int numTBs, int numSM, int threadsPerBlock);

/* Host-thread model of the two-level sense-reversing barrier
 * (Heterosync/cudaLocksBarrierAtomicSRB.cu:63-236 restated with C11 atomics):
 * `nthreads` participants in `ngroups` groups (0 = one level) run `episodes`
 * episodes; each episode every participant writes a stamp, crosses the
 * barrier, reads a peer's stamp, crosses again.  Returns ns per barrier episode;
 * *stale receives the number of stale reads (must be 0). */
double orc_cpu_srb_barrier(int nthreads, int ngroups, int episodes, uint64_t* stale);
/* The same barrier with `nctas` participants (the CTAs of a grid) carried by
 * `nthreads` host threads: thread t arrives for participants t, t + nthreads,
 * ... in turn (group counters by participant % ngroups, as the reference
 * groups CTAs by blockIdx % NUM_SM), then waits once for the episode. */
double orc_cpu_srb_barrier_vcta(int nthreads, int nctas, int ngroups, int episodes, uint64_t* stale);
/* The same with injected stalls: at each stall point (before an arrival, in a
 * group completer, between the root completer's counter reset and its
 * publish) a participant yields or sleeps 5-100 us with probability
 * stall_permille / 1000 (seeded per participant); *stalls (may be NULL)
 * receives how many stalls were taken. */
double orc_cpu_srb_barrier_stalls(int nthreads, int ngroups, int episodes, int stall_permille, uint64_t seed,
                                  uint64_t* stale, uint64_t* stalls);
/* The same with a participant that leaves for good: kill_id stops before
 * episode kill_episode and never arrives again.  Every wait is bounded by
 * deadline_ms; the first wait that runs out raises an abort flag and every
 * other waiter gives up at its next poll (the device's abort-word protocol).
 * Returns when all participants have left; *timeouts receives the number of
 * waits that ran out (>= 1 when someone was killed before the end). */
double orc_cpu_srb_barrier_kill(int nthreads, int ngroups, int episodes, int kill_id, int kill_episode,
                                int deadline_ms, uint64_t* stale, uint64_t* timeouts);

/* Host-thread model of the reader/writer priority semaphore semantics: `nthreads`
 * holders (every `writer_every`-th is a writer) each acquire `iters` times, add
 * `incs` to W (writers, plain read-modify-write) or R (readers, atomic);
 * returns acquires per second and fills the final counters and the largest
 * number of simultaneous readers seen. */
double orc_cpu_semaphore(int nthreads, int capacity, int writer_every, int iters, int incs,
                         uint64_t* W, uint64_t* R, uint32_t* max_readers, uint32_t* violations);
/* The same with injected stalls (before each acquire and while holding the
 * semaphore; see orc_cpu_srb_barrier_stalls). */
double orc_cpu_semaphore_stalls(int nthreads, int capacity, int writer_every, int iters, int incs,
                                int stall_permille, uint64_t seed, uint64_t* W, uint64_t* R,
                                uint32_t* max_readers, uint32_t* violations, uint64_t* stalls);

/* FP64 forward + backward of the policy MLP (12 -> 32 -> 32 -> 4, ReLU; layout
 * of gsrb_mlp_param_count()): masked BCE-with-logits on outputs 0-1, masked
 * 0.5*(z-y)^2 on outputs 2-3, batch mean.  grad: 1604 doubles.  The checker of
 * the GPU training kernels' gradients. */
void orc_mlp_loss_grad(const float* params, const float* X, const float* Y, const float* M, int B, double* grad,
                       double* loss);
void orc_mlp_forward(const float* params, const float* X, int B, double* out);

#ifdef __cplusplus
}
#endif
#endif
