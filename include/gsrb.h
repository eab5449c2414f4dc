/* gsrb.h -- C ABI of libgsrb, a B200 (sm_100a) implementation of the TPDS'22
 * GPU synchronization layer (multi-level sense-reversing grid barrier, mutexes,
 * priority semaphore) and of the persistent barrier-stepped kernels that run on
 * it (reduce, scan, Lonestar BFS / SSSP / PageRank).
 *
 * Conventions
 *   - Every entry point returns gsrb_status_t (0 = success, negative = error);
 *     nothing calls exit() or traps.  Device-side failures (a bounded wait that
 *     ran out) are sticky in the context until gsrb_ctx_status() reads and
 *     clears them.
 *   - Pointers named d_* are device pointers, h_* host pointers.  No torch or
 *     C++ types cross this boundary.
 *   - Work is issued on the context's stream.  Entry points documented as
 *     "synchronous" wait for their work; the others only enqueue it.
 *   - One context may be used by one host thread at a time (calls serialize on
 *     an internal mutex).
 */
#ifndef GSRB_H_
#define GSRB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gsrb_status_t;
enum {
  GSRB_OK = 0,
  GSRB_ERR_ARG = -1,             /* invalid argument */
  GSRB_ERR_CUDA = -2,            /* a CUDA runtime call failed */
  GSRB_ERR_NOT_CORESIDENT = -3,  /* persistent grid larger than the co-resident capacity: refused */
  GSRB_ERR_TIMEOUT = -4,         /* a device-side bounded wait ran out */
  GSRB_ERR_NOMEM = -5,
  GSRB_ERR_STATE = -6,           /* context in a bad state (e.g. sticky device error) */
  GSRB_ERR_UNSUPPORTED = -7,
  GSRB_ERR_OVERFLOW = -8,        /* a device worklist / scratch area would overflow */
  GSRB_ERR_LOCK_TIMEOUT = -9,    /* a mutex / semaphore wait ran out */
  GSRB_ERR_INVARIANT = -10       /* a device-checked invariant failed */
};

typedef struct gsrb_ctx* gsrb_ctx_t;

/* Barrier variants (gsrb_cfg_t.variant). */
enum {
  GSRB_BAR_CLUSTER = 0,          /* 3-level: HW cluster barrier -> L2 counter -> HW cluster release */
  GSRB_BAR_CLUSTER_ALLPOLL = 1,  /* 3-level: HW cluster arrival, every CTA polls the L2 generation */
  GSRB_BAR_DSMEM = 2,            /* 3-level: DSMEM arrival counter / DSMEM release flags */
  GSRB_BAR_SOFT2 = 3,            /* reference GSRB: software per-group counters -> global */
  GSRB_BAR_FLAT = 4,             /* reference GCPUSRB: one counter for all CTAs */
  GSRB_BAR_TREE = 5,             /* HeteroSync atomic tree barrier (paper baseline) */
  GSRB_BAR_CCG = 6,              /* cooperative_groups grid.sync() (library baseline) */
  GSRB_BAR_CLUSTER_RED = 7,      /* 3-level, completer-publishes protocol (red.release arrivals, polling master) */
  GSRB_BAR_FLIP = 8,             /* 2-level: every CTA arrives on the split sum-to-flip words */
  GSRB_BAR_FANOUT = 9,           /* 2-level: counter + generation published to R wake-up lines */
  GSRB_BAR_CLUSTER_FANOUT = 10,  /* 3-level: HW cluster arrival, leader on the counter, R wake-up lines */
  GSRB_BAR_HIER = 11,            /* 3-level: group counters (fanin_groups) -> root counter -> R wake-up lines */
  GSRB_BAR_LOCKFREE = 12,        /* reference HeteroSync lock-free tree barrier (in/out flag arrays; per-SM
                                    local level when there is more than one CTA per SM); barrier benchmark only */
  GSRB_BAR_NONE = 99             /* no barrier (phase-only timing baseline) */
};

/* Data-kernel forms (gsrb_cfg_t.form). */
enum { GSRB_FORM_AUTO = 0, GSRB_FORM_L2 = 1, GSRB_FORM_L1 = 2, GSRB_FORM_REG = 3 };

/* Launch / schedule configuration.  Zero-initialise and call gsrb_cfg_default. */
typedef struct gsrb_cfg {
  int32_t variant;       /* GSRB_BAR_* */
  int32_t cluster;       /* CTAs per cluster for the cluster variants (1,2,4,8,16) */
  int32_t ctas_per_sm;   /* persistent CTAs per SM (grid = ctas_per_sm * #SMs) */
  int32_t threads;       /* threads per CTA */
  int32_t fanin_groups;  /* global fan-in groups (0 = arrive at the root directly) */
  int32_t spin_ns;       /* __nanosleep between polls (0 = hot spin) */
  uint32_t timeout_ms;   /* per-wait device deadline */
  int32_t tile;          /* scan: elements per CTA chunk; reduce: 32 KiB stages (0 = auto) */
  int32_t grid_override; /* exact grid size (0 = ctas_per_sm * #SMs) */
  int32_t launch_mode;   /* 0 = cooperative launch when the driver accepts it, 1 = plain launch (default)
                            (both only after the co-residency check; CCG is always cooperative) */
  int32_t wake_lines;    /* FANOUT / CLUSTER_FANOUT / HIER: wake-up lines the generation is published to (0 = 8) */
  int32_t form;          /* pull PageRank: GSRB_FORM_AUTO and GSRB_FORM_L1 gather x/deg through L1 (ld.ca),
                            GSRB_FORM_L2 through L2 only (ld.cg).  Segmented scans: GSRB_FORM_REG keeps
                            each round's chunk in registers from its sum to its rescan (GSRB_BAR_FANOUT);
                            other forms stage tiles through shared memory and re-read L2.  Other kernels
                            ignore it */
  int32_t overlap;       /* gsrb_reduce_i32 only, plain launches only: 1 = the launch may start, and read
                            d_in, while the kernel before it on the stream is still running (programmatic
                            dependent launch); it touches no other memory until that kernel has finished.
                            Set it only when that kernel does not write d_in -- e.g. in a chain of
                            reductions over inputs that were all ready before the chain began.  0 = off */
  int32_t reserved[3];
} gsrb_cfg_t;

void gsrb_cfg_default(gsrb_cfg_t* cfg);
const char* gsrb_status_string(gsrb_status_t s);

/* ---- context ---------------------------------------------------------------- */
gsrb_status_t gsrb_ctx_create(int device, gsrb_ctx_t* out);
/* Release every graph and batch created on the context first: their free
 * functions synchronise the context stream. */
gsrb_status_t gsrb_ctx_destroy(gsrb_ctx_t ctx);
/* Use an existing cudaStream_t (passed as void*); NULL = the context's own stream. */
gsrb_status_t gsrb_ctx_set_stream(gsrb_ctx_t ctx, void* stream);
/* Device facts: number of SMs, L2 bytes, device ordinal. */
gsrb_status_t gsrb_ctx_info(gsrb_ctx_t ctx, int32_t* num_sms, int64_t* l2_bytes, int32_t* device);
/* Synchronous: wait for the context's stream, read the sticky device status and
 * clear it.  Returns GSRB_OK or the mapped error; `dev_code`, `where`
 * (episode) and `who` (block) describe the first device error (may be NULL). */
gsrb_status_t gsrb_ctx_status(gsrb_ctx_t ctx, uint32_t* dev_code, uint32_t* where, uint32_t* who);
gsrb_status_t gsrb_ctx_synchronize(gsrb_ctx_t ctx);
/* Largest co-resident grid for a barrier configuration (CTAs), for a given kernel family:
 * 0 = barrier microbenchmark, 1 = reduce, 2 = scan, 3 = graph traversal. */
gsrb_status_t gsrb_max_coresident(gsrb_ctx_t ctx, const gsrb_cfg_t* cfg, int32_t family, int32_t* ctas);

/* ---- memory plumbing (device, pinned host) ----------------------------------- */
gsrb_status_t gsrb_malloc(void** d_ptr, size_t bytes);
gsrb_status_t gsrb_free(void* d_ptr);
gsrb_status_t gsrb_host_alloc(void** h_ptr, size_t bytes);   /* pinned */
gsrb_status_t gsrb_host_free(void* h_ptr);
gsrb_status_t gsrb_memcpy_h2d(gsrb_ctx_t ctx, void* d_dst, const void* h_src, size_t bytes);   /* async */
gsrb_status_t gsrb_memcpy_d2h(gsrb_ctx_t ctx, void* h_dst, const void* d_src, size_t bytes);   /* async */
gsrb_status_t gsrb_memset(gsrb_ctx_t ctx, void* d_ptr, int value, size_t bytes);               /* async */

/* ---- timing helpers (CUDA events recorded on the context stream) -------------- */
gsrb_status_t gsrb_event_record(gsrb_ctx_t ctx, int32_t slot);        /* slot 0..63 */
gsrb_status_t gsrb_event_elapsed_ms(gsrb_ctx_t ctx, int32_t a, int32_t b, float* ms); /* synchronous */
/* Write a buffer larger than L2 to evict the inputs of the next timed launch. */
gsrb_status_t gsrb_l2_flush(gsrb_ctx_t ctx);
/* Number of kernels this library has launched in this process (for launch accounting). */
uint64_t gsrb_launch_count(void);

/* ---- grid barrier microbenchmark (148*k CTAs, episodes of F FMAs + one barrier) 
 * One persistent launch of grid = cfg->ctas_per_sm * #SMs CTAs of cfg->threads
 * threads; each CTA runs `episodes` times: `fma_per_episode` dependent FP32 FMAs
 * per thread, then one grid barrier of cfg->variant.  d_episode_count (uint32,
 * zeroed by the caller) receives the sum over CTAs of completed episodes
 * (must equal episodes * grid).  d_sink: >= grid*threads floats, written with
 * the FMA results.  Reference: kernelAtomicTreeBarrierUniqSRB,
 * Heterosync/main.cu:188-226, launched by invokeAtomicTreeBarrierSRB :1532-1562. */
gsrb_status_t gsrb_barrier_bench(gsrb_ctx_t ctx, const gsrb_cfg_t* cfg, int32_t episodes,
                                 int32_t fma_per_episode, float* d_sink, uint32_t* d_episode_count);
/* Message-passing litmus test across the barrier: every episode each thread writes
 * a stamp, barrier, reads another CTA's stamp, barrier.  d_buf: grid*threads
 * uint32; d_stale (uint64, zeroed by caller) receives the number of stale reads. */
gsrb_status_t gsrb_barrier_litmus(gsrb_ctx_t ctx, const gsrb_cfg_t* cfg, int32_t episodes,
                                  uint32_t* d_buf, unsigned long long* d_stale);
/* Fault test: launch a barrier kernel whose expected arrival count is one more
 * than the grid, so every wait must run out after cfg->timeout_ms and report
 * GSRB_ERR_TIMEOUT (synchronous).  The context stays usable afterwards. */
gsrb_status_t gsrb_barrier_fault_short_grid(gsrb_ctx_t ctx, const gsrb_cfg_t* cfg);

/* L2 atomic probes (synchronous, ms via CUDA events): mode 0 = `ctas` CTAs each
 * issue `iters` red.add to one address from one thread (same-address throughput);
 * mode 1 = one thread issues `iters` dependent atom.add (round-trip latency). */
gsrb_status_t gsrb_probe_l2_atomics(gsrb_ctx_t ctx, int32_t ctas, int32_t iters, int32_t mode, float* ms);

/* ---- reduce (2^24 int32, one barrier between partials and combine) ------------
 * Sum of n int32 into *d_out (int64), one persistent launch: each CTA streams a
 * contiguous chunk through a ring of 32 KiB shared-memory stages filled by
 * cp.async.bulk (cfg->tile = stages, 0 = as many as fit, at most 6), one grid
 * barrier, CTA 0 combines the partials in a fixed order.  cfg == NULL: one
 * 1024-thread CTA per SM.  Replaces reduce_kernel/reduce() of
 * Reduce/reduce_gsrb.cu:289-404 (API Reduce/reduce.cuh:19).  Asynchronous. */
gsrb_status_t gsrb_reduce_i32(gsrb_ctx_t ctx, const int32_t* d_in, size_t n, int64_t* d_out,
                              const gsrb_cfg_t* cfg);

/* Allocation-free variant of gsrb_reduce_i32 (no counterpart in the reference).
 * For callers that must not allocate device memory -- code running inside a
 * host framework's fixed memory budget, or a plugin that may not grow the
 * device footprint or call cudaMalloc -- and therefore cannot create a context.
 * The barrier state and the per-CTA partials live in one fixed static device
 * array of 17 KiB, which every GPU that loads the library holds until exit; the
 * call needs only d_in, d_out and a stream (NULL = legacy default stream) and
 * calls no cudaMalloc / cudaFree.  Limits: n <= 2^32 elements (larger n returns
 * GSRB_ERR_ARG), grid = 2 CTAs per SM (at most 2048 CTAs).  The first call on a
 * device looks up the array's device address with that device current; make it
 * before any stream capture.  Every call clears the array's barrier words and
 * reuses it, so calls whose kernels overlap on the GPU race.  The looked-up
 * address is kept for the life of the process: do not call it again after a
 * cudaDeviceReset of that device.  Synchronous with respect to `stream`;
 * returns GSRB_ERR_TIMEOUT if a bounded wait (2 s) ran out -- on a GPU shared
 * with other running kernels this can also mean that the 2-CTAs-per-SM grid
 * could not all be resident at once (the launch is not cooperative, and the
 * occupancy check before it cannot see other processes' kernels). */
gsrb_status_t gsrb_reduce_i32_noalloc(const int32_t* d_in, size_t n, int64_t* d_out, void* stream);

/* ---- scan (three-phase persistent exclusive prefix sum) ---------------------------
 * Exclusive prefix sum, one persistent launch (default one 1024-thread CTA per
 * SM).  The input is walked in segments of one chunk per CTA (cfg->tile
 * elements, 0 = 32768); per segment: chunk sums, one split-phase grid barrier
 * that overlaps the next segment's reads, then the chunk is re-read from L2,
 * scanned and written.  uint32 wraps around like the reference's
 * cpu_sum_scan; the FP32 variant keeps chunk offsets in FP64.
 * In-place (d_in == d_out) is allowed.  Replaces gpu_prescan /
 * sum_scan_blelloch of scan/scan_gsrb.cu:486-804 (API scan/scan.h:16-18).
 * Asynchronous. */
gsrb_status_t gsrb_scan_u32(gsrb_ctx_t ctx, const uint32_t* d_in, uint32_t* d_out, size_t n,
                            const gsrb_cfg_t* cfg);
gsrb_status_t gsrb_scan_f32(gsrb_ctx_t ctx, const float* d_in, float* d_out, size_t n, const gsrb_cfg_t* cfg);

/* ---- batched reduce / scan segments (no counterpart in the reference) -------------
 * k independent segments of uneven lengths, segment i = elements
 * [h_off[i], h_off[i+1]) of d_in (host offsets, non-decreasing, 1 <= k <= 127,
 * total < 2^47), in one persistent launch.  Segment i gets CTAs
 * [first_i, first_i + count_i): first_i = i + floor((grid - k) * (h_off[i] -
 * h_off[0]) / (h_off[k] - h_off[0])) (every segment at least one CTA, the rest
 * in proportion to length), and synchronises them on its own sub-grid barrier
 * (slot 1 + i).  The layout is computed on the device from the launch
 * parameters, so nothing is copied per call and calls can be captured
 * (gsrb_capture_begin/end).  cfg == NULL: GSRB_BAR_FANOUT, 2 x 512 threads per
 * SM for the reduce, 4 x 256 and GSRB_FORM_REG for the scan; cfg->variant must be GSRB_BAR_FANOUT, GSRB_BAR_FLIP or GSRB_BAR_FLAT; grid
 * >= k.  Asynchronous; a bounded wait that ran out is reported by
 * gsrb_ctx_status. */
/* d_out[i] = int64 sum of segment i (0 for an empty segment), bit-exact. */
gsrb_status_t gsrb_reduce_i32_segments(gsrb_ctx_t ctx, const int32_t* d_in, const uint64_t* h_off, int32_t k,
                                       int64_t* d_out, const gsrb_cfg_t* cfg);
/* Exclusive uint32 prefix sum within each segment (wrapping; each segment starts
 * at 0), written at the same offsets of d_out.  Not in place.  A segment is
 * scanned in rounds of cfg->tile elements per CTA (rounded up to whole tiles of
 * 16 x threads; 0 = 4 tiles), chunk sums and one sub-grid barrier per round, so
 * that the rescan re-reads L2.  With cfg->form = GSRB_FORM_REG (GSRB_BAR_FANOUT
 * only) the CTA's threads form 2-4 groups that take the rounds in turn and keep
 * their chunk in registers from its sum to its rescan: cfg->tile is then the
 * chunk, threads x 4 x (16 vectors a lane when ctas_per_sm x threads <= 512,
 * else 8) divided by the number of groups (0 = two groups); other values
 * return GSRB_ERR_ARG. */
gsrb_status_t gsrb_scan_u32_segments(gsrb_ctx_t ctx, const uint32_t* d_in, uint32_t* d_out, const uint64_t* h_off,
                                     int32_t k, const gsrb_cfg_t* cfg);
/* The same for FP32: chunk sums and carries in FP64, each tile scanned in FP32
 * (within 1e-5 relative of an FP64 prefix, as gsrb_scan_f32). */
gsrb_status_t gsrb_scan_f32_segments(gsrb_ctx_t ctx, const float* d_in, float* d_out, const uint64_t* h_off,
                                     int32_t k, const gsrb_cfg_t* cfg);
/* Host: the CTA layout those calls use for a grid of `grid` CTAs (first[k], count[k]). */
gsrb_status_t gsrb_segments_layout(const uint64_t* h_off, int32_t k, int32_t grid, uint32_t* first, uint32_t* count);

/* ---- lock state, mutexes and semaphores (the Heterosync cudaLocks layer) -------
 * The reference-named host API (cudaLocksInit, cudaMutexCreate*, ...) is in
 * gsrb/cudaLocks.h and the device API in gsrb/cudaLocks.cuh; these are the
 * context-scoped equivalents (no global instance). */
typedef struct gsrb_lock_data {  /* device pointers, layout of cudaLockData_t (Heterosync/cudaLocks.h:4-17) */
  int32_t maxBufferSize;
  int32_t arrayStride;
  int32_t mutexCount;
  int32_t semaphoreCount;
  uint32_t* barrierBuffers;
  int32_t* mutexBuffers;
  uint32_t* mutexBufferHeads;
  uint32_t* mutexBufferTails;
  uint32_t* semaphoreBuffers;
} gsrb_lock_data_t;
typedef struct gsrb_locks* gsrb_locks_t;

/* Allocates and initialises lock state like cudaLocksInit (Heterosync/cudaLocks.cu:3-87). */
gsrb_status_t gsrb_locks_create(gsrb_ctx_t ctx, int32_t maxBlocks, int32_t numMutexes, int32_t numSemaphores,
                                int32_t numSM, gsrb_locks_t* out);
gsrb_status_t gsrb_locks_destroy(gsrb_locks_t locks);
gsrb_status_t gsrb_locks_data(gsrb_locks_t locks, gsrb_lock_data_t* out);
/* Semaphore record of cudaSemaphoreCreateSpin (Heterosync/cudaLocksSemaphoreSpin.cu:6-29). */
gsrb_status_t gsrb_semaphore_init(gsrb_locks_t locks, int32_t semNum, uint32_t count, int32_t numSM);
/* Synchronous: first status code recorded by a bounded lock wait (cleared). */
gsrb_status_t gsrb_locks_status(gsrb_locks_t locks, uint32_t* code);

/* Semaphore kinds for gsrb_semaphore_bench. */
enum {
  GSRB_SEM_REF_SPIN = 0,          /* reference spin semaphore protocol (lock word + count) */
  GSRB_SEM_REF_EBO = 1,           /* ... with exponential backoff */
  GSRB_SEM_REF_PRIORITY = 2,      /* reference TPDS'22 priority semaphore protocol */
  GSRB_SEM_REF_PRIORITY_EBO = 3,  /* ... with exponential backoff */
  GSRB_SEM_PRIORITY = 4,          /* B200-native priority semaphore (wait-free posts, writer queue) */
  GSRB_SEM_NONE = 5               /* no semaphore: the critical sections alone (on one CTA, what a hold
                                     costs by itself; counts are not exact on more CTAs) */
};
/* Mutex kinds for gsrb_mutex_bench. */
enum { GSRB_MUTEX_SPIN = 0, GSRB_MUTEX_EBO = 1, GSRB_MUTEX_FA = 2, GSRB_MUTEX_SLEEP = 3 };

/* Semaphore microbenchmark: grid = cfg CTAs; CTA b is a
 * writer when writer_every > 0 and b % writer_every == 0 (writer_every = 0: no
 * writers); each CTA acquires `iters` times and adds 1
 * to a shared counter `incs` times per acquire (writers: plain read-modify-write
 * of W; readers: atomic add to R).  d_counters: 8 uint32, zeroed by the caller:
 * [W, R, inside, max_readers, violations, acquires, timeouts, 0].  Synchronous.
 * Reference: kernelSpinLockSemaphorePriority, Heterosync/main.cu:962-1040. */
gsrb_status_t gsrb_semaphore_bench(gsrb_ctx_t ctx, const gsrb_cfg_t* cfg, int32_t kind, uint32_t capacity,
                                   int32_t writer_every, int32_t iters, int32_t incs, uint32_t* d_counters);
/* Fault test: a semaphore of `capacity` (GSRB_SEM_PRIORITY protocol) is posted
 * once by a CTA that never waited on it (an over-post), then waited on by that
 * CTA as a reader and as a writer.  Both waits see the count above its maximum
 * and fail at once; returns GSRB_ERR_INVARIANT (synchronous).  d_out: 2 uint32,
 * 1 where the reader / writer wait succeeded, else 0. */
gsrb_status_t gsrb_semaphore_fault_overpost(gsrb_ctx_t ctx, uint32_t capacity, uint32_t* d_out);
/* Fault test of a writer that gives up (no counterpart in the reference): one
 * CTA enters a GSRB_SEM_PRIORITY semaphore as a reader, then waits on it as a
 * writer while still holding the reader slot, so that wait is served its turn
 * but runs into a 20 ms deadline on the count; the CTA leaves as a reader and
 * waits as a writer again.  A served writer that gives up hands its turn on,
 * so the second writer wait succeeds.  Returns GSRB_ERR_LOCK_TIMEOUT (the first
 * writer's); d_out: 5 uint32 = [reader entered, first writer entered, second
 * writer entered, count afterwards, serving afterwards].
 * A writer that gives up while still waiting for its turn leaves its ticket
 * unserved: every later writer of that record then runs into its own deadline
 * until the record is re-created (gsrb_semaphore_init / cudaSemaphoreCreate*),
 * as after any wait that reported GSRB_ERR_INVARIANT.  Synchronous. */
gsrb_status_t gsrb_semaphore_fault_writer_timeout(gsrb_ctx_t ctx, uint32_t capacity, uint32_t* d_out);
/* Mutex microbenchmark: every CTA locks `iters` times and adds 1 to W `incs`
 * times with a plain read-modify-write.  Same counter layout.  Synchronous.
 * Reference: kernelSpinLockMutex / EBO / FA / Sleep, Heterosync/main.cu:574-700. */
gsrb_status_t gsrb_mutex_bench(gsrb_ctx_t ctx, const gsrb_cfg_t* cfg, int32_t kind, int32_t iters, int32_t incs,
                               uint32_t* d_counters);

/* ---- graph traversals (BFS / SSSP / PageRank level loops) -------------------------
 * A gsrb_graph_t is a device CSR (row_start[n+1], edge_dst[m], edge_data[m]:
 * the reference CSRGraph layout) plus the traversal scratch (queues, marks,
 * counters, per-level trace ring).  Traversals are synchronous and return
 * statistics.  Replaces the gg_main of LONESTAR/apps/{bfs,sssp,pr}/kernel_gsrb.cu
 * (bfs :712-730, sssp :791-820, pr :683-715). */
typedef struct gsrb_graph* gsrb_graph_t;
typedef struct gsrb_host_csr gsrb_host_csr_t;  /* defined with the host-side graph section below */
typedef struct gsrb_traversal_stats {
  uint32_t levels;        /* BFS levels / SSSP relax rounds / PR iterations */
  uint32_t aux;           /* BFS (learned): first level that fell back to the heuristic (0 = none);
                             SSSP: buckets */
  uint32_t decisions;     /* BFS (learned): levels decided by the policy network */
  uint32_t trace_records; /* per-level trace records available (gsrb_graph_trace) */
  uint64_t edges;         /* BFS: out-edges of reached vertices (the TEPS numerator);
                             SSSP: edges relaxed */
  float kernel_ms;        /* CUDA-event time of the traversal launch */
  uint32_t launch;        /* BFS / SSSP (learned, cfg NULL, launch choices set): 1 + the index of the
                             launch configuration the policy picked; else 0 */
  int32_t delta;          /* SSSP: the bucket width the traversal ran with */
} gsrb_traversal_stats_t;

/* BFS direction modes. */
enum {
  GSRB_BFS_PUSH = 0,      /* worklist push every level (the reference's data-driven BFS) */
  GSRB_BFS_HEURISTIC = 1, /* direction-optimizing with the fixed Beamer thresholds (alpha 15, beta 18) */
  GSRB_BFS_LEARNED = 2,   /* the policy network decides; falls back to the heuristic after a 2x miss */
  GSRB_BFS_PULL = 3,      /* pull every level after the first (trace collection) */
  GSRB_BFS_TOPO = 4,      /* topology-driven push every level (trace collection) */
  /* OR-ed into any mode: push levels with >= 65536 frontier edges expand with
   * the load balancer of the reference's -l option (per-CTA degree totals,
   * prefix offsets, every warp the same number of edges; two extra barriers
   * per such level).  gsrb_bfs only; batches reject it. */
  GSRB_BFS_FLAG_LB = 0x100
};

/* Copy a host CSR to the device (owned by the graph). */
gsrb_status_t gsrb_graph_upload(gsrb_ctx_t ctx, const gsrb_host_csr_t* h, gsrb_graph_t* out);
/* Wrap caller-owned device CSR arrays (not freed by gsrb_graph_free). */
gsrb_status_t gsrb_graph_wrap(gsrb_ctx_t ctx, uint32_t n, uint64_t m, const uint32_t* d_row,
                              const uint32_t* d_dst, const int32_t* d_w, gsrb_graph_t* out);
gsrb_status_t gsrb_graph_free(gsrb_graph_t g);
/* nhubs: vertices of degree > 128, whose rows PageRank splits into 2048-edge chunks. */
gsrb_status_t gsrb_graph_info(gsrb_graph_t g, uint32_t* n, uint64_t* m, uint32_t* nhubs);
/* 1 if every edge (u, v) has its reverse (v, u), else 0; tested when the graph
 * is created (hash sums of the edges and of their reverses).  Pull levels of a
 * BFS and the pull PageRank read a row as the vertex's in-edges, so on a
 * graph that is not symmetric BFS never pulls (GSRB_BFS_PULL and gsrb_pagerank
 * return GSRB_ERR_UNSUPPORTED; gsrb_pagerank_residual pushes and takes any graph). */
gsrb_status_t gsrb_graph_is_symmetric(gsrb_graph_t g, int32_t* symmetric);
/* Policy network weights (gsrb_mlp_* layout, gsrb_mlp_param_count() floats). */
gsrb_status_t gsrb_graph_set_policy(gsrb_graph_t g, const float* h_weights, size_t count);
/* Two launch configurations (barrier variant, CTAs per SM, threads) for
 * learned traversals: gsrb_bfs in GSRB_BFS_LEARNED mode with cfg == NULL then
 * runs the one head 3 of the policy picks.  Both NULL: forget them. */
gsrb_status_t gsrb_graph_set_launch_choices(gsrb_graph_t g, const gsrb_cfg_t* cfg0, const gsrb_cfg_t* cfg1);
/* The policy's launch choice for a BFS from src: head 3 evaluated on the host
 * on the first level's features (frontier = src); *choice = 1 if it is > 0,
 * else 0; *score (may be NULL) = head 3.  GSRB_ERR_STATE without a policy. */
gsrb_status_t gsrb_graph_policy_launch(gsrb_graph_t g, uint32_t src, int32_t* choice, float* score);
/* Copy up to max_records 48-byte per-level trace records of the last traversal. */
gsrb_status_t gsrb_graph_trace(gsrb_graph_t g, void* h_out, uint32_t max_records, uint32_t* records);
/* BFS levels from src into d_level (int32[n]; INT32_MAX = unreachable).
 * cfg == NULL: 2 CTAs x 512 threads per SM. */
gsrb_status_t gsrb_bfs(gsrb_ctx_t ctx, gsrb_graph_t g, uint32_t src, int32_t* d_level, int32_t mode,
                       const gsrb_cfg_t* cfg, gsrb_traversal_stats_t* stats);
/* SSSP distances (near-far buckets of width delta) into d_dist (int32[n]).
 * delta == GSRB_SSSP_DELTA_LEARNED: the graph's SSSP policy picks the width
 * (and, with cfg == NULL and launch choices set, the launch configuration);
 * GSRB_ERR_STATE without one.  The distances do not depend on either. */
enum { GSRB_SSSP_DELTA_LEARNED = 0 };
gsrb_status_t gsrb_sssp(gsrb_ctx_t ctx, gsrb_graph_t g, uint32_t src, int32_t* d_dist, int32_t delta,
                        const gsrb_cfg_t* cfg, gsrb_traversal_stats_t* stats);
/* The SSSP policy (no counterpart in the reference; the reference runs every
 * graph with DELTA = 10000, LONESTAR/apps/sssp/support.cu:10, and one launch
 * shape): the policy network's layout (gsrb_mlp_*), its own weights, evaluated
 * on the host once per traversal on gsrb_sssp_features of the graph and the
 * source.  Head 2: log2 of the bucket width over the graph's mean edge weight;
 * head 3: log2(t0 / t1), the traversal time under launch configuration 0 over
 * that under configuration 1.  h_weights NULL: forget the policy. */
gsrb_status_t gsrb_graph_set_sssp_policy(gsrb_graph_t g, const float* h_weights, size_t count);
/* The policy's plan for an SSSP from src: *delta = round(2^head2 * mean weight)
 * clamped to [1, 2^30]; *choice = head 3 > 0; scores[2] = {head 2, head 3}
 * (any output may be NULL).  GSRB_ERR_STATE without an SSSP policy. */
gsrb_status_t gsrb_graph_sssp_plan(gsrb_graph_t g, uint32_t src, int32_t* delta, int32_t* choice, float* scores);
/* The 12 features of the SSSP policy: log2 of n, m, mean degree, maximum
 * degree, the source's degree, mean / maximum / minimum edge weight (each
 * 1 + x), symmetric (0/1), degree skew, weight spread, log2 n - 2 log2 mean
 * degree.  The graph form reads the statistics taken when the graph was created. */
void gsrb_sssp_features(uint32_t n, uint64_t m, uint32_t max_degree, uint32_t src_degree, double w_mean,
                        int32_t w_min, int32_t w_max, int32_t symmetric, float* h_out12);
gsrb_status_t gsrb_graph_sssp_features(gsrb_graph_t g, uint32_t src, float* h_out12);
/* Pull PageRank: x0 = 1 - alpha, `iters` iterations of x = (1-alpha) + alpha * sum x_u/deg(u). */
gsrb_status_t gsrb_pagerank(gsrb_ctx_t ctx, gsrb_graph_t g, float alpha, int32_t iters, float* d_rank,
                            const gsrb_cfg_t* cfg, gsrb_traversal_stats_t* stats);
/* The gather floor of a pull pass over g (no counterpart in the reference):
 * one edge-parallel launch that gathers an FP32 value at every edge's
 * destination (the pull PageRank's x/deg reads without its per-vertex
 * bookkeeping), through L1 (l1 != 0) or L2 only; *ms = its time, mean of 10
 * back-to-back launches.  Synchronous.  The roofline of the pull PageRank. */
gsrb_status_t gsrb_probe_gather(gsrb_ctx_t ctx, gsrb_graph_t g, int32_t l1, float* ms);
/* The reference's push-residual PageRank (apps/pr/kernel_gsrb.cu:298-508):
 * p = 1 - alpha, residuals seeded with (1 - alpha) * alpha * sum 1/outdeg, then
 * rounds of "take the residual, add it to p, push alpha * res / outdeg along
 * every out-edge" over a worklist of vertices whose residual crossed epsilon,
 * until the worklist is empty or max_iters rounds ran.  FP32 atomics in a
 * run-dependent order (as in the reference).  stats->levels = rounds,
 * stats->edges = worklist pushes. */
gsrb_status_t gsrb_pagerank_residual(gsrb_ctx_t ctx, gsrb_graph_t g, float alpha, float epsilon, int32_t max_iters,
                                     float* d_rank, const gsrb_cfg_t* cfg, gsrb_traversal_stats_t* stats);

/* ---- batched traversals (many graphs, one persistent launch) ----------------------
 * k graphs (k <= 127) traversed in ONE persistent launch: instance i owns a
 * contiguous range of CTAs (in proportion to its edges, at least one) and a
 * sub-grid barrier of its own carved from the context's barrier state, so
 * instances never wait for each other.  cfg->variant must not use hardware
 * cluster barriers (SOFT2, FLAT, TREE, FLIP, FANOUT; default FANOUT).
 * The launches are asynchronous and can be captured in a CUDA graph. */
typedef struct gsrb_batch* gsrb_batch_t;
gsrb_status_t gsrb_batch_create(gsrb_ctx_t ctx, const gsrb_graph_t* graphs, int32_t k, const gsrb_cfg_t* cfg,
                                gsrb_batch_t* out);
gsrb_status_t gsrb_batch_free(gsrb_batch_t b);
/* CTA range of every instance (arrays of k, may be NULL). */
gsrb_status_t gsrb_batch_layout(gsrb_batch_t b, uint32_t* first, uint32_t* count);
/* Asynchronous: BFS of every instance (d_levels[i] int32[n_i]) / SSSP (d_dists[i];
 * delta == GSRB_SSSP_DELTA_LEARNED: every instance the width of its graph's SSSP policy). */
gsrb_status_t gsrb_batch_bfs(gsrb_batch_t b, const uint32_t* srcs, int32_t* const* d_levels, int32_t mode);
gsrb_status_t gsrb_batch_sssp(gsrb_batch_t b, const uint32_t* srcs, int32_t* const* d_dists, int32_t delta);
/* Synchronous: per-instance statistics of the last batched launch (array of k). */
gsrb_status_t gsrb_batch_stats(gsrb_batch_t b, gsrb_traversal_stats_t* stats);

/* CUDA graphs over the context stream: capture asynchronous calls, replay them. */
typedef struct gsrb_exec* gsrb_exec_t;
gsrb_status_t gsrb_capture_begin(gsrb_ctx_t ctx);
gsrb_status_t gsrb_capture_end(gsrb_ctx_t ctx, gsrb_exec_t* out);
gsrb_status_t gsrb_exec_launch(gsrb_ctx_t ctx, gsrb_exec_t exec);
gsrb_status_t gsrb_exec_free(gsrb_exec_t exec);

/* ---- the learned policy: a 12 -> 32 -> 32 -> 4 FP32 MLP -----------------------------
 * Parameter layout (floats): w1[32][12], b1[32], w2[32][32], b2[32], w3[4][32], b3[4].
 * Heads: [0] logit(pull faster than push), [1] logit(topology push faster than
 * worklist push), [2] log2(1 + next frontier size), [3] log2(t0 / t1), the
 * traversal time under launch configuration 0 over that under configuration 1
 * (gsrb_graph_set_launch_choices; read on the first level only).  Loss: masked
 * BCE-with-logits on heads 0-1, masked 0.5*(z-y)^2 on heads 2-3, batch mean.
 * No counterpart in the reference (its traversals use fixed schedules). */
size_t gsrb_mlp_param_count(void);
/* He-uniform initialisation from a seed (host). */
gsrb_status_t gsrb_mlp_init(uint64_t seed, float* h_params);
/* The 12 features of a level, as the traversal computes them on the device. */
void gsrb_level_features(uint32_t n, uint32_t m, uint32_t level, uint32_t nf, uint64_t mf, uint32_t nu, uint64_t mu,
                         uint32_t prev_nf, uint32_t prev_dir, float* h_out12);
/* Inference: d_out[B][4] from d_x[B][12].  Asynchronous. */
gsrb_status_t gsrb_mlp_forward(gsrb_ctx_t ctx, const float* d_params, const float* d_x, int32_t B, float* d_out);
/* One loss + gradient evaluation (d_grad: param_count floats, d_loss: 1 float).  Asynchronous. */
gsrb_status_t gsrb_mlp_loss_grad(gsrb_ctx_t ctx, const float* d_params, const float* d_x, const float* d_y,
                                 const float* d_mask, int32_t B, float* d_grad, float* d_loss);
/* Full-batch Adam training, `steps` steps, in one persistent launch (grid barrier
 * between the forward/backward and the update phases).  d_loss_hist: steps floats
 * (may be NULL).  Asynchronous. */
gsrb_status_t gsrb_mlp_train(gsrb_ctx_t ctx, float* d_params, const float* d_x, const float* d_y,
                             const float* d_mask, int32_t B, int32_t steps, float lr, float* d_loss_hist);

/* ---- host-side graphs and synthetic inputs ----------------------------------------
 * CSR in the layout of the reference CSRGraph (row_start[n+1], edge_dst[m],
 * edge_data[m]; LONESTAR/rt/include/csr_graph.h.prehip:20-103).  Host memory
 * allocated by the library; release with gsrb_host_csr_free. */
typedef struct gsrb_host_csr {
  uint32_t nnodes;
  uint32_t _pad;
  uint64_t nedges;
  uint32_t* row_start;
  uint32_t* edge_dst;
  int32_t* edge_data;
} gsrb_host_csr_t;

void gsrb_host_csr_free(gsrb_host_csr_t* g);
/* Seeded uniform integers in [lo, hi] / floats in [0, 1) (splitmix64-seeded
 * xoshiro256**, one stream per 65536-element block: independent of thread count). */
gsrb_status_t gsrb_gen_uniform_i32(uint64_t seed, size_t n, int32_t lo, int32_t hi, int32_t* h_out);
gsrb_status_t gsrb_gen_uniform_f32(uint64_t seed, size_t n, float* h_out);
/* Symmetric weight of the unordered pair {u, v}, uniform in [lo, hi]. */
uint32_t gsrb_edge_weight(uint32_t u, uint32_t v, uint64_t seed, int32_t lo, int32_t hi);
/* CSR with sorted, duplicate-free rows and no self loops from an edge list
 * (symmetrize != 0 inserts both directions); weights from gsrb_edge_weight. */
gsrb_status_t gsrb_csr_from_edges(uint32_t n, uint64_t m, const uint32_t* h_src, const uint32_t* h_dst,
                                  int symmetrize, uint64_t weight_seed, int32_t wlo, int32_t whi,
                                  gsrb_host_csr_t* out);
/* R-MAT (scale, edge factor, a, b, c), symmetrised and deduplicated. */
gsrb_status_t gsrb_gen_rmat(int32_t scale, int32_t edgefactor, double a, double b, double c, uint64_t seed,
                            int32_t wlo, int32_t whi, gsrb_host_csr_t* out);
/* width x height 4-neighbour grid (vertex id = row * width + col). */
gsrb_status_t gsrb_gen_grid2d(int32_t width, int32_t height, uint64_t seed, int32_t wlo, int32_t whi,
                              gsrb_host_csr_t* out);
/* Galois `.gr` version 1 reader / writer (LONESTAR/rt/src/csr_graph.cu:152-237). */
gsrb_status_t gsrb_gr_read(const char* path, gsrb_host_csr_t* out);
gsrb_status_t gsrb_gr_write(const char* path, const gsrb_host_csr_t* g, int32_t with_weights);

#ifdef __cplusplus
}
#endif
#endif /* GSRB_H_ */
