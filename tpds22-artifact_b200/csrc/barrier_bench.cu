// Grid-barrier microbenchmark, message-passing litmus test and the short-grid
// fault test.
//
// Reference: the Heterosync barrier microbenchmarks (Heterosync/main.cu:111-305,
// launched by invokeAtomicTreeBarrier* :1495-1610) time NUM_REPEATS launches of
// a kernel that alternates a data phase with joinBarrier_helper*().  The
// configuration measured here replaces the cache-line copy phase with F
// dependent FP32 FMAs per thread (so that the phase has no memory traffic) and
// runs 148*k CTAs of 256 threads, k in {1,2,4,8}.
#include "internal.h"

using namespace gsrbrt;

namespace {

constexpr int kNoBarrier = 99;

template <int V>
struct MaybeSync {
  gsrb::GridSync<V> bar;
  __device__ bool init(const gsrb::GridBarrier& g, gsrb::BarrierShared* s) { return bar.init(g, s); }
  __device__ bool sync() { return bar.sync(); }
  __device__ void finish() { bar.finish(); }
};
template <>
struct MaybeSync<kNoBarrier> {
  __device__ bool init(const gsrb::GridBarrier&, gsrb::BarrierShared*) { return true; }
  __device__ bool sync() { return true; }
  __device__ void finish() {}
};

// Fixed-count loop: every CTA calls sync() `episodes` times whatever happens,
// so hardware cluster barriers always see matching arrivals.
template <int V>
__global__ void __launch_bounds__(256, 8)
barrier_bench_kernel(gsrb::GridBarrier gb, int episodes, int fma, float a, float b,
                     float* __restrict__ sink, uint32_t* __restrict__ episode_count) {
  __shared__ gsrb::BarrierShared bsh;
  MaybeSync<V> bar;
  const bool ok0 = bar.init(gb, &bsh);
  // the per-thread FMA state is the kernel's input (sink[] holds the seeds)
  float x = sink[blockIdx.x * blockDim.x + threadIdx.x];
  uint32_t done = 0;
  for (int e = 0; e < episodes; ++e) {
#pragma unroll 1
    for (int f = 0; f < fma; ++f) x = fmaf(x, a, b);
    if (bar.sync() && ok0) ++done;
  }
  sink[blockIdx.x * blockDim.x + threadIdx.x] = x;
  if (threadIdx.x == 0) atomicAdd(episode_count, done);
  bar.finish();
}

// Litmus: message passing through the barrier.  Episode e: every thread stores
// stamp(e) into its own word; barrier; reads the word of the same thread in CTA
// (b + 1 + e) % grid and counts values that are not stamp(e); barrier (so that
// the next stores cannot overtake these reads).
template <int V>
__global__ void __launch_bounds__(256, 8)
barrier_litmus_kernel(gsrb::GridBarrier gb, int episodes, uint32_t* buf, unsigned long long* stale) {
  __shared__ gsrb::BarrierShared bsh;
  gsrb::GridSync<V> bar;
  bar.init(gb, &bsh);
  const uint32_t G = gridDim.x, T = blockDim.x;
  uint32_t bad = 0;
  for (int e = 0; e < episodes; ++e) {
    const uint32_t stamp = 0x9e3779b9u * (uint32_t)(e + 1);
    gsrb::ptx::st_relaxed_gpu(&buf[blockIdx.x * T + threadIdx.x], stamp);
    bar.sync();
    const uint32_t peer = (blockIdx.x + 1u + (uint32_t)e) % G;
    if (gsrb::ptx::ld_relaxed_gpu(&buf[peer * T + threadIdx.x]) != stamp) ++bad;
    bar.sync();
  }
  if (bad) atomicAdd(stale, (unsigned long long)bad);
  bar.finish();
}

struct BenchFn {
  template <int V>
  static const void* get() { return (const void*)barrier_bench_kernel<V>; }
};

const void* bench_fn(int variant) {
  switch (variant) {
    case gsrb::V_CLUSTER: return (const void*)barrier_bench_kernel<gsrb::V_CLUSTER>;
    case gsrb::V_CLUSTER_ALLPOLL: return (const void*)barrier_bench_kernel<gsrb::V_CLUSTER_ALLPOLL>;
    case gsrb::V_DSMEM: return (const void*)barrier_bench_kernel<gsrb::V_DSMEM>;
    case gsrb::V_SOFT2: return (const void*)barrier_bench_kernel<gsrb::V_SOFT2>;
    case gsrb::V_FLAT: return (const void*)barrier_bench_kernel<gsrb::V_FLAT>;
    case gsrb::V_TREE: return (const void*)barrier_bench_kernel<gsrb::V_TREE>;
    case gsrb::V_CCG: return (const void*)barrier_bench_kernel<gsrb::V_CCG>;
    case gsrb::V_CLUSTER_RED: return (const void*)barrier_bench_kernel<gsrb::V_CLUSTER_RED>;
    case gsrb::V_FLIP: return (const void*)barrier_bench_kernel<gsrb::V_FLIP>;
    case gsrb::V_FANOUT: return (const void*)barrier_bench_kernel<gsrb::V_FANOUT>;
    case gsrb::V_CLUSTER_FANOUT: return (const void*)barrier_bench_kernel<gsrb::V_CLUSTER_FANOUT>;
    case gsrb::V_HIER: return (const void*)barrier_bench_kernel<gsrb::V_HIER>;
    case gsrb::V_LOCKFREE: return (const void*)barrier_bench_kernel<gsrb::V_LOCKFREE>;
    case kNoBarrier: return (const void*)barrier_bench_kernel<kNoBarrier>;
    default: return nullptr;
  }
}

const void* litmus_fn(int variant) {
  switch (variant) {
    case gsrb::V_CLUSTER: return (const void*)barrier_litmus_kernel<gsrb::V_CLUSTER>;
    case gsrb::V_CLUSTER_ALLPOLL: return (const void*)barrier_litmus_kernel<gsrb::V_CLUSTER_ALLPOLL>;
    case gsrb::V_DSMEM: return (const void*)barrier_litmus_kernel<gsrb::V_DSMEM>;
    case gsrb::V_SOFT2: return (const void*)barrier_litmus_kernel<gsrb::V_SOFT2>;
    case gsrb::V_FLAT: return (const void*)barrier_litmus_kernel<gsrb::V_FLAT>;
    case gsrb::V_TREE: return (const void*)barrier_litmus_kernel<gsrb::V_TREE>;
    case gsrb::V_CCG: return (const void*)barrier_litmus_kernel<gsrb::V_CCG>;
    case gsrb::V_CLUSTER_RED: return (const void*)barrier_litmus_kernel<gsrb::V_CLUSTER_RED>;
    case gsrb::V_FLIP: return (const void*)barrier_litmus_kernel<gsrb::V_FLIP>;
    case gsrb::V_FANOUT: return (const void*)barrier_litmus_kernel<gsrb::V_FANOUT>;
    case gsrb::V_CLUSTER_FANOUT: return (const void*)barrier_litmus_kernel<gsrb::V_CLUSTER_FANOUT>;
    case gsrb::V_HIER: return (const void*)barrier_litmus_kernel<gsrb::V_HIER>;
    case gsrb::V_LOCKFREE: return (const void*)barrier_litmus_kernel<gsrb::V_LOCKFREE>;
    default: return nullptr;
  }
}


// L2 atomic probes used as the denominator of the barrier roofline.
// mode 0: every CTA's thread 0 issues `iters` red.relaxed.gpu.add to ONE
//         address (same-address reduction throughput at the L2);
// mode 1: a single thread issues `iters` dependent atom.acq_rel.gpu.add
//         (round-trip latency of a same-address atomic).
__global__ void l2_atomic_probe_kernel(uint32_t* addr, int iters, int mode) {
  if (threadIdx.x != 0) return;
  if (mode == 0) {
    for (int i = 0; i < iters; ++i) gsrb::ptx::red_add_relaxed_gpu(addr, 1u);
  } else if (blockIdx.x == 0) {
    // each address depends on the previous result (mode - 1 == 0 at run time)
    const uint32_t dep = (uint32_t)(mode - 1);
    uint32_t* p = addr;
    uint32_t v = 0;
    for (int i = 0; i < iters; ++i) {
      const uint32_t old = gsrb::ptx::atom_add_acq_rel_gpu(p, 1u);
      p = addr + (old & dep);
      v += old;
    }
    if (v == 0xdeadbeefu) addr[1] = v;
  }
}

}  // namespace

// Shared by the data kernels (reduce.cu, scan.cu, graph.cu) for sizing.
const void* gsrb_bench_kernel_for(int variant) { return bench_fn(variant); }

extern "C" {

gsrb_status_t gsrb_barrier_bench(gsrb_ctx_t ctx, const gsrb_cfg_t* cfgin, int32_t episodes,
                                 int32_t fma, float* d_sink, uint32_t* d_count) {
  if (!ctx || episodes < 0 || fma < 0 || !d_sink || !d_count) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  gsrb_cfg_t c = resolve_cfg(ctx, cfgin);
  if (c.threads > 256 || c.threads % 32) return GSRB_ERR_ARG;
  const void* fn = bench_fn(c.variant);
  if (!fn) return GSRB_ERR_ARG;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster) return GSRB_ERR_ARG;
  gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)grid, 0, 0);
  float a = 0.999999f, b = 1e-7f;
  void* args[] = {&gb, &episodes, &fma, &a, &b, &d_sink, &d_count};
  return launch_persistent(ctx, fn, grid, c.threads, 0, c.cluster, coop_of(c), args);
}

gsrb_status_t gsrb_barrier_litmus(gsrb_ctx_t ctx, const gsrb_cfg_t* cfgin, int32_t episodes,
                                  uint32_t* d_buf, unsigned long long* d_stale) {
  if (!ctx || episodes < 0 || !d_buf || !d_stale) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  gsrb_cfg_t c = resolve_cfg(ctx, cfgin);
  if (c.threads > 256 || c.threads % 32) return GSRB_ERR_ARG;
  const void* fn = litmus_fn(c.variant);
  if (!fn) return GSRB_ERR_ARG;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster) return GSRB_ERR_ARG;
  gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)grid, 0, 0);
  void* args[] = {&gb, &episodes, &d_buf, &d_stale};
  return launch_persistent(ctx, fn, grid, c.threads, 0, c.cluster, coop_of(c), args);
}

gsrb_status_t gsrb_barrier_fault_short_grid(gsrb_ctx_t ctx, const gsrb_cfg_t* cfgin) {
  if (!ctx) return GSRB_ERR_ARG;
  gsrb_cfg_t c = resolve_cfg(ctx, cfgin);
  if (c.variant == gsrb::V_CCG || c.variant == gsrb::V_CLUSTER_ALLPOLL || c.variant == gsrb::V_CLUSTER_FANOUT)
    return GSRB_ERR_UNSUPPORTED;
  if (c.threads > 256 || c.threads % 32) return GSRB_ERR_ARG;
  const void* fn = bench_fn(c.variant);
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster) return GSRB_ERR_ARG;
  float* sink = nullptr;
  uint32_t* cnt = nullptr;
  GSRB_CUDA(cudaMalloc(&sink, sizeof(float) * (size_t)grid * c.threads));
  GSRB_CUDA(cudaMalloc(&cnt, sizeof(uint32_t)));
  GSRB_CUDA(cudaMemsetAsync(cnt, 0, sizeof(uint32_t), ctx->stream));
  gsrb_status_t st;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    // One participant (one cluster for the cluster variants) more than launched:
    // the first barrier can never complete, so every wait must run out.
    gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)(grid + c.cluster), 0, 0);
    int episodes = 4, fma = 0;
    float a = 1.f, b = 0.f;
    void* args[] = {&gb, &episodes, &fma, &a, &b, &sink, &cnt};
    st = launch_persistent(ctx, fn, grid, c.threads, 0, c.cluster, false, args);
  }
  gsrb_status_t st2 = gsrb_ctx_status(ctx, nullptr, nullptr, nullptr);
  cudaFree(sink);
  cudaFree(cnt);
  if (st) return st;
  return st2;
}

gsrb_status_t gsrb_probe_l2_atomics(gsrb_ctx_t ctx, int32_t ctas, int32_t iters, int32_t mode, float* ms) {
  if (!ctx || ctas <= 0 || iters <= 0 || !ms || (mode != 0 && mode != 1)) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  uint32_t* addr = nullptr;
  void* s = nullptr;
  gsrb_status_t st = scratch(ctx, 256, &s);
  if (st) return st;
  addr = (uint32_t*)s;
  GSRB_CUDA(cudaMemsetAsync(addr, 0, 256, ctx->stream));
  cudaEvent_t a, b;
  GSRB_CUDA(cudaEventCreate(&a));
  GSRB_CUDA(cudaEventCreate(&b));
  void* args[] = {&addr, &iters, &mode};
  GSRB_CUDA(cudaEventRecord(a, ctx->stream));
  st = launch_plain(ctx, (const void*)l2_atomic_probe_kernel, dim3(mode == 0 ? ctas : 1), dim3(32), 0, args);
  GSRB_CUDA(cudaEventRecord(b, ctx->stream));
  GSRB_CUDA(cudaEventSynchronize(b));
  GSRB_CUDA(cudaEventElapsedTime(ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return st;
}

gsrb_status_t gsrb_max_coresident(gsrb_ctx_t ctx, const gsrb_cfg_t* cfgin, int32_t family, int32_t* ctas);

}  // extern "C"
