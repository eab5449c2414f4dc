// Persistent barrier-stepped sum reduction of int32 into int64.
//
// Reference: reduce_kernel / reduce() in Reduce/reduce_gsrb.cu:289-404 (API
// Reduce/reduce.cuh:47): one element per thread, grid = ceil(N / tpb) CTAs (so
// N is limited to the co-resident thread count, 148*2048 on B200), a
// shared-memory tree per level and one grid barrier per level, int accumulation.
//
// Here: a fixed co-resident grid (default 148 SMs x 2 CTAs x 256 threads) where
// each CTA streams a contiguous chunk with 128-bit non-allocating loads and
// eight independent loads in flight per thread, accumulates in int64, reduces
// with warp shuffles, publishes one partial per CTA, crosses ONE grid barrier,
// and CTA 0 combines the partials in a fixed order (so the result is
// deterministic and bit-exact against a serial int64 sum).
#include "internal.h"

using namespace gsrbrt;

namespace {

__device__ __forceinline__ int4 ld_stream_v4(const int4* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::256B.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

__device__ __forceinline__ long long warp_sum_i64(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; result valid in thread 0.
__device__ __forceinline__ long long block_sum_i64(long long v, long long* warp_buf) {
  v = warp_sum_i64(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_buf[w] = v;
  __syncthreads();
  long long t = 0;
  if (w == 0) {
    t = (lane < (int)(blockDim.x >> 5)) ? warp_buf[lane] : 0;
    t = warp_sum_i64(t);
  }
  return t;
}

// Sum of in[beg, end) by one CTA (every thread returns its share).
__device__ __forceinline__ long long chunk_sum(const int32_t* __restrict__ in, uint64_t beg, uint64_t end) {
  long long acc = 0;
  const int32_t* p = in + beg;
  uint64_t len = end - beg;
  // scalar head until 16-byte alignment
  uint64_t head = ((16u - ((uintptr_t)p & 15u)) & 15u) >> 2;
  if (head > len) head = len;
  if (threadIdx.x < head) acc += p[threadIdx.x];
  p += head;
  len -= head;
  const int4* v = reinterpret_cast<const int4*>(p);
  const uint64_t nv = len >> 2;
  const uint64_t T = blockDim.x;
  uint64_t i = threadIdx.x;
  for (; i + 7 * T < nv; i += 8 * T) {
    int4 x[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) x[u] = ld_stream_v4(v + i + u * T);
#pragma unroll
    for (int u = 0; u < 8; ++u)
      acc += (long long)x[u].x + (long long)x[u].y + (long long)x[u].z + (long long)x[u].w;
  }
  for (; i < nv; i += T) {
    const int4 x = ld_stream_v4(v + i);
    acc += (long long)x.x + (long long)x.y + (long long)x.z + (long long)x.w;
  }
  const uint64_t tail = len & 3u;
  if (threadIdx.x < tail) acc += p[(nv << 2) + threadIdx.x];
  return acc;
}

template <int V>
__global__ void __launch_bounds__(1024)
reduce_i32_kernel(gsrb::GridBarrier gb, const int32_t* __restrict__ in, uint64_t n,
                  long long* __restrict__ partials, long long* __restrict__ out) {
  __shared__ gsrb::BarrierShared bsh;
  __shared__ long long warp_buf[32];
  gsrb::GridSync<V> bar;
  const bool ok0 = bar.init(gb, &bsh);
  const uint64_t G = gridDim.x;
  uint64_t chunk = (n + G - 1) / G;
  chunk = (chunk + 3) & ~3ull;  // keeps every chunk start 16-byte aligned
  const uint64_t beg = min(n, (uint64_t)blockIdx.x * chunk);
  const uint64_t end = min(n, beg + chunk);
  long long acc = ok0 ? chunk_sum(in, beg, end) : 0;
  const long long bsum = block_sum_i64(acc, warp_buf);
  if (threadIdx.x == 0) partials[blockIdx.x] = bsum;
  const bool ok = bar.sync() && ok0;
  if (ok && blockIdx.x == 0) {
    // fixed-order combine of the G partials (deterministic)
    long long s = 0;
    for (uint64_t j = threadIdx.x; j < G; j += blockDim.x) s += partials[j];
    __syncthreads();
    s = block_sum_i64(s, warp_buf);
    if (threadIdx.x == 0) *out = s;
  }
  bar.finish();
}

const void* reduce_fn(int variant) {
  switch (variant) {
    case gsrb::V_CLUSTER: return (const void*)reduce_i32_kernel<gsrb::V_CLUSTER>;
    case gsrb::V_DSMEM: return (const void*)reduce_i32_kernel<gsrb::V_DSMEM>;
    case gsrb::V_SOFT2: return (const void*)reduce_i32_kernel<gsrb::V_SOFT2>;
    case gsrb::V_FLAT: return (const void*)reduce_i32_kernel<gsrb::V_FLAT>;
    case gsrb::V_TREE: return (const void*)reduce_i32_kernel<gsrb::V_TREE>;
    case gsrb::V_CCG: return (const void*)reduce_i32_kernel<gsrb::V_CCG>;
    case gsrb::V_CLUSTER_RED: return (const void*)reduce_i32_kernel<gsrb::V_CLUSTER_RED>;
    case gsrb::V_FLIP: return (const void*)reduce_i32_kernel<gsrb::V_FLIP>;
    case gsrb::V_FANOUT: return (const void*)reduce_i32_kernel<gsrb::V_FANOUT>;
    case gsrb::V_HIER: return (const void*)reduce_i32_kernel<gsrb::V_HIER>;
    default: return nullptr;  // V_CLUSTER_ALLPOLL is kept to fixed-count loops
  }
}

}  // namespace

const void* gsrb_reduce_kernel_for(int variant) { return reduce_fn(variant); }

extern "C" gsrb_status_t gsrb_reduce_i32(gsrb_ctx_t ctx, const int32_t* d_in, size_t n, int64_t* d_out,
                                         const gsrb_cfg_t* cfgin) {
  if (!ctx || !d_out || (n && !d_in)) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  gsrb_cfg_t c = resolve_cfg(ctx, cfgin);
  if (c.threads % 32 || c.threads > 1024) return GSRB_ERR_ARG;
  const void* fn = reduce_fn(c.variant);
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster) return GSRB_ERR_ARG;
  void* part = nullptr;
  gsrb_status_t st = scratch(ctx, sizeof(long long) * (size_t)grid, &part);
  if (st) return st;
  gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)grid, 0, 0);
  uint64_t n64 = n;
  long long* partials = (long long*)part;
  long long* out = (long long*)d_out;
  void* args[] = {&gb, &d_in, &n64, &partials, &out};
  return launch_persistent(ctx, fn, grid, c.threads, 0, c.cluster, coop_of(c), args);
}
