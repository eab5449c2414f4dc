// Allocation-free variant of the persistent int32 -> int64 reduce.
//
// Who needs it: callers that may not allocate device memory at all -- code
// running under a fixed memory budget handed out by a host framework, a plugin
// that must not grow the process's device footprint, or a path that must not
// call cudaMalloc (which can synchronize the device).  Such callers cannot
// create a gsrb context (the context allocates its barrier state and scratch),
// so this entry point needs nothing but the caller's input, output and stream.
//
// How: the kernel's scratch -- the grid barrier state and one partial sum per
// CTA -- lives in one file-scope `static __device__` array of fixed size
// (kNoAllocBytes below), which every GPU that loads the library holds until
// the process exits.  Host code cannot use the array's name as a device
// address (it names a host-side stand-in), so the address is obtained with
// cudaGetSymbolAddress, once per device, on the first call on that device with
// that device current; that first call should come before any stream capture.
//
// The array is shared by every call and keeps the last call's contents: each
// call clears the barrier words (cudaMemsetAsync, which allocates nothing)
// before its launch, and calls whose kernels overlap on the GPU race on it.
#include "internal.h"

namespace {

constexpr int kNoAllocMaxCtas = 2048;                 // grid limit (partials held)
constexpr size_t kNoAllocBarrierBytes = 1024;         // BarrierSlot (512 B) + flip line
constexpr size_t kNoAllocBytes = kNoAllocBarrierBytes + sizeof(long long) * kNoAllocMaxCtas;  // 17 KiB
constexpr uint64_t kNoAllocMaxElems = 1ull << 32;     // int64 sums of int32 cannot overflow below this
constexpr int kNoAllocThreads = 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

__device__ __forceinline__ int4 noalloc_ld_v4(const int4* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

__device__ __forceinline__ long long noalloc_warp_sum(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ long long noalloc_block_sum(long long v, long long* warp_buf) {
  v = noalloc_warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) warp_buf[w] = v;
  __syncthreads();
  long long t = 0;
  if (w == 0) {
    t = (lane < (int)(blockDim.x >> 5)) ? warp_buf[lane] : 0;
    t = noalloc_warp_sum(t);
  }
  __syncthreads();
  return t;
}

// Same computation as the context-based reduce: contiguous chunk per CTA,
// 128-bit loads, int64 accumulation, one grid barrier (the two-level
// sum-to-flip barrier), fixed-order combine by CTA 0.
__global__ void __launch_bounds__(kNoAllocThreads)
reduce_i32_noalloc_kernel(gsrb::GridBarrier gb, const int32_t* __restrict__ in, uint64_t n,
                          long long* __restrict__ out) {
  __shared__ gsrb::BarrierShared bsh;
  __shared__ long long warp_buf[32];
  long long* partials = reinterpret_cast<long long*>(g_noalloc_scratch + kNoAllocBarrierBytes);
  gsrb::GridSync<gsrb::V_FLIP> bar;
  const bool ok0 = bar.init(gb, &bsh);
  const uint64_t G = gridDim.x;
  uint64_t chunk = (n + G - 1) / G;
  chunk = (chunk + 3) & ~3ull;
  const uint64_t beg = min(n, (uint64_t)blockIdx.x * chunk);
  const uint64_t end = min(n, beg + chunk);
  long long acc = 0;
  if (ok0) {
    const int32_t* p = in + beg;
    uint64_t len = end - beg;
    uint64_t head = ((16u - ((uintptr_t)p & 15u)) & 15u) >> 2;
    if (head > len) head = len;
    if (threadIdx.x < head) acc += p[threadIdx.x];
    p += head;
    len -= head;
    const int4* v = reinterpret_cast<const int4*>(p);
    const uint64_t nv = len >> 2;
    for (uint64_t i = threadIdx.x; i < nv; i += blockDim.x) {
      const int4 x = noalloc_ld_v4(v + i);
      acc += (long long)x.x + (long long)x.y + (long long)x.z + (long long)x.w;
    }
    if (threadIdx.x < (len & 3u)) acc += p[(nv << 2) + threadIdx.x];
  }
  const long long bsum = noalloc_block_sum(acc, warp_buf);
  if (threadIdx.x == 0) partials[blockIdx.x] = bsum;
  const bool ok = bar.sync() && ok0;
  if (ok && blockIdx.x == 0) {
    long long s = 0;
    for (uint64_t j = threadIdx.x; j < G; j += blockDim.x) s += __ldcg(partials + j);
    s = noalloc_block_sum(s, warp_buf);
    if (threadIdx.x == 0) *out = s;
  }
  bar.finish();
}

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {};  // device address of the array, per device ordinal

}  // namespace

extern "C" gsrb_status_t gsrb_reduce_i32_noalloc(const int32_t* d_in, size_t n, int64_t* d_out, void* stream) {
  if (!d_out || (n && !d_in)) return GSRB_ERR_ARG;
  if ((uint64_t)n > kNoAllocMaxElems) {
    fprintf(stderr, "[gsrb] gsrb_reduce_i32_noalloc: n = %zu exceeds the maximum of %llu elements\n", n,
            (unsigned long long)kNoAllocMaxElems);
    return GSRB_ERR_ARG;
  }
  int dev = 0;
  GSRB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return GSRB_ERR_UNSUPPORTED;
  void* base = nullptr;
  {
    // once per device, with that device current (the array's name is only a
    // host-side stand-in; the kernel needs the device address)
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) GSRB_CUDA(cudaGetSymbolAddress(&g_noalloc_ptr[dev], g_noalloc_scratch));
    base = g_noalloc_ptr[dev];
  }
  int sms = 0, per_sm = 0;
  GSRB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  GSRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, reduce_i32_noalloc_kernel,
                                                          kNoAllocThreads, 0));
  int grid = 2 * sms;
  if (grid > kNoAllocMaxCtas) grid = kNoAllocMaxCtas;
  if (grid > per_sm * sms) return GSRB_ERR_NOT_CORESIDENT;
  cudaStream_t s = (cudaStream_t)stream;
  // the barrier words must start at zero; the partials are overwritten
  GSRB_CUDA(cudaMemsetAsync(base, 0, kNoAllocBarrierBytes, s));
  gsrb::GridBarrier gb;
  gb.slot = reinterpret_cast<gsrb::BarrierSlot*>(base);
  gb.groups = nullptr;
  gb.nparticipants = (uint32_t)grid;
  gb.first_cta = 0;
  gb.ngroups = 0;
  gb.spin_ns = 0;
  gb.timeout_ns = 2000000000ull;
  gb.flip = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(base) + sizeof(gsrb::BarrierSlot));
  gb.nflip = 1;
  gb._pad = 0;
  uint64_t n64 = n;
  long long* out = reinterpret_cast<long long*>(d_out);
  void* args[] = {&gb, (void*)&d_in, &n64, &out};
  cudaError_t e = cudaLaunchKernel((const void*)reduce_i32_noalloc_kernel, dim3(grid), dim3(kNoAllocThreads), args,
                                   0, s);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return gsrbrt::cuda_err(e, "reduce_i32_noalloc launch");
  }
  gsrbrt::g_launches.fetch_add(1, std::memory_order_relaxed);
  // synchronous: read the barrier's status word of this call
  uint32_t status = 0;
  GSRB_CUDA(cudaMemcpyAsync(&status, &reinterpret_cast<gsrb::BarrierSlot*>(base)->status, sizeof(status),
                            cudaMemcpyDeviceToHost, s));
  GSRB_CUDA(cudaStreamSynchronize(s));
  return gsrbrt::map_dev(status);
}
