// Persistent barrier-stepped sum reduction of int32 into int64.
//
// Reference: reduce_kernel / reduce() in Reduce/reduce_gsrb.cu:289-404 (API
// Reduce/reduce.cuh:19): one element per thread, grid = ceil(N / tpb) CTAs (so
// N is limited to the co-resident thread count, 148*2048 on B200), a
// shared-memory tree per level and one grid barrier per level, int accumulation.
//
// Here: a fixed co-resident grid (default one 1024-thread CTA per SM).  Each
// CTA streams a contiguous chunk through a ring of 32 KiB shared-memory stages
// filled by bulk copies (cp.async.bulk global->shared, completion counted on a
// "full" mbarrier per stage; no multicast).  Thread 0 keeps up to `nbuf`
// stages in flight (192 KiB per SM by default, well above the bytes in flight
// an SM needs to stream its share of HBM bandwidth); every warp sums its part
// of a stage in int64 and frees the stage on an "empty" mbarrier, so warps
// never wait for each other inside the stream.  Warp shuffles reduce the
// CTA's sum to one partial; the CTA arrives at the grid barrier (split phase:
// with the fan-out protocols the CTA whose arrival completes the barrier
// combines and nobody waits; otherwise only CTA 0 waits) and the combiner adds
// the partials in CTA order, so the result is deterministic and bit-exact
// against a serial int64 sum.
#include "internal.h"

using namespace gsrbrt;

namespace {

constexpr uint32_t kStageBytes = 32768;
constexpr uint32_t kMaxStages = 7;
constexpr uint32_t kDefaultStages = 6;

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

// Bounded wait on an mbarrier phase.  On expiry records a timeout and keeps
// waiting once more (bounded) so that no copy is in flight when the CTA leaves.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* mbar, uint32_t parity, const gsrb::GridBarrier& gb) {
  uint64_t t0 = 0;
  bool ok = true;
  for (uint32_t it = 0;; ++it) {
    if (gsrb::ptx::mbar_try_wait(mbar, parity)) return ok;
    if ((it & 63u) == 63u) {
      const uint64_t now = gsrb::ptx::globaltimer_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > gb.timeout_ns) {
        if (!ok) return false;  // second deadline: give up
        gsrb::detail::record_error(gb, gsrb::GSRB_DEV_TIMEOUT, 0xfffffff1u);
        ok = false;
        t0 = now;
      }
    }
  }
}

template <int V>
__global__ void __launch_bounds__(1024)
reduce_i32_kernel(gsrb::GridBarrier gb, const int32_t* __restrict__ in, uint64_t n,
                  long long* __restrict__ partials, long long* __restrict__ out, uint32_t nbuf, uint32_t pdl) {
  extern __shared__ __align__(128) unsigned char stage[];
  __shared__ gsrb::BarrierShared bsh;
  __shared__ long long warp_buf[32];
  __shared__ uint64_t full[kMaxStages], empty[kMaxStages];
  gsrb::GridSync<V> bar;
  const uint32_t tid = threadIdx.x, T = blockDim.x, lane = tid & 31u, nwarps = T >> 5;
  const uint64_t G = gridDim.x;
  uint64_t chunk = (n + G - 1) / G;
  chunk = (chunk + 3) & ~3ull;
  const uint64_t beg = min(n, (uint64_t)blockIdx.x * chunk);
  const uint64_t end = min(n, beg + chunk);
  const int32_t* p = in + beg;
  uint64_t len = end - beg;
  long long acc = 0;
  // scalar head up to 16-byte alignment, scalar tail past the last 16 bytes
  uint64_t head = ((16u - ((uintptr_t)p & 15u)) & 15u) >> 2;
  if (head > len) head = len;
  if (tid < head) acc += p[tid];
  p += head;
  len -= head;
  const uint64_t nbytes = (len * 4u) & ~15ull;
  const uint64_t tail = len - (nbytes >> 2);
  if (tid < tail) acc += p[(nbytes >> 2) + tid];
  const uint32_t nst = (uint32_t)((nbytes + kStageBytes - 1) / kStageBytes);
  const unsigned char* src = reinterpret_cast<const unsigned char*>(p);

  auto bytes_of = [&](uint32_t k) {
    return (uint32_t)min((uint64_t)kStageBytes, nbytes - (uint64_t)k * kStageBytes);
  };
  auto issue = [&](uint32_t k) {
    const uint32_t buf = k % nbuf;
    gsrb::ptx::mbar_arrive_expect_tx(&full[buf], bytes_of(k));
    gsrb::ptx::bulk_g2s(stage + (size_t)buf * kStageBytes, src + (size_t)k * kStageBytes, bytes_of(k), &full[buf]);
  };
  // Chained launches (pdl): the next reduction on the stream may be scheduled
  // as soon as every CTA of this one runs; its CTAs take the SM slots this
  // grid's CTAs free when they leave, so its stream overlaps this grid's
  // barrier and combine.  It reads only its own input before griddep_wait.
  if (pdl) gsrb::ptx::griddep_launch_dependents();
  // The first copies go out before the barrier's set-up reads (two dependent
  // L2 round trips): they only read the input.  Whatever the set-up decides,
  // every issued copy is waited for below before the CTA leaves.
  uint32_t issued = 0;
  if (tid == 0) {
    for (uint32_t i = 0; i < nbuf; ++i) {
      gsrb::ptx::mbar_init(&full[i], 1);
      gsrb::ptx::mbar_init(&empty[i], nwarps);
    }
    gsrb::ptx::fence_mbar_init();
    for (; issued < nst && issued < nbuf; ++issued) issue(issued);
  }
  // Without pdl the barrier set-up comes first (its __syncthreads also
  // publishes the mbarrier set-up).  With pdl it waits until the previous grid
  // on the stream has finished (that grid may still use the barrier state and
  // the partials), so it comes after this CTA's stream.
  bool ok0 = true;
  if (!pdl) ok0 = bar.init(gb, &bsh);
  else __syncthreads();
  bool ok = ok0;
  if (!ok0 && tid == 0) {
    // refused to start (a recorded error): leave no copy in flight
    for (uint32_t k = 0; k < issued; ++k) mbar_wait_bounded(&full[k % nbuf], (k / nbuf) & 1u, gb);
  }
  if (ok0) {
    // No CTA-wide barrier per stage: each warp frees a stage on `empty` when
    // it has read its part; thread 0 refills a stage once every warp has.
    for (uint32_t k = 0; k < nst; ++k) {
      const uint32_t buf = k % nbuf, ph = (k / nbuf) & 1u;
      ok = mbar_wait_bounded(&full[buf], ph, gb) && ok;
      const int4* v = reinterpret_cast<const int4*>(stage + (size_t)buf * kStageBytes);
      const uint32_t nv = bytes_of(k) >> 4;
      for (uint32_t i = tid; i < nv; i += T) {
        const int4 x = v[i];
        acc += (long long)x.x + (long long)x.y + (long long)x.z + (long long)x.w;
      }
      __syncwarp();
      if (lane == 0) gsrb::ptx::mbar_arrive(&empty[buf]);
      if (tid == 0 && k + nbuf < nst) {
        ok = mbar_wait_bounded(&empty[buf], ph, gb) && ok;
        issue(k + nbuf);
      }
    }
  }
  if (pdl) {
    gsrb::ptx::griddep_wait();
    ok = bar.init(gb, &bsh) && ok;
  }
  const long long bsum = block_sum_i64(acc, warp_buf);
  if (tid == 0) partials[blockIdx.x] = bsum;
  bar.arrive();
  // the combiner: the CTA whose arrival completed the barrier when the protocol
  // says so (it has acquired every partial; nobody waits), else CTA 0 after a wait
  __shared__ uint32_t s_comb;
  bool done = true, combiner;
  if (gsrb::GridSync<V>::kCompleter) {
    if (tid == 0) s_comb = bar.arrived_done;
    __syncthreads();
    combiner = s_comb != 0u;
  } else {
    combiner = blockIdx.x == 0;
    if (!gsrb::GridSync<V>::kSplit || combiner) done = bar.wait();
  }
  if (done && ok && combiner) {
    // fixed-order combine of the G partials (deterministic)
    long long s = 0;
    for (uint64_t j = tid; j < G; j += T) s += __ldcg(partials + j);
    __syncthreads();
    s = block_sum_i64(s, warp_buf);
    if (tid == 0) *out = s;
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

// Dynamic shared memory of a reduce launch: cfg->tile stages of 32 KiB; 0 =
// as many as fit 200 KiB per SM over cfg->ctas_per_sm CTAs (at most 6, at least 1).
size_t gsrb_reduce_smem_for(const gsrb_cfg_t& c) {
  uint32_t nb = (uint32_t)c.tile;
  if (c.tile <= 0) {
    const uint32_t k = c.ctas_per_sm > 0 ? (uint32_t)c.ctas_per_sm : 1u;
    nb = (200u * 1024u / k) / kStageBytes;
    if (nb > kDefaultStages) nb = kDefaultStages;
  }
  if (nb < 1) nb = 1;
  if (nb > kMaxStages) nb = kMaxStages;
  return (size_t)nb * kStageBytes;
}

extern "C" gsrb_status_t gsrb_reduce_i32(gsrb_ctx_t ctx, const int32_t* d_in, size_t n, int64_t* d_out,
                                         const gsrb_cfg_t* cfgin) {
  if (!ctx || !d_out || (n && !d_in)) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  gsrb_cfg_t c = resolve_cfg(ctx, cfgin);
  if (!cfgin) {
    // default shape: one 1024-thread CTA per SM, 8 stages (128 KiB) in flight
    c.ctas_per_sm = 1;
    c.threads = 1024;
  }
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
  const size_t smem = gsrb_reduce_smem_for(c);
  uint32_t nbuf = (uint32_t)(smem / kStageBytes);
  // chained launch: plain launches only (a cooperative launch is refused)
  const bool pdl = c.overlap != 0 && coop_of(c) == 0;
  if (c.overlap != 0 && !pdl) return GSRB_ERR_UNSUPPORTED;
  uint32_t pdl32 = pdl ? 1u : 0u;
  void* args[] = {&gb, &d_in, &n64, &partials, &out, &nbuf, &pdl32};
  return launch_persistent(ctx, fn, grid, c.threads, smem, c.cluster, coop_of(c), args, pdl);
}
