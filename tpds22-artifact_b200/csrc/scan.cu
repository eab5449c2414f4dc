// Persistent barrier-stepped exclusive scan (uint32 with wraparound, and FP32
// with FP64 offsets).
//
// Reference: gpu_prescan + sum_scan_blelloch in scan/scan_gsrb.cu:486-804
// (API scan/scan.h:16-18): 64-element Blelloch tiles (32 threads), a grid
// barrier per recursion level, two fix-up launches (gpu_add_block_sums,
// :440-482, :798-799), grid = ceil(N / 64) CTAs that must all be co-resident
// (N <= 148*32*64 on B200).
//
// Here: a fixed co-resident grid (default one 1024-thread CTA per SM).  The
// input is cut into segments of G tiles (one tile per CTA).  Per segment a CTA
//   1. has its tile in shared memory (moved by cp.async.bulk, prefetched one
//      segment ahead into a second buffer, so HBM keeps streaming while the CTA
//      waits at the barrier),
//   2. reduces it (warp shuffles) and publishes one partial,
//   3. crosses ONE grid barrier,
//   4. reads the G partials of the segment: its offset is the running carry
//      plus the partials of the CTAs before it (every CTA computes the same
//      carry, so the reference's separate "scan of block sums" pass and its
//      second barrier are not needed),
//   5. rescans the tile in place from shared memory and writes it back with a
//      bulk store.
// Every element is read from HBM once and written once (8N bytes).  Partials
// are double-buffered by segment parity: a CTA can only write the buffer of
// segment s+2 after the barrier of s+1, which every CTA reaches only after it
// has read the partials of segment s.
#include "internal.h"

using namespace gsrbrt;

namespace {

template <bool F32>
struct ScanT;
template <>
struct ScanT<false> {
  using Elem = uint32_t;
  using Acc = uint32_t;  // uint32 wraparound, like cpu_sum_scan (scan/main.cu:15-20)
};
template <>
struct ScanT<true> {
  using Elem = float;
  using Acc = double;    // tile offsets and carries in FP64
};

__device__ __forceinline__ uint32_t shfl_up(uint32_t v, int o) { return __shfl_up_sync(0xffffffffu, v, o); }
__device__ __forceinline__ double shfl_up(double v, int o) { return __shfl_up_sync(0xffffffffu, v, o); }
__device__ __forceinline__ uint32_t shfl_idx(uint32_t v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ double shfl_idx(double v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ uint32_t shfl_down(uint32_t v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }
__device__ __forceinline__ double shfl_down(double v, int o) { return __shfl_down_sync(0xffffffffu, v, o); }

__device__ __forceinline__ uint64_t acc_bits(uint32_t a) { return a; }
__device__ __forceinline__ uint64_t acc_bits(double a) { return (uint64_t)__double_as_longlong(a); }
__device__ __forceinline__ void acc_from(uint64_t b, uint32_t& a) { a = (uint32_t)b; }
__device__ __forceinline__ void acc_from(uint64_t b, double& a) { a = __longlong_as_double((long long)b); }

template <typename Acc>
__device__ __forceinline__ Acc warp_sum(Acc v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += shfl_down(v, o);
  return v;
}

// Sum of the 4 lanes of a vector, as the accumulation type.
__device__ __forceinline__ uint32_t vsum(uint4 v) { return v.x + v.y + v.z + v.w; }
__device__ __forceinline__ double vsum(float4 v) { return (double)((v.x + v.y) + (v.z + v.w)); }

constexpr uint32_t kChunk = 16384;  // bytes per bulk copy instruction

struct TileGeom {
  uint64_t beg;   // first element of this CTA's tile
  uint32_t cnt;   // valid elements
  uint32_t span;  // tile stride of the segment (multiple of 4)
};

__device__ __forceinline__ TileGeom tile_of(uint64_t s, uint64_t n, uint32_t G, uint32_t tile, uint32_t b) {
  const uint64_t seg = (uint64_t)G * tile;
  const uint64_t base = s * seg;
  const uint64_t rem = n - base;
  TileGeom t;
  if (rem >= seg) {
    t.span = tile;
  } else {
    uint64_t q = (rem + G - 1) / G;
    t.span = (uint32_t)((q + 3) & ~3ull);
  }
  t.beg = base + (uint64_t)b * t.span;
  const uint64_t left = t.beg >= n ? 0ull : n - t.beg;
  t.cnt = (uint32_t)(left < (uint64_t)t.span ? left : (uint64_t)t.span);
  return t;
}

// Bounded wait on an mbarrier phase.  On expiry records a timeout and keeps
// waiting (bounded once more) so that no copy is in flight when the CTA leaves.
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
        gsrb::detail::record_error(gb, gsrb::GSRB_DEV_TIMEOUT, 0xfffffff0u);
        ok = false;
        t0 = now;
      }
    }
  }
}

template <int V, bool F32>
__global__ void __launch_bounds__(1024, 1)
scan_kernel(gsrb::GridBarrier gb, const typename ScanT<F32>::Elem* __restrict__ in,
            typename ScanT<F32>::Elem* __restrict__ out, uint64_t n, uint32_t tile,
            unsigned long long* __restrict__ partials, int in_bulk, int out_bulk) {
  using Elem = typename ScanT<F32>::Elem;
  using Acc = typename ScanT<F32>::Acc;
  using Vec = typename std::conditional<F32, float4, uint4>::type;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ gsrb::BarrierShared bsh;
  __shared__ uint64_t mbar[2];
  __shared__ Acc s_warp[32];
  __shared__ Acc s_red[2][32];
  __shared__ Acc s_bcast[2];

  Elem* buf[2] = {reinterpret_cast<Elem*>(smem), reinterpret_cast<Elem*>(smem + (size_t)tile * sizeof(Elem))};
  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t G = gridDim.x, b = blockIdx.x;

  gsrb::GridSync<V> bar;
  bool ok = bar.init(gb, &bsh);
  if (tid == 0) {
    gsrb::ptx::mbar_init(&mbar[0], 1);
    gsrb::ptx::mbar_init(&mbar[1], 1);
    gsrb::ptx::fence_mbar_init();
  }
  __syncthreads();

  const uint64_t seg = (uint64_t)G * tile;
  const uint64_t nseg = (n + seg - 1) / seg;
  uint32_t phase[2] = {0u, 0u};
  bool pending[2] = {false, false};

  // thread 0: start the bulk load of segment s into buffer `which`
  auto issue = [&](uint64_t s, int which) {
    const TileGeom t = tile_of(s, n, G, tile, b);
    uint32_t bytes = in_bulk ? ((t.cnt * (uint32_t)sizeof(Elem)) & ~15u) : 0u;
    gsrb::ptx::mbar_arrive_expect_tx(&mbar[which], bytes);
    const unsigned char* src = reinterpret_cast<const unsigned char*>(in + t.beg);
    unsigned char* dst = reinterpret_cast<unsigned char*>(buf[which]);
    for (uint32_t off = 0; off < bytes; off += kChunk) {
      const uint32_t sz = min(kChunk, bytes - off);
      gsrb::ptx::bulk_g2s(dst + off, src + off, sz, &mbar[which]);
    }
  };

  if (ok && nseg > 0 && tid == 0) issue(0, 0);
  pending[0] = ok && nseg > 0;
  Acc carry = Acc(0);

  for (uint64_t s = 0; ok && s < nseg; ++s) {
    const int which = (int)(s & 1);
    const TileGeom t = tile_of(s, n, G, tile, b);
    Elem* cur = buf[which];
    // A copy that never lands is recorded in the status word by the wait; the
    // loop is left only on the barrier's verdict, which is the same for every
    // CTA of a cluster (hardware cluster barriers need matching arrivals).
    mbar_wait_bounded(&mbar[which], phase[which], gb);
    phase[which] ^= 1u;
    pending[which] = false;
    // elements the bulk copy did not cover: the ragged end (and everything when
    // the input is not 16-byte aligned), then zeros up to the tile span
    const uint32_t done = in_bulk ? (((t.cnt * (uint32_t)sizeof(Elem)) & ~15u) / (uint32_t)sizeof(Elem)) : 0u;
    for (uint32_t i = done + tid; i < t.cnt; i += blockDim.x) cur[i] = in[t.beg + i];
    for (uint32_t i = t.cnt + tid; i < t.span; i += blockDim.x) cur[i] = Elem(0);
    __syncthreads();

    // prefetch the next segment into the other buffer once its last store has
    // finished reading it
    if (s + 1 < nseg) {
      if (tid == 0) {
        gsrb::ptx::bulk_wait_read_all();
        issue(s + 1, which ^ 1);
      }
      pending[which ^ 1] = true;
    }

    // ---- phase 1: per-warp totals, block total -> partial
    const uint32_t nvec = t.span >> 2;
    const uint32_t vpw = (nvec + nw - 1) / nw;
    const uint32_t v0 = w * vpw, v1 = min(nvec, v0 + vpw);
    const Vec* cv = reinterpret_cast<const Vec*>(cur);
    Acc lsum = Acc(0);
    for (uint32_t v = v0 + lane; v < v1; v += 32) lsum += vsum(cv[v]);
    const Acc wt = warp_sum(lsum);
    if (lane == 0) s_warp[w] = wt;
    __syncthreads();
    if (tid == 0) {
      Acc run = Acc(0);
      for (uint32_t i = 0; i < nw; ++i) {
        const Acc x = s_warp[i];
        s_warp[i] = run;  // exclusive warp offsets within the tile
        run += x;
      }
      __stcg(&partials[(s & 1) * G + b], (unsigned long long)acc_bits(run));
    }

    // ---- the grid barrier of this segment
    ok = bar.sync();
    if (!ok) break;

    // ---- phase 2: offset = carry + sum of the partials of the CTAs before b
    Acc pre = Acc(0), tot = Acc(0);
    for (uint32_t j = tid; j < G; j += blockDim.x) {
      Acc x;
      acc_from(__ldcg(&partials[(s & 1) * G + j]), x);
      tot += x;
      if (j < b) pre += x;
    }
    pre = warp_sum(pre);
    tot = warp_sum(tot);
    if (lane == 0) {
      s_red[0][w] = pre;
      s_red[1][w] = tot;
    }
    __syncthreads();
    if (tid == 0) {
      Acc p = Acc(0), q = Acc(0);
      for (uint32_t i = 0; i < nw; ++i) {
        p += s_red[0][i];
        q += s_red[1][i];
      }
      s_bcast[0] = p;
      s_bcast[1] = q;
    }
    __syncthreads();
    const Acc base = carry + s_bcast[0];
    carry += s_bcast[1];

    // ---- phase 3: rescan the tile in place (exclusive)
    Acc run = base + s_warp[w];
    Vec* wv = reinterpret_cast<Vec*>(cur);
    for (uint32_t r0 = v0; r0 < v1; r0 += 32) {
      const uint32_t v = r0 + lane;
      const bool valid = v < v1;
      Vec x;
      if (valid) x = wv[v];
      else memset(&x, 0, sizeof(x));
      // lane-local inclusive prefix of 4 elements
      const Elem a0 = x.x, a1 = a0 + x.y, a2 = a1 + x.z, a3 = a2 + x.w;
      const Acc lt = Acc(a3);
      Acc incl = lt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const Acc y = shfl_up(incl, o);
        if ((int)lane >= o) incl += y;
      }
      const Acc e0 = run + (incl - lt);
      if (valid) {
        Vec y;
        y.x = Elem(e0);
        y.y = Elem(e0 + Acc(a0));
        y.z = Elem(e0 + Acc(a1));
        y.w = Elem(e0 + Acc(a2));
        wv[v] = y;
      }
      run += shfl_idx(incl, 31);
    }
    gsrb::ptx::fence_proxy_async_smem();
    __syncthreads();

    // ---- write back
    const uint32_t sdone = out_bulk ? (((t.cnt * (uint32_t)sizeof(Elem)) & ~15u) / (uint32_t)sizeof(Elem)) : 0u;
    if (tid == 0 && sdone) {
      unsigned char* dst = reinterpret_cast<unsigned char*>(out + t.beg);
      const unsigned char* src = reinterpret_cast<const unsigned char*>(cur);
      const uint32_t bytes = sdone * (uint32_t)sizeof(Elem);
      for (uint32_t off = 0; off < bytes; off += kChunk) gsrb::ptx::bulk_s2g(dst + off, src + off, min(kChunk, bytes - off));
      gsrb::ptx::bulk_commit();
    }
    for (uint32_t i = sdone + tid; i < t.cnt; i += blockDim.x) out[t.beg + i] = cur[i];
    // the generic stores above must finish reading `cur` before it is refilled
    __syncthreads();
  }

  // leave nothing in flight: a prefetch that was issued but not consumed, and
  // every bulk store
  for (int k = 0; k < 2; ++k)
    if (pending[k]) mbar_wait_bounded(&mbar[k], phase[k], gb);
  if (tid == 0) gsrb::ptx::bulk_wait_all();
  __syncthreads();
  bar.finish();
}

template <bool F32>
const void* scan_fn_t(int variant) {
  switch (variant) {
    case gsrb::V_CLUSTER: return (const void*)scan_kernel<gsrb::V_CLUSTER, F32>;
    case gsrb::V_DSMEM: return (const void*)scan_kernel<gsrb::V_DSMEM, F32>;
    case gsrb::V_SOFT2: return (const void*)scan_kernel<gsrb::V_SOFT2, F32>;
    case gsrb::V_FLAT: return (const void*)scan_kernel<gsrb::V_FLAT, F32>;
    case gsrb::V_TREE: return (const void*)scan_kernel<gsrb::V_TREE, F32>;
    case gsrb::V_CCG: return (const void*)scan_kernel<gsrb::V_CCG, F32>;
    case gsrb::V_CLUSTER_RED: return (const void*)scan_kernel<gsrb::V_CLUSTER_RED, F32>;
    case gsrb::V_FLIP: return (const void*)scan_kernel<gsrb::V_FLIP, F32>;
    case gsrb::V_FANOUT: return (const void*)scan_kernel<gsrb::V_FANOUT, F32>;
    case gsrb::V_HIER: return (const void*)scan_kernel<gsrb::V_HIER, F32>;
    default: return nullptr;
  }
}

constexpr uint32_t kDefaultTile = 24576;  // elements per CTA tile (96 KiB), two buffers per CTA

gsrb_status_t scan_launch(gsrb_ctx_t ctx, const void* d_in, void* d_out, size_t n, const gsrb_cfg_t* cfgin,
                          bool f32) {
  if (!ctx || (n && (!d_in || !d_out))) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  gsrb_cfg_t c;
  if (cfgin) {
    c = resolve_cfg(ctx, cfgin);
  } else {
    c = resolve_cfg(ctx, nullptr);
    c.ctas_per_sm = 1;
    c.threads = 1024;
  }
  if (c.threads % 128 || c.threads > 1024) return GSRB_ERR_ARG;
  if (n == 0) return GSRB_OK;
  uint32_t tile = c.tile > 0 ? (uint32_t)c.tile : kDefaultTile;
  tile = (tile + 3) & ~3u;
  const size_t smem = 2 * (size_t)tile * 4;
  if ((int)smem > ctx->max_smem_optin - 2048) return GSRB_ERR_ARG;
  const void* fn = f32 ? scan_fn_t<true>(c.variant) : scan_fn_t<false>(c.variant);
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster) return GSRB_ERR_ARG;
  void* part = nullptr;
  gsrb_status_t st = scratch(ctx, sizeof(unsigned long long) * 2 * (size_t)grid, &part);
  if (st) return st;
  gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)grid, 0, 0);
  uint64_t n64 = n;
  unsigned long long* partials = (unsigned long long*)part;
  int in_bulk = ((uintptr_t)d_in & 15u) == 0;
  int out_bulk = ((uintptr_t)d_out & 15u) == 0;
  void* args[] = {&gb, (void*)&d_in, &d_out, &n64, &tile, &partials, &in_bulk, &out_bulk};
  return launch_persistent(ctx, fn, grid, c.threads, smem, c.cluster, coop_of(c), args);
}

}  // namespace

const void* gsrb_scan_kernel_for(int variant, int f32) {
  return f32 ? scan_fn_t<true>(variant) : scan_fn_t<false>(variant);
}

extern "C" {

gsrb_status_t gsrb_scan_u32(gsrb_ctx_t ctx, const uint32_t* d_in, uint32_t* d_out, size_t n,
                            const gsrb_cfg_t* cfg) {
  return scan_launch(ctx, d_in, d_out, n, cfg, false);
}

gsrb_status_t gsrb_scan_f32(gsrb_ctx_t ctx, const float* d_in, float* d_out, size_t n, const gsrb_cfg_t* cfg) {
  return scan_launch(ctx, d_in, d_out, n, cfg, true);
}

}  // extern "C"
