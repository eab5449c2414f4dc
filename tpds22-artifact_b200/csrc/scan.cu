// Persistent barrier-stepped exclusive scan (uint32 with wraparound, and FP32
// with FP64 offsets).
//
// Reference: gpu_prescan + sum_scan_blelloch in scan/scan_gsrb.cu:486-804
// (API scan/scan.h:16-18): 64-element Blelloch tiles (32 threads), a grid
// barrier per recursion level, two fix-up launches (gpu_add_block_sums,
// :440-482, :798-799), grid = ceil(N / 64) CTAs that must all be co-resident
// (N <= 148*32*64 on B200).
//
// Here: a fixed co-resident grid (default one 1024-thread CTA per SM) walks the
// input in segments of G chunks (one chunk of `chunk` elements per CTA).  The
// three phases of the reference run per segment, software-pipelined so that
// the grid barrier of segment s overlaps the HBM reads of segment s + 1:
//
//   R(s+1)  every warp sums its slice of the CTA's chunk of segment s+1
//           (128-bit L2-only loads, 8 per lane in flight); warp totals go to
//           shared memory (double-buffered by segment parity)
//   wait(s) the split-phase grid barrier of segment s completes
//   W(s)    offset = running carry + the partials of the CTAs before this one
//           (every CTA reads the G partials of the segment, so the reference's
//           separate scan of block sums and its second barrier are not
//           needed); each warp re-reads its slice (an L2 hit: the segment was
//           read one step earlier and is a few tens of MB), scans it with warp
//           shuffles and writes it with streaming stores
//   arrive(s+1) after publishing the CTA's partial of segment s+1
//
// HBM sees each element read once and written once (8N bytes); the re-read is
// served by the 126 MB L2.  Partials are double-buffered by segment parity: a
// CTA publishes the partial of s+1 only after it has read those of s, and the
// buffer of s+2 is written only after every CTA's arrival at s+1, i.e. after
// every CTA has finished reading the partials of s.
#include "internal.h"

using namespace gsrbrt;

namespace {

template <bool F32>
struct ScanT;
template <>
struct ScanT<false> {
  using Elem = uint32_t;
  using Acc = uint32_t;  // uint32 wraparound, like cpu_sum_scan (scan/main.cu:15-20)
  using Vec = uint4;
};
// FP32: chunk offsets and carries in FP64; the scan inside one warp round (32
// lanes x 4 elements, depth 7 additions of non-negative partial sums) in FP32,
// which adds at most ~7 ulp relative to the round's partial sums; each lane's
// FP64 prefix is rounded to FP32 once and its 3 local prefixes added in FP32
// (out_vec).
template <>
struct ScanT<true> {
  using Elem = float;
  using Acc = double;
  using Vec = float4;
};

__device__ __forceinline__ uint32_t shfl_up(uint32_t v, int o) { return __shfl_up_sync(0xffffffffu, v, o); }
__device__ __forceinline__ float shfl_up(float v, int o) { return __shfl_up_sync(0xffffffffu, v, o); }
__device__ __forceinline__ float shfl_idx(float v, int l) { return __shfl_sync(0xffffffffu, v, l); }
__device__ __forceinline__ uint32_t shfl_idx(uint32_t v, int l) { return __shfl_sync(0xffffffffu, v, l); }
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

// 128-bit loads / stores with L2 eviction-priority hints: the first read of a
// chunk marks its lines evict-last (they are read again one step later), the
// re-read marks them evict-first, the output is written evict-first.  The
// policies come from createpolicy (fraction 1.0).
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint4 ld_hint(const uint4* ptr, uint64_t pol) {
  uint4 v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.u32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(ptr), "l"(pol));
  return v;
}
__device__ __forceinline__ float4 ld_hint(const float4* ptr, uint64_t pol) {
  float4 v;
  asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.f32 {%0,%1,%2,%3}, [%4], %5;"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(ptr), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_hint(uint4* ptr, uint4 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.u32 [%0], {%1,%2,%3,%4}, %5;"
               ::"l"(ptr), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_hint(float4* ptr, float4 v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1,%2,%3,%4}, %5;"
               ::"l"(ptr), "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(pol) : "memory");
}

// Output vector of one lane's 4 elements: e0 is the exclusive prefix before the
// lane's first element (carry in Acc), a0..a2 the lane-local inclusive prefixes.
// uint32 is exact in any order.  FP32: e0 is rounded once to FP32 and the three
// local prefixes are added in FP32, two roundings of at most half an ulp of the
// result each (about 1.2e-7 relative), instead of three FP64 additions.
__device__ __forceinline__ uint4 out_vec(uint32_t e0, uint32_t a0, uint32_t a1, uint32_t a2) {
  return make_uint4(e0, e0 + a0, e0 + a1, e0 + a2);
}
__device__ __forceinline__ float4 out_vec(double e0, float a0, float a1, float a2) {
  const float b = (float)e0;
  return make_float4(b, b + a0, b + a1, b + a2);
}

struct TileGeom {
  uint64_t beg;   // first element of this CTA's chunk
  uint32_t cnt;   // valid elements
  uint32_t span;  // chunk stride of the segment (multiple of 4)
};

// Full segments use chunks of `chunk` elements; the last segment is split
// evenly (span rounded up to a multiple of 4, trailing CTAs may get less).
__device__ __forceinline__ TileGeom tile_of(uint64_t s, uint64_t n, uint32_t G, uint32_t chunk, uint32_t b) {
  const uint64_t seg = (uint64_t)G * chunk;
  const uint64_t base = s * seg;
  const uint64_t rem = n - base;
  TileGeom t;
  if (rem >= seg) {
    t.span = chunk;
  } else {
    uint64_t q = (rem + G - 1) / G;
    t.span = (uint32_t)((q + 3) & ~3ull);
  }
  t.beg = base + (uint64_t)b * t.span;
  const uint64_t left = t.beg >= n ? 0ull : n - t.beg;
  t.cnt = (uint32_t)(left < (uint64_t)t.span ? left : (uint64_t)t.span);
  return t;
}

// Vector v (elements 4v..4v+3) of a chunk; elements past cnt read as zero.
template <bool F32>
__device__ __forceinline__ typename ScanT<F32>::Vec load_vec(const typename ScanT<F32>::Elem* __restrict__ in,
                                                             const TileGeom& t, uint32_t v, bool vec_ok,
                                                             uint64_t pol) {
  using Elem = typename ScanT<F32>::Elem;
  using Vec = typename ScanT<F32>::Vec;
  Vec x;
  const uint32_t e = 4u * v;
  if (vec_ok && e + 3u < t.cnt) {
    x = ld_hint(reinterpret_cast<const Vec*>(in + t.beg + e), pol);
  } else {
    Elem y[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) y[k] = (e + k < t.cnt) ? in[t.beg + e + k] : Elem(0);
    x.x = y[0];
    x.y = y[1];
    x.z = y[2];
    x.w = y[3];
  }
  return x;
}

template <int V, bool F32>
__global__ void __launch_bounds__(1024, 1)
scan_kernel(gsrb::GridBarrier gb, const typename ScanT<F32>::Elem* __restrict__ in,
            typename ScanT<F32>::Elem* __restrict__ out, uint64_t n, uint32_t chunk,
            unsigned long long* __restrict__ partials, int vec_in, int vec_out) {
  using Elem = typename ScanT<F32>::Elem;
  using Acc = typename ScanT<F32>::Acc;
  using Vec = typename ScanT<F32>::Vec;
  constexpr uint32_t kInFlight = 8;  // 128-bit loads per lane in flight in the reduce phase
  __shared__ gsrb::BarrierShared bsh;
  __shared__ Acc s_wsum[2][32];  // warp totals -> exclusive warp offsets, by segment parity
  __shared__ Acc s_red[2][32];
  __shared__ Acc s_bcast[2];

  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t G = gridDim.x, b = blockIdx.x;
  const uint64_t pol_keep = l2_policy_evict_last(), pol_drop = l2_policy_evict_first();
  gsrb::GridSync<V> bar;
  bool ok = bar.init(gb, &bsh);

  const uint64_t seg = (uint64_t)G * chunk;
  const uint64_t nseg = (n + seg - 1) / seg;

  // R(s): warp totals of this CTA's chunk of segment s into s_wsum[s & 1]
  auto reduce_phase = [&](uint64_t s) {
    const TileGeom t = tile_of(s, n, G, chunk, b);
    const uint32_t nvec = t.span >> 2;
    const uint32_t vpw = (nvec + nw - 1) / nw;
    const uint32_t v0 = w * vpw, v1 = min(nvec, v0 + vpw);
    Acc lsum = Acc(0);
    for (uint32_t v = v0 + lane; v < v1; v += 32u * kInFlight) {
      Vec x[kInFlight];
#pragma unroll
      for (uint32_t k = 0; k < kInFlight; ++k) {
        const uint32_t vk = v + 32u * k;
        if (vk < v1) x[k] = load_vec<F32>(in, t, vk, vec_in != 0, pol_keep);
        else memset(&x[k], 0, sizeof(Vec));
      }
#pragma unroll
      for (uint32_t k = 0; k < kInFlight; ++k) lsum += vsum(x[k]);
    }
    const Acc wt = warp_sum(lsum);
    if (lane == 0) s_wsum[s & 1][w] = wt;
  };
  // after a __syncthreads: exclusive warp offsets, and the CTA's partial
  auto publish = [&](uint64_t s) {
    if (tid == 0) {
      Acc run = Acc(0);
      for (uint32_t i = 0; i < nw; ++i) {
        const Acc x = s_wsum[s & 1][i];
        s_wsum[s & 1][i] = run;
        run += x;
      }
      __stcg(&partials[(s & 1) * G + b], (unsigned long long)acc_bits(run));
    }
  };
  // W(s): re-read, scan and write this CTA's chunk of segment s
  auto write_phase = [&](uint64_t s, Acc base) {
    const TileGeom t = tile_of(s, n, G, chunk, b);
    const uint32_t nvec = t.span >> 2;
    const uint32_t vpw = (nvec + nw - 1) / nw;
    const uint32_t v0 = w * vpw, v1 = min(nvec, v0 + vpw);
    Acc run = base + s_wsum[s & 1][w];
    for (uint32_t r0 = v0; r0 < v1; r0 += 32u * kInFlight) {
      // all re-reads of this step in flight together (L2 hits), then the rounds
      Vec xs[kInFlight];
#pragma unroll
      for (uint32_t k = 0; k < kInFlight; ++k) {
        const uint32_t v = r0 + 32u * k + lane;
        if (v < v1) xs[k] = load_vec<F32>(in, t, v, vec_in != 0, pol_drop);
        else memset(&xs[k], 0, sizeof(Vec));
      }
#pragma unroll
      for (uint32_t k = 0; k < kInFlight; ++k) {
        if (r0 + 32u * k >= v1) break;  // warp-uniform
        const uint32_t v = r0 + 32u * k + lane;
        const Vec x = xs[k];
        // lane-local inclusive prefix of 4 elements
        const Elem a0 = x.x, a1 = a0 + x.y, a2 = a1 + x.z, a3 = a2 + x.w;
        const Elem lt = a3;
        Elem incl = lt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const Elem y = shfl_up(incl, o);
          if ((int)lane >= o) incl += y;
        }
        const Acc e0 = run + Acc(incl - lt);
        const Vec y = out_vec(e0, a0, a1, a2);
        const uint32_t e = 4u * v;
        if (v < v1) {
          if (vec_out && e + 3u < t.cnt) {
            st_hint(reinterpret_cast<Vec*>(out + t.beg + e), y, pol_drop);
          } else {
            const Elem ys[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
            for (int q = 0; q < 4; ++q)
              if (e + q < t.cnt) out[t.beg + e + q] = ys[q];
          }
        }
        run += Acc(shfl_idx(incl, 31));
      }
    }
  };

  if (ok && nseg > 0) {
    reduce_phase(0);
    __syncthreads();
    publish(0);
    bar.arrive();
  }
  Acc carry = Acc(0);
  for (uint64_t s = 0; ok && s < nseg; ++s) {
    if (s + 1 < nseg) reduce_phase(s + 1);  // overlaps the barrier of segment s
    ok = bar.wait();
    if (!ok) break;

    // offset = carry + sum of the partials of the CTAs before b
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
    write_phase(s, base);

    if (s + 1 < nseg) {
      __syncthreads();  // warp totals of s+1 are in shared memory; s_red/s_bcast reads are done
      publish(s + 1);
      bar.arrive();
    }
  }
  bar.finish();
}

// ---------------------------------------------------------------------------
// Warp-specialised form (barriers with a thread-level split protocol: V_FANOUT
// and V_HIER).  Readers (warps [0, NR)) run the chunk sums R(s) one segment
// ahead; writers (warps [NR, 2 NR)) wait for the grid barrier of s, read the
// partials and run W(s) (re-read from L2, scan, stream out).  The HBM reads of
// s+1 then overlap the barrier latency, the partial reads and the re-read of s
// instead of alternating with them.  Reader warp j and writer warp j own the
// same slice of the chunk.
//
// Ordering (all waits bounded):
//  * readers start R(s) only after the writers finished W(s-2), so at most two
//    segments (the one being read, the one being written) are in L2 between
//    their first read and their re-read;
//  * the reader leader arrives for s only after the writer leader passed the
//    barrier of s-1 (each episode's counter is reset by its completer);
//  * slice offsets and partials rotate over kBufs = 4 buffers: partial(s) is
//    written after this CTA's writer passed s-1, so every CTA arrived at s-1,
//    so every writer passed s-2 and has finished reading the partials of s-3
//    and older; offsets(s) are written after this CTA's writers finished
//    W(s-2), the last user of buffer (s + 2) % 4 ... and of s % 4 (W(s-4)).
__device__ __forceinline__ void named_sync(uint32_t id, uint32_t nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Bounded wait for a shared counter written by another warp of the CTA.
__device__ __forceinline__ bool smem_wait_ge(const volatile uint32_t* p, uint32_t target,
                                             const gsrb::GridBarrier& gb) {
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    if ((int32_t)(*p - target) >= 0) {
      __threadfence_block();
      return true;
    }
    if ((it & 63u) == 63u) {
      if (gsrb::ptx::ld_relaxed_gpu(&gb.slot->status) != 0u) return false;
      const uint64_t now = gsrb::ptx::globaltimer_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > gb.timeout_ns) {
        gsrb::detail::record_error(gb, gsrb::GSRB_DEV_TIMEOUT, 0xfffffff2u);
        return false;
      }
    }
  }
}

template <int V>
__device__ __forceinline__ void ws_arrive(const gsrb::GridBarrier& gb, uint32_t idx, uint32_t n, uint32_t epoch) {
  if (V == gsrb::V_HIER) gsrb::detail::hier_arrive(gb, idx, n, epoch);
  else gsrb::detail::fanout_arrive(gb, n, epoch);
}

template <int V, bool F32>
__global__ void __launch_bounds__(1024, 1)
scan_ws_kernel(gsrb::GridBarrier gb, const typename ScanT<F32>::Elem* __restrict__ in,
               typename ScanT<F32>::Elem* __restrict__ out, uint64_t n, uint32_t chunk,
               unsigned long long* __restrict__ partials, int vec_in, int vec_out) {
  using Elem = typename ScanT<F32>::Elem;
  using Acc = typename ScanT<F32>::Acc;
  using Vec = typename ScanT<F32>::Vec;
  constexpr uint32_t kInFlight = 8;
  constexpr uint32_t kBufs = 4;
  __shared__ gsrb::BarrierShared bsh;
  __shared__ Acc s_rtmp[2][16];     // reader warp totals, by parity of s
  __shared__ Acc s_off[kBufs][16];  // exclusive slice offsets, by s % kBufs
  __shared__ Acc s_wred[2][16];
  __shared__ Acc s_wb[2];
  __shared__ volatile uint32_t s_wr_passed, s_wr_done, s_rfail, s_wfail;
  __shared__ uint32_t s_epoch0;

  const uint32_t tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
  const uint32_t NR = nw >> 1, rth = NR * 32u;  // readers: warps [0, NR); writers: [NR, 2 NR)
  const uint32_t G = gridDim.x, b = blockIdx.x;
  const uint64_t pol_keep = l2_policy_evict_last(), pol_drop = l2_policy_evict_first();
  gsrb::GridSync<V> bar;
  const bool ok0 = bar.init(gb, &bsh);
  if (tid == 0) {
    s_epoch0 = bar.epoch;
    s_wr_passed = 0;
    s_wr_done = 0;
    s_rfail = ok0 ? 0u : 1u;
    s_wfail = ok0 ? 0u : 1u;
  }
  __syncthreads();
  const uint32_t epoch0 = s_epoch0;
  const uint64_t seg = (uint64_t)G * chunk;
  const uint64_t nseg = (n + seg - 1) / seg;

  if (w < NR) {
    // ------------------------------------------------------------ readers
    for (uint64_t s = 0; s < nseg; ++s) {
      if (s >= 1) {
        if (tid == 0 && s >= 2 && !smem_wait_ge(&s_wr_done, (uint32_t)(s - 1), gb)) s_rfail = 1u;  // W(s-2) done
        named_sync(1, rth);
      }
      // s_rfail is only written by the leader before a reader barrier (or
      // before the block-wide one ahead of the loop): every reader sees the
      // same value here
      if (s_rfail) break;
      const TileGeom t = tile_of(s, n, G, chunk, b);
      const uint32_t nvec = t.span >> 2;
      const uint32_t vps = (nvec + NR - 1) / NR;
      const uint32_t v0 = w * vps, v1 = min(nvec, v0 + vps);
      Acc lsum = Acc(0);
      for (uint32_t v = v0 + lane; v < v1; v += 32u * kInFlight) {
        Vec x[kInFlight];
#pragma unroll
        for (uint32_t k = 0; k < kInFlight; ++k) {
          const uint32_t vk = v + 32u * k;
          if (vk < v1) x[k] = load_vec<F32>(in, t, vk, vec_in != 0, pol_keep);
          else memset(&x[k], 0, sizeof(Vec));
        }
#pragma unroll
        for (uint32_t k = 0; k < kInFlight; ++k) lsum += vsum(x[k]);
      }
      const Acc wt = warp_sum(lsum);
      if (lane == 0) s_rtmp[s & 1][w] = wt;
      named_sync(1, rth);
      if (tid == 0) {
        bool ok = s == 0 || smem_wait_ge(&s_wr_passed, (uint32_t)s, gb);  // writers passed s-1
        if (ok) {
          Acc run = Acc(0);
          for (uint32_t i = 0; i < NR; ++i) {
            const Acc x = s_rtmp[s & 1][i];
            s_off[s % kBufs][i] = run;
            run += x;
          }
          __stcg(&partials[(s % kBufs) * G + b], (unsigned long long)acc_bits(run));
          ws_arrive<V>(gb, b - gb.first_cta, gb.nparticipants, epoch0 + (uint32_t)s);
        } else {
          s_rfail = 1u;
        }
      }
    }
  } else {
    // ------------------------------------------------------------ writers
    const uint32_t wt_id = tid - rth, ww = w - NR;
    const bool leader = wt_id == 0;
    Acc carry = Acc(0);
    for (uint64_t s = 0; s < nseg; ++s) {
      if (leader) {
        const bool ok = gsrb::detail::fanout_wait(gb, b - gb.first_cta, epoch0 + (uint32_t)s, (uint32_t)s);
        if (!ok) s_wfail = 1u;
        __threadfence_block();
        s_wr_passed = (uint32_t)s + 1u;
      }
      named_sync(2, rth);
      if (s_wfail) break;  // uniform: written by the leader before this barrier
      // offset = carry + partials of the CTAs before b
      Acc pre = Acc(0), tot = Acc(0);
      for (uint32_t j = wt_id; j < G; j += rth) {
        Acc x;
        acc_from(__ldcg(&partials[(s % kBufs) * G + j]), x);
        tot += x;
        if (j < b) pre += x;
      }
      pre = warp_sum(pre);
      tot = warp_sum(tot);
      if (lane == 0) {
        s_wred[0][ww] = pre;
        s_wred[1][ww] = tot;
      }
      named_sync(2, rth);
      if (leader) {
        Acc p = Acc(0), q = Acc(0);
        for (uint32_t i = 0; i < NR; ++i) {
          p += s_wred[0][i];
          q += s_wred[1][i];
        }
        s_wb[0] = p;
        s_wb[1] = q;
      }
      named_sync(2, rth);
      const Acc base = carry + s_wb[0];
      carry += s_wb[1];
      // W(s): re-read the slice (L2), scan, stream out
      const TileGeom t = tile_of(s, n, G, chunk, b);
      const uint32_t nvec = t.span >> 2;
      const uint32_t vps = (nvec + NR - 1) / NR;
      const uint32_t v0 = ww * vps, v1 = min(nvec, v0 + vps);
      Acc run = base + s_off[s % kBufs][ww];
      for (uint32_t r0 = v0; r0 < v1; r0 += 32u * kInFlight) {
        Vec xs[kInFlight];
#pragma unroll
        for (uint32_t k = 0; k < kInFlight; ++k) {
          const uint32_t v = r0 + 32u * k + lane;
          if (v < v1) xs[k] = load_vec<F32>(in, t, v, vec_in != 0, pol_drop);
          else memset(&xs[k], 0, sizeof(Vec));
        }
#pragma unroll
        for (uint32_t k = 0; k < kInFlight; ++k) {
          if (r0 + 32u * k >= v1) break;  // warp-uniform
          const uint32_t v = r0 + 32u * k + lane;
          const Vec x = xs[k];
          const Elem a0 = x.x, a1 = a0 + x.y, a2 = a1 + x.z, a3 = a2 + x.w;
          const Elem lt = a3;
          Elem incl = lt;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const Elem y = shfl_up(incl, o);
            if ((int)lane >= o) incl += y;
          }
          const Acc e0 = run + Acc(incl - lt);
          const Vec y = out_vec(e0, a0, a1, a2);
          const uint32_t e = 4u * v;
          if (v < v1) {
            if (vec_out && e + 3u < t.cnt) {
              st_hint(reinterpret_cast<Vec*>(out + t.beg + e), y, pol_drop);
            } else {
              const Elem ys[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
              for (int q = 0; q < 4; ++q)
                if (e + q < t.cnt) out[t.beg + e + q] = ys[q];
            }
          }
          run += Acc(shfl_idx(incl, 31));
        }
      }
      named_sync(2, rth);
      if (leader) {
        __threadfence_block();
        s_wr_done = (uint32_t)s + 1u;
      }
    }
  }
  __syncthreads();
  bar.finish();
}

template <bool F32>
const void* scan_ws_fn_t(int variant) {
  switch (variant) {
    case gsrb::V_FANOUT: return (const void*)scan_ws_kernel<gsrb::V_FANOUT, F32>;
    case gsrb::V_HIER: return (const void*)scan_ws_kernel<gsrb::V_HIER, F32>;
    default: return nullptr;
  }
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

constexpr uint32_t kDefaultChunk = 32768;  // elements per CTA per segment (128 KiB; a segment of 148 is 19 MiB)

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
  // barriers with a thread-level split protocol run the warp-specialised form
  const void* fn = f32 ? scan_ws_fn_t<true>(c.variant) : scan_ws_fn_t<false>(c.variant);
  if (!fn) fn = f32 ? scan_fn_t<true>(c.variant) : scan_fn_t<false>(c.variant);
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  uint32_t tile = c.tile > 0 ? (uint32_t)c.tile : kDefaultChunk;
  tile = (tile + 3) & ~3u;
  const size_t smem = 0;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster) return GSRB_ERR_ARG;
  void* part = nullptr;
  gsrb_status_t st = scratch(ctx, sizeof(unsigned long long) * 4 * (size_t)grid, &part);
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
  const void* fn = f32 ? scan_ws_fn_t<true>(variant) : scan_ws_fn_t<false>(variant);
  return fn ? fn : (f32 ? scan_fn_t<true>(variant) : scan_fn_t<false>(variant));
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
