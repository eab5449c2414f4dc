// Batched reduce and scan: k independent segments of uneven lengths in one
// persistent launch, each on its own sub-grid barrier.
//
// Reference: the single-array forms reduce() (Reduce/reduce_gsrb.cu:289-404)
// and sum_scan_blelloch (scan/scan_gsrb.cu:486-804), which take one array per
// launch and synchronise the whole grid per level.  Here the segments of a
// call share one launch: segment i gets CTAs [first_i, first_i + count_i), in
// proportion to its length and at least one, and barrier slot 1 + i (sub-grid
// barriers carved from the same state block as the whole-grid barrier, as the
// batched traversals do).  The layout is a pure function of the offsets, the
// number of segments and the grid, so every CTA computes it itself from the
// launch parameters: nothing is copied to the device per call, and a call can
// be captured into a CUDA graph and replayed.
//
//   reduce  each CTA sums a contiguous slice of its segment (int64), stores
//           the partial, arrives on the segment's barrier; the combiner (the
//           completing CTA for the fan-out protocol, else the segment's first
//           CTA after a wait) adds the segment's partials in CTA order.
//   scan    (exclusive; uint32 wrapping, or FP32 with FP64 chunk sums and
//           carries) in rounds, so that the re-read comes from L2:
//           in round j the team's CTAs take consecutive chunks of `chunk`
//           elements (CTA r the r-th); chunk sums -> segment barrier -> every
//           CTA adds the round's sums of the CTAs before it to the running
//           total of the earlier rounds -> rescan of the chunk in tiles of
//           16 x blockDim elements staged through shared memory (coalesced
//           loads and stores whatever the offsets' alignment).  One round has
//           grid x chunk elements in flight (about 38 MB at the default shape),
//           so the rescan re-reads L2, not HBM.  The barrier is split: a CTA
//           arrives for round j, reads round j + 1's chunk sum from HBM, then
//           waits.  The round sums are double buffered: a CTA writes round
//           j + 1's sum only after the barrier of round j, which every CTA
//           reaches after reading round j - 1's.
#include "internal.h"

#include <string.h>

using namespace gsrbrt;

namespace {

constexpr int kMaxSegments = kSlots - 1;

struct SegParams {
  gsrb::GridBarrier gb;   // slot 1's descriptor (nparticipants/first_cta set per segment)
  uint64_t flip_stride;   // words between consecutive slots' flip areas
  uint32_t k;
  uint32_t chunk;         // scan: elements per CTA per round (whole tiles of kScanV x blockDim)
  uint64_t off[kMaxSegments + 1];
};

// First CTA of segment i: i + floor(left * off[i] / total), left = grid - k
// (so every segment has at least one CTA and the rest go in proportion to
// length); with no elements at all, segment i < k - 1 gets CTA i and the last
// segment the rest.  Strictly increasing in i; first(k) = grid.
__host__ __device__ __forceinline__ uint32_t seg_first(const uint64_t* off, uint32_t k, uint32_t grid, uint32_t i) {
  const uint64_t total = off[k] - off[0];
  if (i >= k) return grid;
  if (total == 0) return i;
  const uint64_t left = (uint64_t)(grid - k);
  return i + (uint32_t)((left * (off[i] - off[0])) / total);
}

// Segment of CTA b (the last i with seg_first(i) <= b).
__host__ __device__ __forceinline__ uint32_t seg_of(const uint64_t* off, uint32_t k, uint32_t grid, uint32_t b) {
  uint32_t lo = 0, hi = k - 1;
  while (lo < hi) {
    const uint32_t mid = (lo + hi + 1) >> 1;
    if (seg_first(off, k, grid, mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

struct SegTeam {
  uint32_t seg, first, count, rank;
  uint64_t a, b;  // this CTA's slice [a, b) (absolute element indices)
};

__device__ __forceinline__ SegTeam seg_team(const SegParams& p) {
  SegTeam t;
  t.seg = seg_of(p.off, p.k, gridDim.x, blockIdx.x);
  t.first = seg_first(p.off, p.k, gridDim.x, t.seg);
  t.count = seg_first(p.off, p.k, gridDim.x, t.seg + 1) - t.first;
  t.rank = blockIdx.x - t.first;
  const uint64_t o0 = p.off[t.seg], o1 = p.off[t.seg + 1];
  const uint64_t len = o1 - o0;
  uint64_t per = (len + t.count - 1) / t.count;
  per = (per + 3) & ~3ull;
  t.a = o0 + per * t.rank;
  if (t.a > o1) t.a = o1;
  t.b = t.a + per < o1 ? t.a + per : o1;
  return t;
}

__device__ __forceinline__ gsrb::GridBarrier seg_barrier(const SegParams& p, const SegTeam& t) {
  gsrb::GridBarrier gb = p.gb;
  gb.slot += t.seg;
  gb.flip += p.flip_stride * t.seg;
  gb.nparticipants = t.count;
  gb.first_cta = t.first;
  return gb;
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum, valid in every thread (fixed order).
template <typename T>
__device__ __forceinline__ T block_sum(T v, T* buf) {
  v = warp_sum(v);
  const uint32_t lane = threadIdx.x & 31u, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();
  if (lane == 0) buf[w] = v;
  __syncthreads();
  T s = lane < nw ? buf[lane] : T(0);
  return warp_sum(s);
}

// Sum of in[a, b) by the CTA: 16-byte loads over the aligned body, four in
// flight per thread, scalar head and tail.
__device__ __forceinline__ long long slice_sum_i32(const int32_t* __restrict__ in, uint64_t a, uint64_t b) {
  const uint32_t tid = threadIdx.x, T = blockDim.x;
  long long acc = 0;
  uint64_t h = a;
  while (h < b && (reinterpret_cast<uintptr_t>(in + h) & 15u)) ++h;
  const uint64_t nv = (b - h) >> 2;
  const uint64_t t0 = h + (nv << 2);
  for (uint64_t i = a + tid; i < h; i += T) acc += __ldg(in + i);
  const int4* v = reinterpret_cast<const int4*>(in + h);
  uint64_t i = tid;
  for (; i + 3ull * T < nv; i += 4ull * T) {
    const int4 x0 = __ldcs(v + i), x1 = __ldcs(v + i + T), x2 = __ldcs(v + i + 2ull * T), x3 = __ldcs(v + i + 3ull * T);
    acc += (long long)x0.x + x0.y + x0.z + x0.w;
    acc += (long long)x1.x + x1.y + x1.z + x1.w;
    acc += (long long)x2.x + x2.y + x2.z + x2.w;
    acc += (long long)x3.x + x3.y + x3.z + x3.w;
  }
  for (; i < nv; i += T) {
    const int4 x = __ldcs(v + i);
    acc += (long long)x.x + x.y + x.z + x.w;
  }
  for (uint64_t j = t0 + tid; j < b; j += T) acc += __ldg(in + j);
  return acc;
}

// Scan element traits: uint32 scans wrap (bit-exact against cpu_sum_scan);
// FP32 scans keep chunk sums and carries in FP64 and scan within a tile in
// FP32 (the error of an element is then a few ulps of its prefix).
template <typename T> struct ScanT;
template <> struct ScanT<uint32_t> {
  using Acc = uint32_t;
  using Vec = uint4;
  __device__ static __forceinline__ Acc vsum(uint4 x) { return (x.x + x.y) + (x.z + x.w); }
  __device__ static __forceinline__ uint32_t out(Acc carry, uint32_t e) { return carry + e; }
};
template <> struct ScanT<float> {
  using Acc = double;
  using Vec = float4;
  __device__ static __forceinline__ Acc vsum(float4 x) { return ((double)x.x + x.y) + ((double)x.z + x.w); }
  __device__ static __forceinline__ float out(Acc carry, float e) { return (float)(carry + (double)e); }
};

// Sum of in[a, b) by the CTA (per thread, in the accumulation type): 16-byte
// loads over the aligned body, four in flight per thread, kept in L2 for the
// rescan; scalar head and tail.
template <typename T>
__device__ __forceinline__ typename ScanT<T>::Acc slice_sum(const T* __restrict__ in, uint64_t a, uint64_t b) {
  using Acc = typename ScanT<T>::Acc;
  using Vec = typename ScanT<T>::Vec;
  const uint32_t tid = threadIdx.x, NT = blockDim.x;
  Acc acc = 0;
  uint64_t h = a;
  while (h < b && (reinterpret_cast<uintptr_t>(in + h) & 15u)) ++h;
  const uint64_t nv = (b - h) >> 2;
  const uint64_t t0 = h + (nv << 2);
  for (uint64_t i = a + tid; i < h; i += NT) acc += (Acc)__ldg(in + i);
  const Vec* v = reinterpret_cast<const Vec*>(in + h);
  uint64_t i = tid;
  for (; i + 3ull * NT < nv; i += 4ull * NT) {
    const Vec x0 = __ldcg(v + i), x1 = __ldcg(v + i + NT), x2 = __ldcg(v + i + 2ull * NT), x3 = __ldcg(v + i + 3ull * NT);
    acc += ScanT<T>::vsum(x0) + ScanT<T>::vsum(x1);
    acc += ScanT<T>::vsum(x2) + ScanT<T>::vsum(x3);
  }
  for (; i < nv; i += NT) acc += ScanT<T>::vsum(__ldcg(v + i));
  for (uint64_t j = t0 + tid; j < b; j += NT) acc += (Acc)__ldg(in + j);
  return acc;
}

template <int V>
__global__ void __launch_bounds__(1024)
reduce_segments_kernel(SegParams p, const int32_t* __restrict__ in, long long* __restrict__ partials,
                       long long* __restrict__ out) {
  __shared__ gsrb::BarrierShared bsh;
  __shared__ long long buf[32];
  __shared__ uint32_t s_comb;
  const SegTeam t = seg_team(p);
  gsrb::GridSync<V> bar;
  const bool ok = bar.init(seg_barrier(p, t), &bsh);
  long long s = 0;
  if (ok) s = slice_sum_i32(in, t.a, t.b);
  s = block_sum(s, buf);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  bar.arrive();
  bool done = true, combiner;
  if (gsrb::GridSync<V>::kCompleter) {
    if (threadIdx.x == 0) s_comb = bar.arrived_done;
    __syncthreads();
    combiner = s_comb != 0u;
  } else {
    combiner = t.rank == 0;
    if (!gsrb::GridSync<V>::kSplit || combiner) done = bar.wait();
  }
  if (ok && done && combiner) {
    long long c = 0;
    for (uint32_t j = threadIdx.x; j < t.count; j += blockDim.x) c += __ldcg(partials + t.first + j);
    c = block_sum(c, buf);
    if (threadIdx.x == 0) out[t.seg] = c;
  }
  bar.finish();
}

// Elements per thread of a scan tile, and the shared-memory word of tile
// element e: one pad word per 32 elements, so that the coalesced fill (32
// consecutive elements per warp) and the per-thread reads (kScanV consecutive
// elements per lane, lanes kScanV apart) both touch 32 distinct banks.
constexpr uint32_t kScanV = 16;
__device__ __forceinline__ uint32_t tpos(uint32_t e) { return e + (e >> 5); }

// Exclusive scan of one tile of up to kScanV * blockDim elements starting at
// `base` (n elements valid), offset by `carry`; returns the tile's total.  All
// kScanV loads of a thread are issued before the first is used.
template <typename T>
__device__ __forceinline__ typename ScanT<T>::Acc scan_tile(const T* __restrict__ in, T* __restrict__ out,
                                                            uint64_t base, uint32_t n,
                                                            typename ScanT<T>::Acc carry, T* tile, T* wsum) {
  const uint32_t tid = threadIdx.x, NT = blockDim.x;
  const uint32_t lane = tid & 31u, w = tid >> 5, nw = NT >> 5;
  T x[kScanV];
#pragma unroll
  for (uint32_t r = 0; r < kScanV; ++r) {
    const uint32_t j = r * NT + tid;
    x[r] = j < n ? __ldcg(in + base + j) : T(0);
  }
#pragma unroll
  for (uint32_t r = 0; r < kScanV; ++r) tile[tpos(r * NT + tid)] = x[r];
  __syncthreads();
  T sum = 0;
#pragma unroll
  for (uint32_t r = 0; r < kScanV; ++r) {
    const T v = tile[tpos(kScanV * tid + r)];
    x[r] = sum;
    sum += v;
  }
  // block exclusive scan of the per-thread sums
  T inc = sum;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(0xffffffffu, inc, o);
    if ((int)lane >= o) inc += y;
  }
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  if (w == 0) {
    T v = lane < nw ? wsum[lane] : T(0);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(0xffffffffu, v, o);
      if ((int)lane >= o) v += y;
    }
    wsum[lane] = v;  // inclusive warp prefix; wsum[31] = tile total
  }
  __syncthreads();
  const T excl = (w ? wsum[w - 1] : T(0)) + (inc - sum);
#pragma unroll
  for (uint32_t r = 0; r < kScanV; ++r) tile[tpos(kScanV * tid + r)] = ScanT<T>::out(carry, excl + x[r]);
  __syncthreads();
#pragma unroll
  for (uint32_t r = 0; r < kScanV; ++r) {
    const uint32_t j = r * NT + tid;
    if (j < n) __stcs(out + base + j, tile[tpos(j)]);
  }
  const typename ScanT<T>::Acc total = wsum[31];
  __syncthreads();  // tile and wsum are reused by the next tile
  return total;
}

template <int V, typename T>
__global__ void __launch_bounds__(1024)
scan_segments_kernel(SegParams p, const T* __restrict__ in, T* __restrict__ out,
                     typename ScanT<T>::Acc* __restrict__ partials) {
  using Acc = typename ScanT<T>::Acc;
  __shared__ gsrb::BarrierShared bsh;
  __shared__ Acc buf[32];
  __shared__ T wsum[32];
  extern __shared__ __align__(16) unsigned char tile_raw[];  // tpos(kScanV * blockDim) elements
  T* tile = reinterpret_cast<T*>(tile_raw);
  const SegTeam t = seg_team(p);
  gsrb::GridSync<V> bar;
  bool ok = bar.init(seg_barrier(p, t), &bsh);
  const uint64_t o0 = p.off[t.seg], o1 = p.off[t.seg + 1];
  const uint64_t C = p.chunk, R = C * t.count;
  const uint64_t rounds = (o1 - o0 + R - 1) / R;  // the same in every CTA of the team
  const uint32_t step = kScanV * blockDim.x;
  Acc base_carry = 0;
  auto chunk = [&](uint64_t j, uint64_t* a, uint64_t* b) {
    const uint64_t a0 = o0 + j * R + C * t.rank;
    *a = a0 < o1 ? a0 : o1;
    *b = *a + C < o1 ? *a + C : o1;
  };
  uint64_t a = o0, b = o0;
  if (rounds && ok) {
    chunk(0, &a, &b);
    const Acc s = block_sum(slice_sum(in, a, b), buf);
    if (threadIdx.x == 0) partials[t.first + t.rank] = s;
    bar.arrive();
  }
  for (uint64_t j = 0; j < rounds && ok; ++j) {
    // split phase: the next round's chunk sum is read from HBM while this
    // round's barrier completes (a full barrier for the protocols without a
    // split form, still correct)
    uint64_t na = b, nb = b;
    Acc s_next = 0;
    if (j + 1 < rounds) {
      chunk(j + 1, &na, &nb);
      s_next = block_sum(slice_sum(in, na, nb), buf);
    }
    ok = bar.wait() && ok;
    if (!ok) break;
    // this round's sums of the team: before this CTA, and in total
    const Acc* part = partials + (j & 1) * gridDim.x + t.first;
    Acc pre = 0, tot = 0;
    for (uint32_t r = threadIdx.x; r < t.count; r += blockDim.x) {
      const Acc x = __ldcg(part + r);
      tot += x;
      if (r < t.rank) pre += x;
    }
    pre = block_sum(pre, buf);
    tot = block_sum(tot, buf);
    Acc c = base_carry + pre;
    for (uint64_t x = a; x < b; x += step) {
      const uint64_t left = b - x;
      const uint32_t n = left < step ? (uint32_t)left : step;
      c += scan_tile<T>(in, out, x, n, c, tile, wsum);
    }
    base_carry += tot;
    if (j + 1 < rounds) {
      // round j + 1's buffer held round j - 1's sums, which every CTA has read
      // before arriving at barrier j
      if (threadIdx.x == 0) partials[((j + 1) & 1) * gridDim.x + t.first + t.rank] = s_next;
      bar.arrive();
      a = na;
      b = nb;
    }
  }
  bar.finish();
}

// ---------------------------------------------------------------------------
// Register-resident scan of segments (cfg.form = GSRB_FORM_REG; fan-out
// sub-grid barrier).  The CTA's threads form NG groups that take the team's
// rounds in turn (group g: rounds g, g + NG, ...).  In a round every CTA of the
// team takes one chunk of GT x D x 4 elements (GT threads a group, D 128-bit
// vectors a lane), which the group loads once into registers, sums, publishes
// and -- after the segment's barrier of that round -- scans and writes from the
// same registers: no element is read twice and nothing waits in L2 between a
// read and a re-read.  While one group waits for its round's barrier the
// others load or write theirs.  Chunks sit on a vector grid anchored at the
// first position at or before the segment's start where `in` is 16-byte
// aligned, so whole vectors are loaded with 128-bit loads (the elements of a
// vector outside the segment read as zero and are not written); outputs go
// out as 128-bit stores when `out` has the same alignment as `in`, else as
// scalars.
//
// Ordering (every wait bounded):
//  * the group of round j arrives at j only after this CTA passed the barrier
//    of round j-1 (s_passed);
//  * the group of round j takes the team's running total from the group of
//    round j-1 (s_carry, sequence s_cseq) and hands on total + sum(j);
//  * round sums rotate over NG + 2 buffers of one word per CTA: the sum of
//    round j is written after this CTA passed j-1, so every CTA of the team
//    arrived at j-1, which its group of j-1 did after reading the sums of
//    j-1-NG and older; the last user of buffer j % (NG + 2) was j-NG-2;
//  * a group's control flow is uniform: its leader decides (s_gfail) before a
//    named barrier of the group that every thread of the group then passes.
constexpr uint32_t kRegMaxGroups = 4;  // named barriers 1..4

__device__ __forceinline__ void group_sync(uint32_t id, uint32_t nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Bounded wait for a shared counter written by another group of the CTA.
__device__ __forceinline__ bool group_wait_ge(const volatile uint32_t* p, uint32_t target,
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
        gsrb::detail::record_error(gb, gsrb::GSRB_DEV_TIMEOUT, 0xfffffff3u);
        return false;
      }
    }
  }
}

template <typename T> struct RegT;
template <> struct RegT<uint32_t> {
  using Vec = uint4;
  // read once: streaming (evict-first) loads and stores
  __device__ static __forceinline__ uint4 ld(const uint32_t* p) { return __ldcs(reinterpret_cast<const uint4*>(p)); }
  __device__ static __forceinline__ void st(uint32_t* p, uint4 v) { __stcs(reinterpret_cast<uint4*>(p), v); }
  // one lane's outputs: exclusive prefix before its first element e0 plus its
  // local inclusive prefixes a0..a2 (uint32 wraps: exact in any order)
  __device__ static __forceinline__ uint4 out(uint32_t e0, uint32_t a0, uint32_t a1, uint32_t a2) {
    return make_uint4(e0, e0 + a0, e0 + a1, e0 + a2);
  }
};
template <> struct RegT<float> {
  using Vec = float4;
  __device__ static __forceinline__ float4 ld(const float* p) { return __ldcs(reinterpret_cast<const float4*>(p)); }
  __device__ static __forceinline__ void st(float* p, float4 v) { __stcs(reinterpret_cast<float4*>(p), v); }
  // FP32: the FP64 prefix rounded once, the lane's local prefixes added in FP32
  __device__ static __forceinline__ float4 out(double e0, float a0, float a1, float a2) {
    const float b = (float)e0;
    return make_float4(b, b + a0, b + a1, b + a2);
  }
};

template <typename T>
__device__ __forceinline__ T shfl_up_t(T v, int o) { return __shfl_up_sync(0xffffffffu, v, o); }
template <typename T>
__device__ __forceinline__ T shfl_idx_t(T v, int l) { return __shfl_sync(0xffffffffu, v, l); }

template <typename T, int D, int MAXT>
__global__ void __launch_bounds__(MAXT, 1)
scan_segments_reg_kernel(SegParams p, const T* __restrict__ in, T* __restrict__ out,
                         typename ScanT<T>::Acc* __restrict__ partials, uint32_t ngroups) {
  using Acc = typename ScanT<T>::Acc;
  using Vec = typename RegT<T>::Vec;
  __shared__ gsrb::BarrierShared bsh;
  __shared__ Acc s_wt[kRegMaxGroups][32];  // warp totals -> exclusive warp offsets
  __shared__ Acc s_red[kRegMaxGroups][2][32];
  __shared__ Acc s_base[kRegMaxGroups];
  __shared__ uint32_t s_gfail[kRegMaxGroups];
  __shared__ volatile uint32_t s_passed, s_cseq, s_fail;
  __shared__ volatile Acc s_carry;
  __shared__ uint32_t s_epoch0;

  const uint32_t tid = threadIdx.x, lane = tid & 31u;
  const uint32_t NG = ngroups, GT = blockDim.x / NG, GW = GT >> 5;
  const uint32_t g = tid / GT, gt = tid - g * GT, gw = gt >> 5;
  const bool leader = gt == 0;
  const uint32_t NB = NG + 2;
  const uint64_t C = (uint64_t)GT * D * 4u;  // elements of one CTA's chunk
  const SegTeam t = seg_team(p);
  const gsrb::GridBarrier gb = seg_barrier(p, t);
  gsrb::GridSync<gsrb::V_FANOUT> bar;
  const bool ok0 = bar.init(gb, &bsh);
  if (tid == 0) {
    s_epoch0 = bar.epoch;
    s_passed = 0;
    s_cseq = 0;
    s_carry = Acc(0);
    s_fail = ok0 ? 0u : 1u;
  }
  __syncthreads();
  const uint32_t epoch0 = s_epoch0;
  const uint64_t o0 = p.off[t.seg], o1 = p.off[t.seg + 1];
  // Positions are relative to the vector grid's origin, lo (0..3) elements
  // before the segment's start, where `in` is 16-byte aligned: the segment is
  // [lo, hi), and relative position u is element o0 + (u - lo).
  const uint32_t ia = (uint32_t)((reinterpret_cast<uintptr_t>(in) >> 2) & 3u);
  const uint64_t lo = (o0 + ia) & 3u, hi = o1 - o0 + lo;
  const bool vec_in = (reinterpret_cast<uintptr_t>(in) & 3u) == 0;
  const bool vec_out = vec_in && (reinterpret_cast<uintptr_t>(out) & 3u) == 0 &&
                       ((reinterpret_cast<uintptr_t>(out) >> 2) & 3u) == ia;
  const uint64_t R = C * t.count;
  const uint32_t rounds = o1 > o0 ? (uint32_t)((hi + R - 1) / R) : 0u;
  const uint32_t me = t.rank;

  for (uint32_t j = g; j < rounds; j += NG) {
    // A. this group's chunk of round j into registers, and its sum
    const uint64_t cb = ((uint64_t)j * t.count + t.rank) * C;  // chunk base (relative, vector-aligned)
    const uint32_t v0 = gw * 32u * D + lane;
    Vec x[D];
#pragma unroll
    for (uint32_t k = 0; k < D; ++k) {
      const uint64_t u = cb + 4ull * (v0 + 32u * k);
      if (vec_in && u >= lo && u + 4 <= hi) {
        x[k] = RegT<T>::ld(in + o0 + (u - lo));
      } else {
        T y[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) y[q] = (u + q >= lo && u + q < hi) ? __ldg(in + o0 + (u + q - lo)) : T(0);
        x[k].x = y[0];
        x[k].y = y[1];
        x[k].z = y[2];
        x[k].w = y[3];
      }
    }
    Acc lsum = Acc(0);
#pragma unroll
    for (uint32_t k = 0; k < D; ++k) lsum += ScanT<T>::vsum(x[k]);
    const Acc wt = warp_sum(lsum);
    if (lane == 0) s_wt[g][gw] = wt;
    group_sync(1u + g, GT);
    // B. leader: warp offsets, the round's sum, arrival after j-1 was passed, barrier of j
    if (leader) {
      bool ok = s_fail == 0u;
      Acc run = Acc(0);
      for (uint32_t i = 0; i < GW; ++i) {
        const Acc y = s_wt[g][i];
        s_wt[g][i] = run;
        run += y;
      }
      if (ok && j > 0) ok = group_wait_ge(&s_passed, j, gb);
      if (ok) {
        __stcg(&partials[(j % NB) * gridDim.x + t.first + t.rank], run);
        gsrb::detail::fanout_arrive(gb, t.count, epoch0 + j);
        ok = gsrb::detail::fanout_wait(gb, me, epoch0 + j, j);
      }
      if (ok) {
        __threadfence_block();
        s_passed = j + 1u;
      } else {
        s_fail = 1u;
      }
      s_gfail[g] = ok ? 0u : 1u;
    }
    group_sync(1u + g, GT);
    if (s_gfail[g]) break;  // uniform: written by the leader before the group barrier
    // C. offset = running total + the round's sums of the CTAs before this one
    Acc pre = Acc(0), tot = Acc(0);
    const Acc* part = partials + (j % NB) * gridDim.x + t.first;
    for (uint32_t r = gt; r < t.count; r += GT) {
      const Acc y = __ldcg(part + r);
      tot += y;
      if (r < t.rank) pre += y;
    }
    pre = warp_sum(pre);
    tot = warp_sum(tot);
    if (lane == 0) {
      s_red[g][0][gw] = pre;
      s_red[g][1][gw] = tot;
    }
    group_sync(1u + g, GT);
    if (leader) {
      Acc pp = Acc(0), qq = Acc(0);
      for (uint32_t i = 0; i < GW; ++i) {
        pp += s_red[g][0][i];
        qq += s_red[g][1][i];
      }
      const bool ok = j == 0 || group_wait_ge(&s_cseq, j, gb);  // running total of rounds < j handed on
      const Acc cin = j == 0 ? Acc(0) : Acc(s_carry);
      s_base[g] = cin + pp;
      s_carry = cin + qq;
      __threadfence_block();
      s_cseq = j + 1u;
      if (!ok) s_fail = 1u;
      s_gfail[g] = ok ? 0u : 1u;
    }
    group_sync(1u + g, GT);
    if (s_gfail[g]) break;
    // D. scan the registers and write the segment's elements
    Acc run = s_base[g] + s_wt[g][gw];
#pragma unroll
    for (uint32_t k = 0; k < D; ++k) {
      const uint64_t u = cb + 4ull * (v0 + 32u * k);
      const Vec xv = x[k];
      const T a0 = xv.x, a1 = a0 + xv.y, a2 = a1 + xv.z, a3 = a2 + xv.w;
      T incl = a3;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const T y = shfl_up_t(incl, o);
        if ((int)lane >= o) incl += y;
      }
      const Vec y = RegT<T>::out(run + Acc(incl - a3), a0, a1, a2);
      if (vec_out && u >= lo && u + 4 <= hi) {
        RegT<T>::st(out + o0 + (u - lo), y);
      } else {
        const T ys[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
        for (int q = 0; q < 4; ++q)
          if (u + q >= lo && u + q < hi) out[o0 + (u + q - lo)] = ys[q];
      }
      run += Acc(shfl_idx_t(incl, 31));
    }
  }
  __syncthreads();
  bar.finish();
}

// 16 vectors a lane when an SM holds at most 512 of the launch's threads
// (about 128 registers a thread), else 8 (64 registers, 1024 threads an SM)
template <typename T>
const void* scan_segments_reg_fn(bool wide) {
  return wide ? (const void*)scan_segments_reg_kernel<T, 16, 512> : (const void*)scan_segments_reg_kernel<T, 8, 1024>;
}

const void* reduce_segments_fn(int v) {
  switch (v) {  // sub-grid protocols whose state does not depend on the team size
    case gsrb::V_FLAT: return (const void*)reduce_segments_kernel<gsrb::V_FLAT>;
    case gsrb::V_FLIP: return (const void*)reduce_segments_kernel<gsrb::V_FLIP>;
    case gsrb::V_FANOUT: return (const void*)reduce_segments_kernel<gsrb::V_FANOUT>;
    default: return nullptr;
  }
}

template <typename T>
const void* scan_segments_fn(int v) {
  switch (v) {
    case gsrb::V_FLAT: return (const void*)scan_segments_kernel<gsrb::V_FLAT, T>;
    case gsrb::V_FLIP: return (const void*)scan_segments_kernel<gsrb::V_FLIP, T>;
    case gsrb::V_FANOUT: return (const void*)scan_segments_kernel<gsrb::V_FANOUT, T>;
    default: return nullptr;
  }
}

// Shared checks and the launch parameters of a segmented call.
gsrb_status_t seg_setup(gsrb_ctx* ctx, const gsrb_cfg_t* cfgin, const uint64_t* h_off, int32_t k,
                        const void* (*pick)(int), int def_ctas, int def_threads, gsrb_cfg_t* c, int* grid,
                        const void** fn, SegParams* p) {
  if (!ctx || !h_off || k <= 0 || k > kMaxSegments) return GSRB_ERR_ARG;
  for (int32_t i = 0; i < k; ++i)
    if (h_off[i + 1] < h_off[i]) return GSRB_ERR_ARG;
  if (h_off[k] - h_off[0] >= (1ull << 47)) return GSRB_ERR_ARG;
  *c = resolve_cfg(ctx, cfgin);
  if (!cfgin) {
    c->variant = gsrb::V_FANOUT;
    c->ctas_per_sm = def_ctas;
    c->threads = def_threads;
  }
  c->cluster = 1;
  if (c->threads % 32 || c->threads > 1024 || c->threads < 64) return GSRB_ERR_ARG;
  *fn = pick(c->variant);
  if (!*fn) return GSRB_ERR_UNSUPPORTED;
  *grid = grid_of(ctx, *c);
  if (*grid < k || *grid > 65535) return GSRB_ERR_ARG;
  memset(p, 0, sizeof(*p));
  p->gb = make_barrier(ctx, *c, 1, 1u, 0u, 0u);
  p->flip_stride = (uint64_t)kMaxFlip * 32u;
  p->k = (uint32_t)k;
  // scan rounds: cfg->tile elements per CTA (rounded to whole tiles), 0 = 4 tiles
  const uint32_t tile_elems = kScanV * (uint32_t)c->threads;
  uint32_t chunk = c->tile > 0 ? (uint32_t)c->tile : 4u * tile_elems;
  chunk = (chunk + tile_elems - 1) / tile_elems * tile_elems;
  if (chunk > (1u << 24)) return GSRB_ERR_ARG;
  p->chunk = chunk;
  for (int32_t i = 0; i <= k; ++i) p->off[i] = h_off[i];
  return GSRB_OK;
}

template <typename T>
gsrb_status_t scan_segments(gsrb_ctx* ctx, const T* d_in, T* d_out, const uint64_t* h_off, int32_t k,
                            const gsrb_cfg_t* cfgin) {
  if (!h_off || (k > 0 && h_off[k] > h_off[0] && (!d_in || !d_out || d_in == d_out))) return GSRB_ERR_ARG;
  if (!ctx) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  gsrb_cfg_t c;
  int grid = 0;
  const void* fn = nullptr;
  SegParams p;
  gsrb_status_t st = seg_setup(ctx, cfgin, h_off, k, scan_segments_fn<T>, 4, 256, &c, &grid, &fn, &p);
  if (st) return st;
  using Acc = typename ScanT<T>::Acc;
  void* part = nullptr;
  if (!cfgin) c.form = GSRB_FORM_REG;  // default: fan-out, 4 x 256, two groups of 4096-element chunks
  if (c.form == GSRB_FORM_REG) {
    // register-resident rounds (fan-out sub-grid barrier only): cfg->tile =
    // elements of a CTA's chunk, threads x 4 x (16 vectors a lane when an
    // SM holds at most 512 of the launch's threads, else 8) divided by 2..4
    // groups (0 = two groups)
    if (c.variant != gsrb::V_FANOUT) return GSRB_ERR_UNSUPPORTED;
    const bool wide = c.threads * c.ctas_per_sm <= 512;
    const uint32_t per = (uint32_t)c.threads * (wide ? 16u : 8u) * 4u;
    uint32_t ng = 2;
    if (c.tile > 0) {
      if (per % (uint32_t)c.tile) return GSRB_ERR_ARG;
      ng = per / (uint32_t)c.tile;
    }
    if (ng < 2 || ng > kRegMaxGroups || (c.threads / ng) % 32) return GSRB_ERR_ARG;
    st = scratch(ctx, sizeof(Acc) * (kRegMaxGroups + 2) * (size_t)grid, &part);
    if (st) return st;
    Acc* partials = (Acc*)part;
    const void* rf = scan_segments_reg_fn<T>(wide);
    void* args[] = {&p, &d_in, &d_out, &partials, &ng};
    return launch_persistent(ctx, rf, grid, c.threads, 0, 1, coop_of(c), args);
  }
  st = scratch(ctx, sizeof(Acc) * 2 * (size_t)grid, &part);
  if (st) return st;
  Acc* partials = (Acc*)part;
  const uint32_t tw = kScanV * (uint32_t)c.threads;
  const size_t smem = sizeof(T) * (size_t)(tw + (tw >> 5));
  void* args[] = {&p, &d_in, &d_out, &partials};
  return launch_persistent(ctx, fn, grid, c.threads, smem, 1, coop_of(c), args);
}

}  // namespace

extern "C" {

gsrb_status_t gsrb_segments_layout(const uint64_t* h_off, int32_t k, int32_t grid, uint32_t* first, uint32_t* count) {
  if (!h_off || k <= 0 || k > kMaxSegments || grid < k) return GSRB_ERR_ARG;
  for (int32_t i = 0; i < k; ++i) {
    if (h_off[i + 1] < h_off[i]) return GSRB_ERR_ARG;
    const uint32_t f = seg_first(h_off, (uint32_t)k, (uint32_t)grid, (uint32_t)i);
    if (first) first[i] = f;
    if (count) count[i] = seg_first(h_off, (uint32_t)k, (uint32_t)grid, (uint32_t)i + 1) - f;
  }
  return GSRB_OK;
}

gsrb_status_t gsrb_reduce_i32_segments(gsrb_ctx_t ctx, const int32_t* d_in, const uint64_t* h_off, int32_t k,
                                       int64_t* d_out, const gsrb_cfg_t* cfgin) {
  if (!d_out || !h_off || (k > 0 && h_off[k] > h_off[0] && !d_in)) return GSRB_ERR_ARG;
  if (!ctx) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  gsrb_cfg_t c;
  int grid = 0;
  const void* fn = nullptr;
  SegParams p;
  gsrb_status_t st = seg_setup(ctx, cfgin, h_off, k, reduce_segments_fn, 2, 512, &c, &grid, &fn, &p);
  if (st) return st;
  void* part = nullptr;
  st = scratch(ctx, sizeof(long long) * (size_t)grid, &part);
  if (st) return st;
  long long* partials = (long long*)part;
  long long* out = (long long*)d_out;
  void* args[] = {&p, &d_in, &partials, &out};
  return launch_persistent(ctx, fn, grid, c.threads, 0, 1, coop_of(c), args);
}

gsrb_status_t gsrb_scan_u32_segments(gsrb_ctx_t ctx, const uint32_t* d_in, uint32_t* d_out, const uint64_t* h_off,
                                     int32_t k, const gsrb_cfg_t* cfgin) {
  return scan_segments<uint32_t>(ctx, d_in, d_out, h_off, k, cfgin);
}

gsrb_status_t gsrb_scan_f32_segments(gsrb_ctx_t ctx, const float* d_in, float* d_out, const uint64_t* h_off,
                                     int32_t k, const gsrb_cfg_t* cfgin) {
  return scan_segments<float>(ctx, d_in, d_out, h_off, k, cfgin);
}

}  // extern "C"
