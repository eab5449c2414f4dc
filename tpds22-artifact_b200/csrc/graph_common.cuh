// Shared device pieces of the persistent graph traversals (BFS, SSSP, PR):
// the device CSR view, warp-aggregated worklist appends, warp-synchronous
// frontier expansion with hub vertices split across the whole grid, the
// per-level trace record and the small MLP used by the learned policy.
//
// Reference structures restated: the CSRGraph layout
// (LONESTAR/rt/include/csr_graph.h.prehip:20-103), the two-slot worklists with
// warp-aggregated pushes (LONESTAR/rt/include/worklist.h.prehip:348-420,
// cutil_subset.h.prehip:43-48) and the nested-parallel edge expansion with
// thread / warp / thread-block granularity (internal.h.prehip:99-158,
// apps/bfs/kernel_gsrb.cu:400-553).
#pragma once
#include <stdint.h>
#include "gsrb/ptx.cuh"

namespace gsrbg {

constexpr int32_t kInf = 0x7fffffff;        // INF = INT_MAX (apps/bfs/kernel_gsrb.cu:295)
constexpr uint32_t kBigDegree = 4096;       // vertices above this are expanded by the whole grid
constexpr uint32_t kWarpDegree = 32;        // above this a warp expands the vertex cooperatively
constexpr uint32_t kPrHubDegree = 128;      // PageRank: above this a vertex's edges are cut into chunks
constexpr uint32_t kPrChunk = 2048;         // PageRank: edges per hub chunk (one warp each)
constexpr uint32_t kLbChunk = 256;          // load-balanced BFS: edges per warp chunk
constexpr uint32_t kLbMaxCtas = 8192;       // load-balanced BFS: largest team (per-CTA totals)
constexpr unsigned long long kLbMinEdges = 65536;  // load-balanced BFS: smaller push levels expand as usual

struct DevCSR {
  uint32_t n;
  uint32_t m;
  const uint32_t* __restrict__ row;  // n + 1
  const uint32_t* __restrict__ dst;  // m
  const int32_t* __restrict__ w;     // m (may be null for BFS / PR)
};

// One record per level / bucket step, written by CTA 0 after the barrier.
struct LevelTrace {
  uint32_t level;
  uint32_t dir;          // 0 push-worklist, 1 pull, 2 push-topology, 3 push by a single CTA
  uint32_t nf;           // frontier vertices entering this level
  uint32_t nu;           // unvisited vertices before this level
  unsigned long long mf; // frontier out-edges
  unsigned long long mu; // out-edges of unvisited vertices
  unsigned long long t_ns;  // %globaltimer when the level started
  float pred;            // policy's predicted log2(1 + next nf) (NaN if none)
  uint32_t fallback;     // 1 once the policy fell back to the heuristic
};
static_assert(sizeof(LevelTrace) == 48, "trace layout");

// Per-level counters (three rotating sets; see the BFS kernel for the protocol).
struct LevelCounters {
  unsigned long long n_reg;   // regular-queue appends
  unsigned long long n_big;   // hub-queue appends
  unsigned long long m_next;  // out-edges of appended vertices
  unsigned long long n_real;  // BFS: regular entries (n_reg counts slots, reservation holes included)
};

// The CTAs working on one traversal: the whole grid for a single traversal, a
// contiguous CTA range (with its own sub-grid barrier) for one instance of a
// batch.  All work distribution is relative to the team.
struct Team {
  uint32_t cta;   // this CTA's index in the team
  uint32_t ncta;  // CTAs in the team
  __device__ __forceinline__ uint32_t tid() const { return cta * blockDim.x + threadIdx.x; }
  __device__ __forceinline__ uint32_t nthreads() const { return ncta * blockDim.x; }
  __device__ __forceinline__ uint32_t warp() const { return tid() >> 5; }
  __device__ __forceinline__ uint32_t nwarps() const { return nthreads() >> 5; }
};

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp-aggregated append of `v` (where `pred`) to queue q with counter *cnt.
// Must be called by all 32 lanes (warp-synchronous).  Returns nothing; the
// queue capacity is checked by the caller's sizing (<= n distinct vertices).
template <class T>
__device__ __forceinline__ void warp_append(bool pred, T v, T* q, unsigned long long* cnt, uint32_t cap,
                                            uint32_t* overflow) {
  const uint32_t mask = __ballot_sync(0xffffffffu, pred);
  if (!mask) return;
  const uint32_t leader = __ffs(mask) - 1;
  unsigned long long base = 0;
  if (lane_id() == leader) base = atomicAdd(cnt, (unsigned long long)__popc(mask));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (pred) {
    const unsigned long long pos = base + __popc(mask & lanemask_lt());
    if (pos < cap) q[pos] = v;
    else atomicExch(overflow, 1u);
  }
}

// Warp-aggregated append of up to K values per lane (v[r] where pred[r]) with
// ONE reservation on the counter for the whole warp: the K appends of a lane
// step cost one atomic round trip instead of K.  Warp-synchronous.
template <int K, class T>
__device__ __forceinline__ void warp_append_k(const bool* pred, const T* v, T* q, unsigned long long* cnt,
                                              uint32_t cap, uint32_t* overflow) {
  uint32_t mask[K];
  uint32_t tot = 0;
#pragma unroll
  for (int r = 0; r < K; ++r) {
    mask[r] = __ballot_sync(0xffffffffu, pred[r]);
    tot += __popc(mask[r]);
  }
  if (!tot) return;
  unsigned long long base = 0;
  if (lane_id() == 0) base = atomicAdd(cnt, (unsigned long long)tot);
  base = __shfl_sync(0xffffffffu, base, 0);
  const uint32_t lt = lanemask_lt();
#pragma unroll
  for (int r = 0; r < K; ++r) {
    if (pred[r]) {
      const unsigned long long pos = base + __popc(mask[r] & lt);
      if (pos < cap) q[pos] = v[r];
      else atomicExch(overflow, 1u);
    }
    base += __popc(mask[r]);
  }
}

// Queue slots reserved by a warp in chunks: one atomic on the shared counter
// per chunk instead of one per warp step (every warp of a large round appends
// at almost every step, and those atomics serialise on one L2 line).  Slots a
// warp reserved but did not fill hold kHole, which readers skip; a queue then
// holds at most (chunk - 1) holes per warp more than its entries.
constexpr uint32_t kHole = 0xffffffffu;
struct WarpRes {
  unsigned long long base;  // next reserved slot (warp-uniform)
  uint32_t left;            // reserved slots not yet filled
  uint32_t chunk;           // slots per reservation (0: no reservation, append directly)
};

template <int K, class T>
__device__ __forceinline__ uint32_t warp_append_res(const bool* pred, const T* v, T* q, unsigned long long* cnt,
                                                    uint32_t cap, uint32_t* overflow, WarpRes& res, T hole) {
  uint32_t mask[K];
  uint32_t tot = 0;
#pragma unroll
  for (int r = 0; r < K; ++r) {
    mask[r] = __ballot_sync(0xffffffffu, pred[r]);
    tot += __popc(mask[r]);
  }
  if (!tot) return 0;
  if (tot > res.left) {
    for (uint32_t i = lane_id(); i < res.left; i += 32) {
      const unsigned long long pos = res.base + i;
      if (pos < cap) q[pos] = hole;
    }
    const uint32_t want = tot > res.chunk ? tot : res.chunk;
    unsigned long long b = 0;
    if (lane_id() == 0) b = atomicAdd(cnt, (unsigned long long)want);
    res.base = __shfl_sync(0xffffffffu, b, 0);
    res.left = want;
  }
  const uint32_t lt = lanemask_lt();
  unsigned long long base = res.base;
#pragma unroll
  for (int r = 0; r < K; ++r) {
    if (pred[r]) {
      const unsigned long long pos = base + __popc(mask[r] & lt);
      if (pos < cap) q[pos] = v[r];
      else atomicExch(overflow, 1u);
    }
    base += __popc(mask[r]);
  }
  res.base = base;
  res.left -= tot;
  return tot;
}

// Fills the warp's unused reserved slots with holes (end of a round).
template <class T>
__device__ __forceinline__ void warp_res_close(T* q, uint32_t cap, WarpRes& res, T hole) {
  for (uint32_t i = lane_id(); i < res.left; i += 32) {
    const unsigned long long pos = res.base + i;
    if (pos < cap) q[pos] = hole;
  }
  res.left = 0;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return __shfl_sync(0xffffffffu, v, 0);
}
__device__ __forceinline__ uint32_t warp_max_u32(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Expand the regular queue q[0, nq): calls f(u, edge_index) warp-synchronously
// (every lane calls f in every step, with `active` telling whether the lane has
// an edge).  Vertices of degree <= kWarpDegree: one lane each; larger: the warp
// strides over the edges together.  Warps take 32-vertex groups grid-stride.
template <class F>
__device__ __forceinline__ void expand_queue(const Team& t, const DevCSR& g, const uint32_t* __restrict__ q,
                                             uint32_t nq, F& f) {
  const uint32_t lane = lane_id();
  const uint32_t gw = t.warp();
  const uint32_t nwarps = t.nwarps();
  for (uint32_t base = gw * 32u; base < nq; base += nwarps * 32u) {
    const uint32_t i = base + lane;
    uint32_t u = 0, b = 0, e = 0;
    if (i < nq) {
      u = __ldcg(q + i);
      b = __ldg(g.row + u);
      e = __ldg(g.row + u + 1);
    }
    const uint32_t deg = e - b;
    // warp-cooperative vertices
    uint32_t coop = __ballot_sync(0xffffffffu, deg > kWarpDegree);
    while (coop) {
      const int src = __ffs(coop) - 1;
      coop &= coop - 1;
      const uint32_t uu = __shfl_sync(0xffffffffu, u, src);
      const uint32_t bb = __shfl_sync(0xffffffffu, b, src);
      const uint32_t ee = __shfl_sync(0xffffffffu, e, src);
      for (uint32_t j0 = bb; j0 < ee; j0 += 32) {
        const uint32_t j = j0 + lane;
        f(uu, j, j < ee);
      }
    }
    // lane-per-vertex for the small ones
    const uint32_t mine = deg <= kWarpDegree ? deg : 0u;
    const uint32_t kmax = warp_max_u32(mine);
    for (uint32_t k = 0; k < kmax; ++k) f(u, b + k, k < mine);
  }
}

// BFS frontier queues hold each vertex's edge range {row[v], row[v+1]} instead
// of v (the discoverer has loaded both to learn the degree anyway), so a level
// starts on its edges without first looking the rows up: one dependent round
// trip less per level.  Queues of n entries, 8 bytes each.
//
// Expand a range queue q[0, nq): ranges of more than kWarpDegree edges are
// walked by the whole warp, calling f(0, edge, active) warp-synchronously; the
// rest go to `lanes(b, mine, kmax)`, called by all 32 lanes once per 32-entry
// group with the lane's first edge b, its edge count `mine` (0 for the warp's
// ranges) and the warp's largest count, so that the callee can keep several of
// a lane's edges in flight.
template <class F, class FL>
__device__ __forceinline__ void expand_range_queue(const Team& t, const uint2* __restrict__ q, uint32_t nq, F& f,
                                                   FL& lanes) {
  const uint32_t lane = lane_id();
  const uint32_t gw = t.warp();
  const uint32_t nwarps = t.nwarps();
  for (uint32_t base = gw * 32u; base < nq; base += nwarps * 32u) {
    const uint32_t i = base + lane;
    uint32_t b = 0, e = 0;
    if (i < nq) {
      const uint2 r = __ldcg(q + i);
      b = r.x;
      e = r.y;
    }
    const uint32_t deg = e - b;
    uint32_t coop = __ballot_sync(0xffffffffu, deg > kWarpDegree);
    while (coop) {
      const int src = __ffs(coop) - 1;
      coop &= coop - 1;
      const uint32_t bb = __shfl_sync(0xffffffffu, b, src);
      const uint32_t ee = __shfl_sync(0xffffffffu, e, src);
      for (uint32_t j0 = bb; j0 < ee; j0 += 32) {
        const uint32_t j = j0 + lane;
        f(0u, j, j < ee);
      }
    }
    const uint32_t mine = deg <= kWarpDegree ? deg : 0u;
    lanes(b, mine, warp_max_u32(mine));
  }
}

// Expand a queue of hub ranges: every CTA takes an equal slice of every hub.
template <class F>
__device__ __forceinline__ void expand_hub_ranges(const Team& t, const uint2* __restrict__ hq, uint32_t nh, F& f) {
  const uint32_t G = t.ncta;
  for (uint32_t k = 0; k < nh; ++k) {
    const uint2 r = __ldcg(hq + k);
    const uint64_t len = r.y - r.x;
    const uint32_t s0 = r.x + (uint32_t)(len * t.cta / G);
    const uint32_t s1 = r.x + (uint32_t)(len * (t.cta + 1) / G);
    for (uint32_t j0 = s0 + (threadIdx.x & ~31u); j0 < s1; j0 += blockDim.x) {
      const uint32_t j = j0 + lane_id();
      f(0u, j, j < s1);
    }
  }
}

// Where a BFS push step puts the vertices it discovers (as edge ranges).
struct PushSink {
  uint2* qout;                 // regular queue of the next level
  uint2* hout;                 // hub queue of the next level
  unsigned long long* n_reg;   // their counters (global, or shared in the one-CTA phase)
  unsigned long long* n_big;
  uint32_t cap;
  uint32_t* overflow;
  WarpRes* res;                // regular-queue reservation (null: append directly)
  uint32_t* real;              // regular entries appended by this warp (with res)
  uint32_t rcap;               // regular-queue slots (with res)
};

// Appends the regular entries of a push step: through the warp's reservation
// when there is one (counting the entries), else directly.
template <int K>
__device__ __forceinline__ void push_append_reg(const bool* reg, const uint2* rg, const PushSink& s) {
  if (s.res && s.res->chunk) {
    *s.real += warp_append_res<K>(reg, rg, s.qout, s.n_reg, s.rcap, s.overflow, *s.res, make_uint2(0u, 0u));
  } else {
    if (s.real) {
      uint32_t tot = 0;
#pragma unroll
      for (int r = 0; r < K; ++r) tot += __popc(__ballot_sync(0xffffffffu, reg[r]));
      *s.real += tot;
    }
    warp_append_k<K>(reg, rg, s.qout, s.n_reg, s.cap, s.overflow);
  }
}

// Frontiers up to this size check a destination's level only through the
// claim itself (compare-and-swap INF -> L) and load its row range alongside
// the claim; larger ones read the level first and load rows only for claimed
// vertices (throughput over latency).
constexpr uint32_t kPushPrecheckFrontier = 16384;

// BFS push of four edges per lane at once: edge r of the lane is j[r] (where
// bit r of `act` is set).  The four destinations are loaded together, their
// claims (compare-and-swap INF -> L) are issued together (with the row ranges
// of the candidates, or after a level check when `precheck`), and the warp
// reserves queue space once per step for all of them.  Levels are the same as
// with one edge at a time (a vertex gets L from whichever claim lands first);
// only the order of the next queue differs.  Warp-synchronous.
__device__ __forceinline__ void bfs_push4e(const DevCSR& g, int32_t* level, int32_t Li, const uint32_t* j,
                                           uint32_t act, bool precheck, const PushSink& s,
                                           unsigned long long& m_acc) {
  uint32_t v[4];
  uint32_t live = act;
#pragma unroll
  for (int r = 0; r < 4; ++r) v[r] = ((live >> r) & 1u) ? __ldg(g.dst + j[r]) : 0u;
  uint2 rg[4];
  if (precheck) {
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (((live >> r) & 1u) && __ldcg(level + v[r]) != kInf) live &= ~(1u << r);
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (((live >> r) & 1u) && atomicCAS(level + v[r], kInf, Li) != kInf) live &= ~(1u << r);
#pragma unroll
    for (int r = 0; r < 4; ++r)
      rg[r] = ((live >> r) & 1u) ? make_uint2(__ldg(g.row + v[r]), __ldg(g.row + v[r] + 1)) : make_uint2(0u, 0u);
  } else {
#pragma unroll
    for (int r = 0; r < 4; ++r)
      rg[r] = ((live >> r) & 1u) ? make_uint2(__ldg(g.row + v[r]), __ldg(g.row + v[r] + 1)) : make_uint2(0u, 0u);
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if (((live >> r) & 1u) && atomicCAS(level + v[r], kInf, Li) != kInf) live &= ~(1u << r);
  }
  bool reg[4], big[4];
  bool any_big = false;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const uint32_t d = ((live >> r) & 1u) ? rg[r].y - rg[r].x : 0u;
    reg[r] = ((live >> r) & 1u) && d <= kBigDegree;
    big[r] = ((live >> r) & 1u) && d > kBigDegree;
    any_big |= big[r];
    m_acc += d;
  }
  push_append_reg<4>(reg, rg, s);
  if (__any_sync(0xffffffffu, any_big)) warp_append_k<4>(big, rg, s.hout, s.n_big, s.cap, s.overflow);
}

// BFS push over the lane-per-vertex edges of a 32-entry group, four edges per
// lane in flight: the four destinations are loaded together, their claims are
// issued together (with the row ranges of the candidates, or after a level
// check when `precheck`), and the warp reserves queue space once per step for
// all of them.  Small frontiers thus cost three dependent round trips per four
// edges (destination, claim and rows, reservation) instead of five per edge.
// Levels are the same as with one edge at a time (a vertex gets L from
// whichever claim lands first); only the order of the next queue differs.
// Warp-synchronous.  (bfs_push4e does the same for arbitrary edge indices; this
// contiguous form keeps fewer registers live in the level loop.)
__device__ __forceinline__ void bfs_push_lanes(const DevCSR& g, int32_t* level, int32_t Li, uint32_t b,
                                               uint32_t mine, uint32_t kmax, bool precheck, const PushSink& s,
                                               unsigned long long& m_acc) {
  for (uint32_t k0 = 0; k0 < kmax; k0 += 4) {
    uint32_t v[4];
    uint32_t live = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      v[r] = 0;
      if (k0 + r < mine) {
        v[r] = __ldg(g.dst + b + k0 + r);
        live |= 1u << r;
      }
    }
    uint2 rg[4];
    if (precheck) {
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (((live >> r) & 1u) && __ldcg(level + v[r]) != kInf) live &= ~(1u << r);
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (((live >> r) & 1u) && atomicCAS(level + v[r], kInf, Li) != kInf) live &= ~(1u << r);
#pragma unroll
      for (int r = 0; r < 4; ++r)
        rg[r] = ((live >> r) & 1u) ? make_uint2(__ldg(g.row + v[r]), __ldg(g.row + v[r] + 1)) : make_uint2(0u, 0u);
    } else {
#pragma unroll
      for (int r = 0; r < 4; ++r)
        rg[r] = ((live >> r) & 1u) ? make_uint2(__ldg(g.row + v[r]), __ldg(g.row + v[r] + 1)) : make_uint2(0u, 0u);
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (((live >> r) & 1u) && atomicCAS(level + v[r], kInf, Li) != kInf) live &= ~(1u << r);
    }
    bool reg[4], big[4];
    bool any_big = false;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint32_t d = ((live >> r) & 1u) ? rg[r].y - rg[r].x : 0u;
      reg[r] = ((live >> r) & 1u) && d <= kBigDegree;
      big[r] = ((live >> r) & 1u) && d > kBigDegree;
      any_big |= big[r];
      m_acc += d;
    }
    push_append_reg<4>(reg, rg, s);
    if (__any_sync(0xffffffffu, any_big)) warp_append_k<4>(big, rg, s.hout, s.n_big, s.cap, s.overflow);
  }
}

// Largest i in [0, cnt) with p[i] <= t (p non-decreasing, p[0] <= t).
__device__ __forceinline__ uint32_t list_owner(const uint32_t* p, uint32_t cnt, uint32_t t) {
  uint32_t lo = 0, hi = cnt;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (p[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Hub queues up to this long are expanded edge-balanced over the whole team
// (each CTA builds the hubs' edge prefix in shared memory, no barrier needed);
// longer ones fall back to every CTA taking a slice of every hub in turn.
constexpr uint32_t kHubList = 2048;

// Shared-memory lists of the edge-balanced tiers (one instance per CTA, shared
// by every traversal kernel that inlines them): edge prefix, first edges,
// source distances (SSSP), and scan scratch.
struct ListSmem {
  uint32_t p[kHubList + 1];
  uint32_t b[kHubList];
  int32_t d[kHubList];
  uint32_t scan[32];
};
__device__ __forceinline__ ListSmem& list_smem() {
  __shared__ ListSmem s;
  return s;
}

// BFS push of a list of ranges, edge-balanced: prefix p[0..cnt] and first edges
// b[] in shared memory; thread x of nthr takes edges (x & ~31) + lane + k * nthr,
// four per step, each finding its range by binary search.  Warp-synchronous.
__device__ __forceinline__ void bfs_push_list(const DevCSR& g, int32_t* level, int32_t Li, const uint32_t* p,
                                              const uint32_t* b, uint32_t cnt, uint32_t x, uint32_t nthr,
                                              const PushSink& s, unsigned long long& m_acc) {
  const uint32_t total = p[cnt];
  for (uint32_t t0 = (x & ~31u) + lane_id(); t0 - lane_id() < total; t0 += 4u * nthr) {
    uint32_t j[4];
    uint32_t act = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint32_t t = t0 + (uint32_t)r * nthr;
      j[r] = 0;
      if (t < total) {
        const uint32_t o = list_owner(p, cnt, t);
        j[r] = b[o] + (t - p[o]);
        act |= 1u << r;
      }
    }
    bfs_push4e(g, level, Li, j, act, true, s, m_acc);
  }
}

// Expand the hub queue: every CTA takes an equal slice of every hub's edges.
template <class F>
__device__ __forceinline__ void expand_hubs(const Team& t, const DevCSR& g, const uint32_t* __restrict__ hq,
                                            uint32_t nh, F& f) {
  const uint32_t G = t.ncta;
  for (uint32_t k = 0; k < nh; ++k) {
    const uint32_t u = __ldcg(hq + k);
    const uint32_t b = __ldg(g.row + u), e = __ldg(g.row + u + 1);
    const uint64_t len = e - b;
    const uint32_t s0 = b + (uint32_t)(len * t.cta / G);
    const uint32_t s1 = b + (uint32_t)(len * (t.cta + 1) / G);
    // warp-synchronous strides of the CTA over its slice
    for (uint32_t j0 = s0 + (threadIdx.x & ~31u); j0 < s1; j0 += blockDim.x) {
      const uint32_t j = j0 + lane_id();
      f(u, j, j < s1);
    }
  }
}

// ---------------------------------------------------------------- MLP -------
// 12 -> 32 -> 32 -> 4 fully connected, ReLU; outputs: [0] logit(pull), [1]
// logit(topology push), [2] predicted log2(1 + next frontier size), [3] spare.
constexpr int kFeat = 12, kHid = 32, kOut = 4;
struct MLPWeights {
  float w1[kHid][kFeat];
  float b1[kHid];
  float w2[kHid][kHid];
  float b2[kHid];
  float w3[kOut][kHid];
  float b3[kOut];
};

// Warp-cooperative forward pass (lane j computes hidden unit j); every lane
// returns the 4 outputs.  Deterministic: same inputs give the same outputs in
// every CTA, so every CTA takes the same decision without communicating.
__device__ __forceinline__ void mlp_forward_warp(const MLPWeights* __restrict__ W, const float* feat, float out[kOut]) {
  const uint32_t j = lane_id();
  float h1 = W->b1[j];
#pragma unroll
  for (int i = 0; i < kFeat; ++i) h1 = fmaf(W->w1[j][i], feat[i], h1);
  h1 = fmaxf(h1, 0.f);
  float h2 = W->b2[j];
#pragma unroll
  for (int i = 0; i < kHid; ++i) h2 = fmaf(W->w2[j][i], __shfl_sync(0xffffffffu, h1, i), h2);
  h2 = fmaxf(h2, 0.f);
#pragma unroll
  for (int o = 0; o < kOut; ++o) {
    float p = W->w3[o][j] * h2;
#pragma unroll
    for (int s = 16; s > 0; s >>= 1) p += __shfl_xor_sync(0xffffffffu, p, s);
    out[o] = p + W->b3[o];
  }
}

// The same network staged in shared memory, weights transposed so that lane j
// reads column j of every layer without bank conflicts.  Filled once per CTA
// (mlp_stage) and evaluated by one warp per level (mlp_forward_smem), with the
// additions in the same order as mlp_forward_warp.
struct MLPShared {
  float w1t[kFeat][kHid];
  float b1[kHid];
  float w2t[kHid][kHid];
  float b2[kHid];
  float w3[kOut][kHid];
  float b3[kOut];
  float h1[kHid];
};

__device__ __forceinline__ void mlp_stage(const MLPWeights* __restrict__ W, MLPShared* m) {
  for (uint32_t i = threadIdx.x; i < kFeat * kHid; i += blockDim.x) m->w1t[i % kFeat][i / kFeat] = W->w1[i / kFeat][i % kFeat];
  for (uint32_t i = threadIdx.x; i < kHid * kHid; i += blockDim.x) m->w2t[i % kHid][i / kHid] = W->w2[i / kHid][i % kHid];
  for (uint32_t i = threadIdx.x; i < kOut * kHid; i += blockDim.x) m->w3[i / kHid][i % kHid] = W->w3[i / kHid][i % kHid];
  for (uint32_t i = threadIdx.x; i < kHid; i += blockDim.x) {
    m->b1[i] = W->b1[i];
    m->b2[i] = W->b2[i];
  }
  for (uint32_t i = threadIdx.x; i < kOut; i += blockDim.x) m->b3[i] = W->b3[i];
}

// One warp; every lane returns the 4 outputs.
__device__ __forceinline__ void mlp_forward_smem(MLPShared* m, const float* feat, float out[kOut]) {
  const uint32_t j = lane_id();
  float h1 = m->b1[j];
#pragma unroll
  for (int i = 0; i < kFeat; ++i) h1 = fmaf(m->w1t[i][j], feat[i], h1);
  h1 = fmaxf(h1, 0.f);
  m->h1[j] = h1;
  __syncwarp();
  float h2 = m->b2[j];
#pragma unroll
  for (int i = 0; i < kHid; ++i) h2 = fmaf(m->w2t[i][j], m->h1[i], h2);
  h2 = fmaxf(h2, 0.f);
  __syncwarp();  // h1 may be rewritten by the next call
  float p[kOut];
#pragma unroll
  for (int o = 0; o < kOut; ++o) p[o] = m->w3[o][j] * h2;
#pragma unroll
  for (int sft = 16; sft > 0; sft >>= 1)
#pragma unroll
    for (int o = 0; o < kOut; ++o) p[o] += __shfl_xor_sync(0xffffffffu, p[o], sft);
#pragma unroll
  for (int o = 0; o < kOut; ++o) out[o] = p[o] + m->b3[o];
}

// Feature vector of a level (all log-scaled or normalised to O(1)).  The same
// function builds training rows on the host from trace records.
__host__ __device__ __forceinline__ void level_features(float feat[kFeat], uint32_t n, uint32_t m, uint32_t level,
                                               uint32_t nf, unsigned long long mf, uint32_t nu,
                                               unsigned long long mu, uint32_t prev_nf, uint32_t prev_dir) {
  feat[0] = log2f(1.f + (float)nf);
  feat[1] = log2f(1.f + (float)mf);
  feat[2] = log2f(1.f + (float)nu);
  feat[3] = log2f(1.f + (float)mu);
  feat[4] = (float)nf / (float)(n ? n : 1);
  feat[5] = (float)((double)mf / (double)(mu + 1));
  feat[6] = log2f(1.f + (float)((double)mf / (double)(nf ? nf : 1)));  // mean frontier degree
  feat[7] = log2f(1.f + (float)level);
  feat[8] = (float)prev_dir;
  feat[9] = log2f((float)(n ? n : 1));
  feat[10] = log2f(1.f + (float)m) - log2f((float)(n ? n : 1));  // log mean degree
  feat[11] = log2f(1.f + (float)nf) - log2f(1.f + (float)prev_nf);  // growth
}

}  // namespace gsrbg
