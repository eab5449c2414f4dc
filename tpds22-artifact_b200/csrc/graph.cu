// Persistent Lonestar-style graph traversals on the grid barrier: BFS (push
// worklist, pull, topology push; direction chosen per level by a fixed
// heuristic or by the learned policy), SSSP (near-far buckets with atomicMin)
// and pull PageRank (FP32 state, FP64 per-vertex accumulation, fixed
// iteration count).  One kernel launch per traversal; one grid barrier per
// level / bucket step / iteration.
//
// Reference: the GGC "outlined iterate" kernels gg_main_pipe_1_gpu_gb of
// LONESTAR/apps/bfs/kernel_gsrb.cu:591-626 (BFS), apps/sssp/kernel_gsrb.cu:637-687
// (SSSP, DELTA default 10000, apps/sssp/support.cu:10), apps/pr/kernel_gsrb.cu:543-587
// (push-residual PR), all launched as one persistent kernel that hits
// kernelAtomicTreeBarrierUniqSRB once per level.  Level and distance
// conventions: source 0, unreachable INT_MAX, BFS level L for vertices first
// reached in round L (bfs/kernel_gsrb.cu:299-311, :473-479, :724).
#include "internal.h"
#include "graph_common.cuh"

#include <algorithm>
#include <string.h>
#include <utility>
#include <vector>

using namespace gsrbrt;
using namespace gsrbg;

namespace {

enum BfsDir : uint32_t { DIR_PUSH = 0, DIR_PULL = 1, DIR_TOPO = 2 };

struct BfsArgs {
  DevCSR g;
  uint32_t src;
  int32_t* level;
  uint32_t* q[2];
  uint32_t* hq[2];
  LevelCounters* cnt;  // [3]
  uint32_t* overflow;
  LevelTrace* trace;
  uint32_t trace_cap;
  const MLPWeights* mlp;
  int32_t mode;        // GSRB_BFS_* (include/gsrb.h)
  float alpha, beta;   // direction-optimizing thresholds (Beamer, Asanovic, Patterson, SC'12)
  uint32_t* out;       // [0] levels, [1] fallback level (0 = none), [2] policy decisions, [3] overflow
  unsigned long long* out_edges;
  uint32_t* solo;      // [0] last level, [1] nu, [2] prev_nf, [3] solo levels, [4..5] mu, [6..7] edges
  bool symmetric;      // rows are also in-edge lists: pull levels allowed
  bool lb;             // load-balanced expansion of large push levels (GSRB_BFS_FLAG_LB)
  uint32_t* lb_pre;    // [n] edge offset of each regular-queue entry
  uint32_t* lb_own;    // [m / kLbChunk + 2] entry owning each chunk's first edge
  uint32_t* lb_part;   // [kLbMaxCtas] per-CTA edge totals
};

// Single-CTA phase: when a push level's frontier fits one pass of one CTA
// (<= blockDim.x vertices and <= 4 blockDim.x out-edges) the heuristic and
// learned schedules hand the following levels to the team's first CTA, which
// runs them with __syncthreads and shared-memory queue counters while the
// other CTAs wait at one grid barrier; it hands back when the frontier grows
// past 2x the entry limits, after kSoloMaxLevels levels, or when the traversal
// ends.  Small-frontier levels of high-diameter graphs (meshes, road
// networks) then cost no grid barrier.
constexpr uint32_t kSoloMaxLevels = 16384;
// The policy's topology-push output must exceed this logit (probability 0.88).
constexpr float kTopoLogit = 2.f;

// The single-CTA phase, run by every thread of the team's first CTA from level
// L (whose frontier, nreg + nbig vertices of level L-1, is in the global
// queues; the caller has already done level L's accounting).  Leaves the
// frontier of the last level it ran in the global queues and counters, and
// that level, nu, mu, edges and prev_nf (accounting not yet applied for the
// last level's discoveries, as the level loop expects) in a.solo.
__device__ __noinline__ void bfs_solo(const BfsArgs& a, uint32_t L, uint32_t nreg, uint32_t nbig, uint32_t nu,
                                      unsigned long long mu, unsigned long long edges, uint32_t prev_nf) {
  __shared__ LevelCounters s_c;
  const DevCSR& g = a.g;
  const Team one{0u, 1u};
  uint32_t levels = 0;
  for (;;) {
    const uint2* qin = reinterpret_cast<const uint2*>(a.q[(L - 1) & 1]);
    const uint2* hin = reinterpret_cast<const uint2*>(a.hq[(L - 1) & 1]);
    uint2* qout = reinterpret_cast<uint2*>(a.q[L & 1]);
    uint2* hout = reinterpret_cast<uint2*>(a.hq[L & 1]);
    if (threadIdx.x == 0) {
      s_c.n_reg = 0;
      s_c.n_big = 0;
      s_c.m_next = 0;
    }
    __syncthreads();
    unsigned long long m_acc = 0;
    const int32_t Li = (int32_t)L;
    auto push_edge = [&](uint32_t, uint32_t j, bool active) {
      uint2 r = make_uint2(0u, 0u);
      bool disc = false;
      if (active) {
        const uint32_t v = __ldg(g.dst + j);
        if (__ldcg(a.level + v) == kInf) disc = atomicCAS(a.level + v, kInf, Li) == kInf;
        if (disc) r = make_uint2(__ldg(g.row + v), __ldg(g.row + v + 1));
      }
      const uint32_t d = r.y - r.x;
      warp_append(disc && d <= kBigDegree, r, qout, &s_c.n_reg, g.n, a.overflow);
      warp_append(disc && d > kBigDegree, r, hout, &s_c.n_big, g.n, a.overflow);
      m_acc += d;
    };
    expand_hub_ranges(one, hin, nbig, push_edge);
    const PushSink sink{qout, hout, &s_c.n_reg, &s_c.n_big, g.n, a.overflow, nullptr, nullptr, 0u};
    auto lanes = [&](uint32_t b, uint32_t mine, uint32_t kmax) {
      bfs_push_lanes(g, a.level, Li, b, mine, kmax, false, sink, m_acc);
    };
    expand_range_queue(one, qin, nreg, push_edge, lanes);
    const unsigned long long ws = warp_sum_u64(m_acc);
    if (lane_id() == 0 && ws) atomicAdd(&s_c.m_next, ws);
    __syncthreads();
    ++levels;
    const uint32_t nr = (uint32_t)s_c.n_reg, nb = (uint32_t)s_c.n_big;
    const uint32_t nf = nr + nb;
    const unsigned long long mf = s_c.m_next;
    const bool stop = nf == 0 || nf > 2u * blockDim.x || mf > 8ull * blockDim.x || levels >= kSoloMaxLevels;
    if (stop) {
      if (threadIdx.x == 0) {
        a.cnt[L % 3].n_reg = nr;
        a.cnt[L % 3].n_real = nr;
        a.cnt[L % 3].n_big = nb;
        a.cnt[L % 3].m_next = mf;
        a.cnt[(L + 1) % 3].n_reg = 0;
        a.cnt[(L + 1) % 3].n_real = 0;
        a.cnt[(L + 1) % 3].n_big = 0;
        a.cnt[(L + 1) % 3].m_next = 0;
        a.solo[0] = L;
        a.solo[1] = nu;
        a.solo[2] = prev_nf;
        a.solo[3] += levels;
        *reinterpret_cast<unsigned long long*>(a.solo + 4) = mu;
        *reinterpret_cast<unsigned long long*>(a.solo + 6) = edges;
      }
      return;  // the caller's grid barrier publishes all of it
    }
    // next level (the level loop's accounting, done here)
    ++L;
    nu -= nf;
    mu -= mf;
    edges += mf;
    if (threadIdx.x == 0 && L - 1 < a.trace_cap) {
      LevelTrace t;
      t.level = L;
      t.dir = 3u;  // single-CTA push
      t.nf = nf;
      t.nu = nu;
      t.mf = mf;
      t.mu = mu;
      t.t_ns = gsrb::ptx::globaltimer_ns();
      t.pred = __int_as_float(0x7fc00000);
      t.fallback = 0u;
      a.trace[L - 1] = t;
    }
    prev_nf = nf;
    nreg = nr;
    nbig = nb;
  }
}

// Block-wide exclusive prefix sum of x (blockDim.x a multiple of 32, <= 1024);
// *total receives the block's sum.  `s` holds 32 words of shared memory.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t x, uint32_t* s, uint32_t* total) {
  const uint32_t lane = lane_id(), wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= (uint32_t)o) inc += y;
  }
  if (lane == 31) s[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    uint32_t v = lane < nw ? s[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= (uint32_t)o) v += y;
    }
    s[lane] = v;
  }
  __syncthreads();
  const uint32_t before = wid ? s[wid - 1] : 0u;
  *total = s[nw - 1];
  __syncthreads();
  return before + inc - x;
}

// Load-balanced expansion of a push level's regular queue (the reference's
// thread-block load balancer, apps/bfs/kernel_gsrb.cu:312-399, inspector
// :360-383, with its prefix sum and binary-search edge assignment): every warp
// gets the same number of edges whatever the degrees.
//   1. each CTA sums the degrees of its slice of the queue;      (team barrier)
//   2. each CTA offsets its slice by the totals of the CTAs before it, writes
//      every entry's first-edge offset (lb_pre) and, for every kLbChunk-edge
//      chunk that starts inside an entry's edges, the entry (lb_own);  (barrier)
//   3. warps take chunks grid-stride; a warp walks its chunk 32 edges at a
//      time with a window of 32 queue entries, each lane finding its edge's
//      entry by a binary search over the window's offsets in registers.
// Returns false if a team barrier failed.
template <int V, class F>
__device__ __forceinline__ bool bfs_lb_expand(gsrb::GridSync<V>& bar, const BfsArgs& a, const Team& team,
                                              const uint2* __restrict__ qin, uint32_t nq, F& push_edge) {
  uint32_t* s_scan = list_smem().scan;
  __shared__ uint32_t s_off, s_tot;
  const uint32_t G = team.ncta, c = team.cta;
  const uint32_t s0 = (uint32_t)((uint64_t)nq * c / G), s1 = (uint32_t)((uint64_t)nq * (c + 1) / G);
  // 1. slice totals
  uint32_t local = 0;
  for (uint32_t i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
    const uint2 r = __ldcg(qin + i);
    local += r.y - r.x;
  }
  uint32_t tsum = 0;
  (void)block_exclusive_scan(local, s_scan, &tsum);
  if (threadIdx.x == 0) a.lb_part[c] = tsum;
  if (!bar.sync()) return false;
  // 2. offsets, owners of chunk starts
  uint32_t off = 0, tot = 0;
  for (uint32_t k = threadIdx.x; k < G; k += blockDim.x) {
    const uint32_t v = __ldcg(a.lb_part + k);
    tot += v;
    if (k < c) off += v;
  }
  uint32_t t1 = 0, t2 = 0;
  (void)block_exclusive_scan(off, s_scan, &t1);
  (void)block_exclusive_scan(tot, s_scan, &t2);
  if (threadIdx.x == 0) {
    s_off = t1;
    s_tot = t2;
  }
  __syncthreads();
  uint32_t carry = s_off;
  const uint32_t W = s_tot;
  for (uint32_t base = s0; base < s1; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    uint32_t d = 0;
    if (i < s1) {
      const uint2 r = __ldcg(qin + i);
      d = r.y - r.x;
    }
    uint32_t tile = 0;
    const uint32_t ex = block_exclusive_scan(d, s_scan, &tile);
    if (i < s1) {
      const uint32_t P = carry + ex;
      a.lb_pre[i] = P;
      for (uint32_t k = (P + kLbChunk - 1) / kLbChunk; k * kLbChunk < P + d; ++k) a.lb_own[k] = i;
    }
    carry += tile;
  }
  if (!bar.sync()) return false;
  // 3. edge-balanced walk
  const uint32_t lane = lane_id();
  const uint32_t nchunks = (W + kLbChunk - 1) / kLbChunk;
  for (uint32_t chunk = team.warp(); chunk < nchunks; chunk += team.nwarps()) {
    uint32_t o = __ldcg(a.lb_own + chunk);
    uint32_t t0 = chunk * kLbChunk;
    const uint32_t t_end = min(t0 + kLbChunk, W);
    for (;;) {
      const uint32_t wi = o + lane;
      uint32_t p = W, b = 0;
      if (wi < nq) {
        p = __ldcg(a.lb_pre + wi);
        b = __ldcg(&qin[wi].x);
      }
      const uint32_t p_next = o + 32 < nq ? __ldcg(a.lb_pre + o + 32) : W;
      const uint32_t t_lim = min(t_end, p_next);
      const uint32_t t = t0 + lane;
      // largest window slot j with p_j <= t (offsets are non-decreasing)
      uint32_t j = 0;
#pragma unroll
      for (uint32_t st = 16; st > 0; st >>= 1) {
        const uint32_t pc = __shfl_sync(0xffffffffu, p, j + st);
        if (pc <= t) j += st;
      }
      const uint32_t pj = __shfl_sync(0xffffffffu, p, j), bj = __shfl_sync(0xffffffffu, b, j);
      push_edge(0u, bj + (t - pj), t < t_lim);
      if (t0 + 32 <= t_lim) {
        o += __shfl_sync(0xffffffffu, j, 31);
        t0 += 32;
        if (t0 == t_end) break;
      } else if (t_lim == t_end) {
        break;
      } else {
        o += 32;  // the window's entries end before the chunk does
        t0 = t_lim;
      }
    }
  }
  return true;
}

// A push level's hub queue (2..kHubList ranges) expanded edge-balanced over the
// team: every CTA builds the ranges' edge prefix in shared memory (the same in
// every CTA, so no barrier is needed) and its threads take edges grid-stride.
__device__ __forceinline__ void bfs_push_hubs(const BfsArgs& a, const Team& team, const uint2* __restrict__ hin,
                                           uint32_t nbig, int32_t Li, const PushSink sink,
                                           unsigned long long& m_acc) {
  ListSmem& L_ = list_smem();
  uint32_t carry = 0;
  for (uint32_t base = 0; base < nbig; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    uint32_t d = 0;
    if (i < nbig) {
      const uint2 r = __ldcg(hin + i);
      L_.b[i] = r.x;
      d = r.y - r.x;
    }
    uint32_t tile = 0;
    const uint32_t ex = block_exclusive_scan(d, L_.scan, &tile);
    if (i < nbig) L_.p[i] = carry + ex;
    carry += tile;
  }
  if (threadIdx.x == 0) L_.p[nbig] = carry;
  __syncthreads();
  bfs_push_list(a.g, a.level, Li, L_.p, L_.b, nbig, team.tid(), team.nthreads(), sink, m_acc);
  __syncthreads();
}

// The traversal body, relative to a team (the whole grid, or one instance's
// CTA range in a batch, synchronised by `bar`).
template <int V>
__device__ __forceinline__ void bfs_run(gsrb::GridSync<V>& bar, bool ok, const BfsArgs& a, const Team team) {
  __shared__ uint32_t s_dir;
  __shared__ float s_pred;
  __shared__ MLPShared s_mlp;
  const DevCSR& g = a.g;
  const uint32_t tid = team.tid(), nthreads = team.nthreads();
  if (a.mode == GSRB_BFS_LEARNED) mlp_stage(a.mlp, &s_mlp);  // visible after the barrier below

  // init (bfs_init, bfs/kernel_gsrb.cu:299-311) fused into the persistent kernel
  for (uint32_t v = tid; v < g.n; v += nthreads) a.level[v] = (v == a.src) ? 0 : kInf;
  const uint32_t dsrc = g.row[a.src + 1] - g.row[a.src];
  if (tid == 0) {
    const bool hub = dsrc > kBigDegree;
    reinterpret_cast<uint2*>(hub ? a.hq[0] : a.q[0])[0] = make_uint2(g.row[a.src], g.row[a.src + 1]);
    a.cnt[0].n_reg = a.cnt[0].n_real = hub ? 0 : 1;
    a.cnt[0].n_big = hub ? 1 : 0;
    a.cnt[0].m_next = dsrc;
    a.cnt[1].n_reg = a.cnt[1].n_real = a.cnt[1].n_big = a.cnt[1].m_next = 0;
    a.cnt[2].n_reg = a.cnt[2].n_real = a.cnt[2].n_big = a.cnt[2].m_next = 0;
  }
  ok = bar.sync() && ok;

  uint32_t nu = g.n - 1;
  unsigned long long mu = (unsigned long long)g.m - dsrc;
  unsigned long long edges = dsrc;
  uint32_t dir = DIR_PUSH, prev_nf = 1;
  bool fallback = a.mode != GSRB_BFS_LEARNED;
  uint32_t fb_level = 0;  // level at which the policy fell back (0 = never)
  float pred = __int_as_float(0x7fc00000);
  uint32_t L = 1;
  uint32_t decisions = 0;
  uint32_t last_dir = DIR_PUSH, last_nf = 0;  // the policy's last decision and the frontier it saw
  unsigned long long last_mf = 0;
  for (; ok; ++L) {
    const LevelCounters cur = {__ldcg(&a.cnt[(L - 1) % 3].n_reg), __ldcg(&a.cnt[(L - 1) % 3].n_big),
                               __ldcg(&a.cnt[(L - 1) % 3].m_next), __ldcg(&a.cnt[(L - 1) % 3].n_real)};
    // nreg counts queue slots (the expansion's bound), n_real the entries
    const uint32_t nreg = (uint32_t)cur.n_reg, nbig = (uint32_t)cur.n_big;
    const uint32_t nf = (uint32_t)cur.n_real + nbig;
    if (nf == 0) break;
    const unsigned long long mf = cur.m_next;
    if (L > 1) {
      nu -= nf;
      mu -= mf;
      edges += mf;
    }
    // ---- choose the level's direction (identical in every CTA)
    if (!fallback && L > 1 && pred == pred) {
      const float actual = log2f(1.f + (float)nf);
      if (fabsf(actual - pred) > 1.f) {  // missed by more than 2x
        fallback = true;
        fb_level = L;
      }
    }
    uint32_t nd = DIR_PUSH;
    if (a.mode == GSRB_BFS_PULL) {
      nd = L == 1 ? DIR_PUSH : DIR_PULL;
    } else if (a.mode == GSRB_BFS_TOPO) {
      nd = DIR_TOPO;
    } else if (a.mode == GSRB_BFS_HEURISTIC || (a.mode == GSRB_BFS_LEARNED && fallback)) {
      nd = dir;
      if (dir != DIR_PULL && (double)mf > (double)mu / a.alpha) nd = DIR_PULL;
      else if (dir == DIR_PULL && (double)nf < (double)g.n / a.beta) nd = DIR_PUSH;
    } else if (a.mode == GSRB_BFS_LEARNED) {
      // the network is evaluated again only when the frontier's size or edge
      // count has moved by more than 2x since its last decision (on meshes and
      // road networks that skips most levels); a reused decision carries no
      // prediction, so it cannot trigger the fallback
      const bool reuse = decisions > 0 && nf <= 2u * last_nf && 2u * nf >= last_nf && mf <= 2ull * last_mf &&
                         2ull * mf >= last_mf;
      if (reuse) {
        nd = last_dir;
        pred = __int_as_float(0x7fc00000);
      } else {
        if (threadIdx.x < 32) {
          float feat[kFeat], out[kOut];
          level_features(feat, g.n, g.m, L, nf, mf, nu, mu, prev_nf, dir);
          mlp_forward_smem(&s_mlp, feat, out);
          if (threadIdx.x == 0) {
            // the topology push scans all n vertices: taken only on a confident
            // output; the first level always pushes (its frontier is the source,
            // and the training labels hold no pull decision for it)
            s_dir = (out[0] > 0.f && L > 1) ? DIR_PULL : (out[1] > kTopoLogit ? DIR_TOPO : DIR_PUSH);
            s_pred = out[2];
          }
        }
        __syncthreads();
        nd = s_dir;
        pred = s_pred;
        last_dir = nd;
        last_nf = nf;
        last_mf = mf;
        ++decisions;
      }
    }
    // a pull level reads rows as in-edges: only on symmetric graphs
    if (nd == DIR_PULL && !a.symmetric) nd = DIR_PUSH;
    dir = nd;
    if (team.cta == 0 && threadIdx.x == 0) {
      // the counter set of level L + 1 was last read before barrier L - 1
      a.cnt[(L + 1) % 3].n_reg = 0;
      a.cnt[(L + 1) % 3].n_real = 0;
      a.cnt[(L + 1) % 3].n_big = 0;
      a.cnt[(L + 1) % 3].m_next = 0;
      if (L - 1 < a.trace_cap) {
        LevelTrace t;
        t.level = L;
        t.dir = dir;
        t.nf = nf;
        t.nu = nu;
        t.mf = mf;
        t.mu = mu;
        t.t_ns = gsrb::ptx::globaltimer_ns();
        t.pred = (a.mode == GSRB_BFS_LEARNED && !fallback) ? pred : __int_as_float(0x7fc00000);
        t.fallback = fallback ? 1u : 0u;
        a.trace[L - 1] = t;
      }
    }
    prev_nf = nf;

    if (team.ncta > 1 && dir == DIR_PUSH && nf <= blockDim.x && mf <= 4ull * blockDim.x &&
        (a.mode == GSRB_BFS_HEURISTIC || a.mode == GSRB_BFS_LEARNED)) {
      if (team.cta == 0) bfs_solo(a, L, nreg, nbig, nu, mu, edges, prev_nf);
      ok = bar.sync();
      if (!ok) break;
      L = __ldcg(a.solo + 0);
      nu = __ldcg(a.solo + 1);
      prev_nf = __ldcg(a.solo + 2);
      mu = __ldcg(reinterpret_cast<const unsigned long long*>(a.solo + 4));
      edges = __ldcg(reinterpret_cast<const unsigned long long*>(a.solo + 6));
      dir = DIR_PUSH;
      pred = __int_as_float(0x7fc00000);  // no prediction for the level after the phase
      continue;
    }

    const uint2* qin = reinterpret_cast<const uint2*>(a.q[(L - 1) & 1]);
    const uint2* hin = reinterpret_cast<const uint2*>(a.hq[(L - 1) & 1]);
    uint2* qout = reinterpret_cast<uint2*>(a.q[L & 1]);
    uint2* hout = reinterpret_cast<uint2*>(a.hq[L & 1]);
    LevelCounters* c = &a.cnt[L % 3];
    unsigned long long m_acc = 0;
    const int32_t Li = (int32_t)L;
    // regular-queue slots reserved per warp in chunks of 64 (one counter atomic
    // per chunk) when the queue's 2n slots can hold every warp's holes
    WarpRes res{0ull, 0u, 63ull * team.nwarps() <= g.n ? 64u : 0u};
    uint32_t real_w = 0;  // regular entries this warp appended (warp-uniform)
    const PushSink sink{qout, hout, &c->n_reg, &c->n_big, g.n, a.overflow, &res, &real_w, 2u * g.n};

    auto discover = [&](bool disc, uint32_t v) {
      uint2 r = make_uint2(0u, 0u);
      if (disc) r = make_uint2(__ldg(g.row + v), __ldg(g.row + v + 1));
      const uint32_t d = r.y - r.x;
      const bool reg1[1] = {disc && d <= kBigDegree};
      push_append_reg<1>(reg1, &r, sink);
      warp_append(disc && d > kBigDegree, r, hout, &c->n_big, g.n, a.overflow);
      m_acc += d;
    };
    auto push_edge = [&](uint32_t, uint32_t j, bool active) {
      uint32_t v = 0;
      bool disc = false;
      if (active) {
        v = __ldg(g.dst + j);
        if (__ldcg(a.level + v) == kInf) disc = atomicCAS(a.level + v, kInf, Li) == kInf;
      }
      discover(disc, v);
    };

    if (dir == DIR_PUSH) {
      if (nbig > 1 && nbig <= kHubList) {
        // hubs edge-balanced over the team: every CTA builds the same prefix
        bfs_push_hubs(a, team, hin, nbig, Li, sink, m_acc);
      } else {
        expand_hub_ranges(team, hin, nbig, push_edge);
      }
      if (a.lb && team.ncta > 1 && mf >= kLbMinEdges) {
        // uniform across the team: every CTA takes the two extra barriers
        if (!bfs_lb_expand(bar, a, team, qin, nreg, push_edge)) {
          ok = false;
          break;
        }
      } else {
        const bool precheck = nf > kPushPrecheckFrontier;
        auto lanes = [&](uint32_t b, uint32_t mine, uint32_t kmax) {
          bfs_push_lanes(g, a.level, Li, b, mine, kmax, precheck, sink, m_acc);
        };
        expand_range_queue(team, qin, nreg, push_edge, lanes);
      }
    } else if (dir == DIR_TOPO) {
      // topology-driven push: scan every vertex, expand those at level L - 1
      expand_hub_ranges(team, hin, nbig, push_edge);
      const uint32_t lane = lane_id();
      const uint32_t gw = tid >> 5, nw = nthreads >> 5;
      for (uint32_t base = gw * 32u; base < g.n; base += nw * 32u) {
        const uint32_t u = base + lane;
        uint32_t b = 0, e = 0;
        if (u < g.n && __ldcg(a.level + u) == Li - 1) {
          b = __ldg(g.row + u);
          e = __ldg(g.row + u + 1);
          if (e - b > kBigDegree) e = b;  // hubs were expanded above
        }
        const uint32_t deg = e - b;
        uint32_t coop = __ballot_sync(0xffffffffu, deg > kWarpDegree);
        while (coop) {
          const int s = __ffs(coop) - 1;
          coop &= coop - 1;
          const uint32_t bb = __shfl_sync(0xffffffffu, b, s), ee = __shfl_sync(0xffffffffu, e, s);
          for (uint32_t j0 = bb; j0 < ee; j0 += 32) push_edge(0, j0 + lane, j0 + lane < ee);
        }
        const uint32_t mine = deg <= kWarpDegree ? deg : 0u;
        const uint32_t kmax = warp_max_u32(mine);
        for (uint32_t k = 0; k < kmax; ++k) push_edge(u, b + k, k < mine);
      }
    } else {
      // pull: every unvisited vertex looks for a neighbour at level L - 1
      const uint32_t lane = lane_id();
      const uint32_t gw = tid >> 5, nw = nthreads >> 5;
      for (uint32_t base = gw * 32u; base < g.n; base += nw * 32u) {
        const uint32_t v = base + lane;
        bool unv = false;
        uint32_t b = 0, e = 0;
        if (v < g.n && __ldcg(a.level + v) == kInf) {
          unv = true;
          b = __ldg(g.row + v);
          e = __ldg(g.row + v + 1);
        }
        const uint32_t deg = e - b;
        bool found = false;
        if (unv && deg <= kWarpDegree) {
          for (uint32_t j = b; j < e; ++j)
            if (__ldcg(a.level + __ldg(g.dst + j)) == Li - 1) { found = true; break; }
        }
        uint32_t coop = __ballot_sync(0xffffffffu, unv && deg > kWarpDegree);
        while (coop) {
          const int s = __ffs(coop) - 1;
          coop &= coop - 1;
          const uint32_t bb = __shfl_sync(0xffffffffu, b, s), ee = __shfl_sync(0xffffffffu, e, s);
          bool hit = false;
          for (uint32_t j0 = bb; j0 < ee && !hit; j0 += 32) {
            const uint32_t j = j0 + lane;
            const bool h = j < ee && __ldcg(a.level + __ldg(g.dst + j)) == Li - 1;
            hit = __ballot_sync(0xffffffffu, h) != 0u;
          }
          if ((int)lane == s) found = hit;
        }
        if (found) gsrb::ptx::st_relaxed_gpu_s32(a.level + v, Li);
        discover(found, v);
      }
    }
    // per-warp edge sums and entry counts of the new frontier
    warp_res_close(qout, 2u * g.n, res, make_uint2(0u, 0u));
    const unsigned long long ws = warp_sum_u64(m_acc);
    if (lane_id() == 0 && ws) atomicAdd(&c->m_next, ws);
    if (lane_id() == 0 && real_w) atomicAdd(&c->n_real, (unsigned long long)real_w);
    ok = bar.sync();
  }
  if (team.cta == 0 && threadIdx.x == 0) {
    a.out[0] = L - 1;  // levels with a non-empty frontier beyond the source
    a.out[2] = decisions;
    a.out[3] = ok ? 0u : 1u;
    *a.out_edges = edges;
  }
  // first level at which the policy fell back (0 = never), kept in a
  // register: scanning the trace for it here cost one thread a dependent load
  // per level (about 1 ms on a 4095-level mesh)
  if (team.cta == 0 && threadIdx.x == 0 && a.mode == GSRB_BFS_LEARNED) a.out[1] = fb_level;
}

constexpr int kGraphMaxThreads = 1024;

template <int V>
__global__ void __launch_bounds__(kGraphMaxThreads)
bfs_kernel(gsrb::GridBarrier gb, BfsArgs a) {
  __shared__ gsrb::BarrierShared bsh;
  gsrb::GridSync<V> bar;
  const bool ok = bar.init(gb, &bsh);
  bfs_run<V>(bar, ok, a, Team{blockIdx.x, gridDim.x});
  bar.finish();
}

// ------------------------------------------------------------------- SSSP ---
struct SsspArgs {
  DevCSR g;
  uint32_t src;
  int32_t* dist;
  uint32_t* q[2];
  uint32_t* hq[2];
  uint32_t* far[2];
  uint32_t* mark;       // near-queue stamps
  uint32_t* fmark;      // far-pile stamps
  LevelCounters* cnt;   // [3] near counters
  unsigned long long* fcnt;  // [2] far counters
  uint32_t* overflow;
  LevelTrace* trace;
  uint32_t trace_cap;
  int32_t delta;
  uint32_t* out;        // [0] relax rounds, [1] buckets, [3] failure
  unsigned long long* out_edges;
};

// Where an SSSP relax step puts the vertices whose distance it lowered.
struct RelaxSink {
  uint32_t* qout;               // near queue of the next round
  uint32_t* hout;               // near hub queue
  unsigned long long* n_reg;
  unsigned long long* n_big;
  uint32_t* fout;               // far pile
  unsigned long long* fc;
  uint32_t stamp;               // near-queue stamp of this round
  uint32_t fgen;                // far-pile generation
  long long T;                  // near threshold
  WarpRes* res;                 // the warp's near-queue reservation
  uint32_t near_cap;            // near-queue capacity in slots (holes included)
  bool precheck;                // read a distance before claiming it (large rounds)
};

// Relax four edges per lane at once: edge r of the lane is j[r] (where bit r of
// `act` is set), leaving a vertex at distance du[r].  Every dependent step is
// issued for all four before the next (destinations and weights, distance
// probes, the atomicMin claims, the stamps), and the warp reserves queue space
// once per step.  The row range of a destination (its degree, for the queue
// it enters) is loaded alongside its stamp exchange; in small rounds
// (!s.precheck) the distance probe is skipped -- the atomicMin itself tells
// whether the edge improves -- and the row range goes out with the claim.
// The same claims land either way, so distances are the same.
// Warp-synchronous.
__device__ __forceinline__ void sssp_relax4e(const SsspArgs& a, const long long* du, const uint32_t* j, uint32_t act,
                                             const RelaxSink& s, unsigned long long& my_edges) {
  const DevCSR& g = a.g;
  uint32_t v[4];
  long long nd[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const bool on = (act >> r) & 1u;
    v[r] = on ? __ldg(g.dst + j[r]) : 0u;
    nd[r] = on ? du[r] + (long long)__ldg(g.w + j[r]) : (long long)kInf;
    my_edges += on ? 1u : 0u;
  }
  bool imp[4];
  uint32_t rb[4], re[4];
  if (s.precheck) {
    int32_t cur[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) cur[r] = nd[r] < (long long)kInf ? __ldcg(a.dist + v[r]) : kInf;
#pragma unroll
    for (int r = 0; r < 4; ++r)
      imp[r] = nd[r] < (long long)cur[r] && nd[r] < (long long)atomicMin(a.dist + v[r], (int32_t)nd[r]);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      rb[r] = imp[r] && nd[r] < s.T ? __ldg(g.row + v[r]) : 0u;
      re[r] = imp[r] && nd[r] < s.T ? __ldg(g.row + v[r] + 1) : 0u;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const bool on = nd[r] < (long long)kInf;
      rb[r] = on && nd[r] < s.T ? __ldg(g.row + v[r]) : 0u;
      re[r] = on && nd[r] < s.T ? __ldg(g.row + v[r] + 1) : 0u;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r)
      imp[r] = nd[r] < (long long)kInf && nd[r] < (long long)atomicMin(a.dist + v[r], (int32_t)nd[r]);
  }
  bool to_near[4], to_far[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    to_near[r] = imp[r] && nd[r] < s.T && atomicExch(a.mark + v[r], s.stamp) != s.stamp;
    to_far[r] = imp[r] && nd[r] >= s.T && atomicExch(a.fmark + v[r], s.fgen) != s.fgen;
  }
  uint32_t d[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) d[r] = to_near[r] ? re[r] - rb[r] : 0u;
  bool reg[4], big[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    reg[r] = to_near[r] && d[r] <= kBigDegree;
    big[r] = to_near[r] && d[r] > kBigDegree;
  }
  if (s.res->chunk) warp_append_res<4>(reg, v, s.qout, s.n_reg, s.near_cap, a.overflow, *s.res, kHole);
  else warp_append_k<4>(reg, v, s.qout, s.n_reg, g.n, a.overflow);
  warp_append_k<4>(big, v, s.hout, s.n_big, g.n, a.overflow);
  warp_append_k<4>(to_far, v, s.fout, s.fc, g.n, a.overflow);
}

// The same from one vertex: edge r is jbase + r * stride while below jend.
__device__ __forceinline__ void sssp_relax4(const SsspArgs& a, long long du, uint32_t jbase, uint32_t stride,
                                            uint32_t jend, const RelaxSink& s, unsigned long long& my_edges) {
  long long dd[4];
  uint32_t j[4];
  uint32_t act = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    dd[r] = du;
    j[r] = jbase + (uint32_t)r * stride;
    if (j[r] < jend) act |= 1u << r;
  }
  sssp_relax4e(a, dd, j, act, s, my_edges);
}

// A list of vertices relaxed edge-balanced: their edge counts' prefix p[0..cnt]
// (p[cnt] = total), first edges b[] and distances d[] in shared memory.  Thread
// x of nthr takes edges (x & ~31) + lane + k * nthr, four per step, each
// finding its vertex by binary search over p.  Warp-synchronous loops.
__device__ __forceinline__ void sssp_relax_list(const SsspArgs& a, const uint32_t* p, const uint32_t* b,
                                                const int32_t* d, uint32_t cnt, uint32_t x, uint32_t nthr,
                                                const RelaxSink& s, unsigned long long& my_edges) {
  const uint32_t total = p[cnt];
  for (uint32_t t0 = (x & ~31u) + lane_id(); t0 - lane_id() < total; t0 += 4u * nthr) {
    long long du[4];
    uint32_t j[4];
    uint32_t act = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint32_t t = t0 + (uint32_t)r * nthr;
      du[r] = 0;
      j[r] = 0;
      if (t < total) {
        const uint32_t o = list_owner(p, cnt, t);
        j[r] = b[o] + (t - p[o]);
        du[r] = d[o];
        act |= 1u << r;
      }
    }
    sssp_relax4e(a, du, j, act, s, my_edges);
  }
}

// Vertices of the regular queue with more edges than this are relaxed by their
// whole CTA (after the CTA's warps have walked their queue groups), so that one
// warp does not walk thousands of edges while the rest of the grid waits at
// the round's barrier (the thread-block tier of the reference's nested
// parallelism, LONESTAR/rt/include/internal.h.prehip:99-158).
constexpr uint32_t kCtaDegree = 256;
constexpr uint32_t kCtaListCap = 256;

template <int V>
__device__ __forceinline__ void sssp_run(gsrb::GridSync<V>& bar, bool ok, const SsspArgs& a, const Team team) {
  const DevCSR& g = a.g;
  const uint32_t tid = team.tid(), nthreads = team.nthreads();
  for (uint32_t v = tid; v < g.n; v += nthreads) {
    a.dist[v] = (v == a.src) ? 0 : kInf;
    a.mark[v] = 0;
    a.fmark[v] = 0;
  }
  const uint32_t dsrc = g.row[a.src + 1] - g.row[a.src];
  if (tid == 0) {
    const bool hub = dsrc > kBigDegree;
    if (hub) a.hq[0][0] = a.src;
    else a.q[0][0] = a.src;
    for (int k = 0; k < 3; ++k) a.cnt[k].n_reg = a.cnt[k].n_big = a.cnt[k].m_next = 0;
    a.cnt[0].n_reg = hub ? 0 : 1;
    a.cnt[0].n_big = hub ? 1 : 0;
    a.fcnt[0] = a.fcnt[1] = 0;
  }
  ok = bar.sync() && ok;

  // near threshold: vertices with dist < T are relaxed in the current bucket
  long long T = a.delta;
  uint32_t step = 1;       // index of the near counter set in use (rotating by 3)
  uint32_t fpar = 0;       // far pile parity
  uint32_t fgen = 1;       // generation of the current far pile (fmark stamps: a vertex enters a pile once)
  uint32_t rounds = 0, buckets = 1;
  unsigned long long relaxed_edges = 0;
  while (ok) {
    const LevelCounters cur = {__ldcg(&a.cnt[(step - 1) % 3].n_reg), __ldcg(&a.cnt[(step - 1) % 3].n_big), 0, 0};
    const uint32_t nreg = (uint32_t)cur.n_reg, nbig = (uint32_t)cur.n_big;
    const uint32_t nf = nreg + nbig;
    if (team.cta == 0 && threadIdx.x == 0) {
      a.cnt[(step + 1) % 3].n_reg = 0;
      a.cnt[(step + 1) % 3].n_big = 0;
      a.cnt[(step + 1) % 3].m_next = 0;
    }
    if (nf == 0) {
      // ---- near bucket empty: advance the threshold and refill from the far pile
      const uint32_t nfar = (uint32_t)__ldcg(&a.fcnt[fpar]);
      if (nfar == 0) break;
      T += a.delta;
      ++buckets;
      const uint32_t* fin = a.far[fpar];
      uint32_t* fout = a.far[fpar ^ 1];
      unsigned long long* fc_out = &a.fcnt[fpar ^ 1];
      uint32_t* qout = a.q[step & 1];
      uint32_t* hout = a.hq[step & 1];
      LevelCounters* c = &a.cnt[step % 3];
      const uint32_t stamp = step;
      const uint32_t next_gen = fgen + 1;
      if (team.cta == 0 && threadIdx.x == 0) *fc_out = 0;  // last read before the previous barrier
      // fc_out must be zero before anyone appends: appends happen below, after
      // this CTA's store, so publish it through the barrier first
      ok = bar.sync();
      if (!ok) break;
      const uint32_t lane = lane_id();
      const uint32_t gw = tid >> 5, nw = nthreads >> 5;
      for (uint32_t base = gw * 32u; base < nfar; base += nw * 32u) {
        const uint32_t i = base + lane;
        uint32_t v = 0;
        bool near = false, keep = false;
        if (i < nfar) {
          v = __ldcg(fin + i);
          const int32_t dv = __ldcg(a.dist + v);
          if ((long long)dv < T) near = atomicExch(a.mark + v, stamp) != stamp;
          else keep = atomicExch(a.fmark + v, next_gen) != next_gen;
        }
        uint32_t d = 0;
        if (near) d = __ldg(g.row + v + 1) - __ldg(g.row + v);
        warp_append(near && d <= kBigDegree, v, qout, &c->n_reg, g.n, a.overflow);
        warp_append(near && d > kBigDegree, v, hout, &c->n_big, g.n, a.overflow);
        warp_append(keep, v, fout, fc_out, g.n, a.overflow);
      }
      fpar ^= 1;
      fgen = next_gen;
      ++step;
      ok = bar.sync();
      continue;
    }
    // ---- relax the near frontier
    ++rounds;
    if (team.cta == 0 && threadIdx.x == 0 && rounds - 1 < a.trace_cap) {
      LevelTrace t;
      t.level = rounds;
      t.dir = 0;
      t.nf = nf;
      t.nu = buckets;
      t.mf = 0;
      t.mu = (unsigned long long)T;
      t.t_ns = gsrb::ptx::globaltimer_ns();
      t.pred = __int_as_float(0x7fc00000);
      t.fallback = 0;
      a.trace[rounds - 1] = t;
    }
    const uint32_t* qin = a.q[(step - 1) & 1];
    const uint32_t* hin = a.hq[(step - 1) & 1];
    uint32_t* qout = a.q[step & 1];
    uint32_t* hout = a.hq[step & 1];
    LevelCounters* c = &a.cnt[step % 3];
    uint32_t* fout = a.far[fpar];
    unsigned long long* fc = &a.fcnt[fpar];
    const uint32_t stamp = step + 1;  // stamps of vertices queued for the next round
    unsigned long long my_edges = 0;
    auto relax = [&](uint32_t u, uint32_t j, bool active) {
      uint32_t v = 0;
      bool to_near = false, to_far = false;
      if (active) {
        ++my_edges;
        v = __ldg(g.dst + j);
        const long long nd = (long long)__ldcg(a.dist + u) + (long long)__ldg(g.w + j);
        if (nd < (long long)__ldcg(a.dist + v)) {
          const int32_t old = atomicMin(a.dist + v, (int32_t)nd);
          if (nd < (long long)old) {
            if (nd < T) to_near = atomicExch(a.mark + v, stamp) != stamp;
            else to_far = atomicExch(a.fmark + v, fgen) != fgen;
          }
        }
      }
      uint32_t d = 0;
      if (to_near) d = __ldg(g.row + v + 1) - __ldg(g.row + v);
      // (the near queue's slots may include reservation holes: 2n of them)
      warp_append(to_near && d <= kBigDegree, v, qout, &c->n_reg, 2u * g.n, a.overflow);
      warp_append(to_near && d > kBigDegree, v, hout, &c->n_big, g.n, a.overflow);
      warp_append(to_far, v, fout, fc, g.n, a.overflow);
    };
    // near-queue reservations in chunks of 64 slots when the queue (2n slots)
    // can hold the holes of every warp
    WarpRes res{0ull, 0u, 63ull * team.nwarps() <= g.n ? 64u : 0u};
    const RelaxSink sink{qout, hout, &c->n_reg, &c->n_big, fout, fc, stamp, fgen, T, &res, 2u * g.n,
                         nf > kPushPrecheckFrontier};
    // vertex lists relaxed edge-balanced: edge prefix, first edge, distance
    ListSmem& L_ = list_smem();
    uint32_t* s_lp = L_.p;
    uint32_t* s_lb = L_.b;
    int32_t* s_ld = L_.d;
    uint32_t* s_scan = L_.scan;
    // builds the list's arrays from vertex ids (CTA-wide)
    auto build_list = [&](auto id_of, uint32_t cnt) {
      uint32_t carry = 0;
      for (uint32_t base = 0; base < cnt; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t d = 0;
        if (i < cnt) {
          const uint32_t u = id_of(i);
          const uint32_t b = __ldg(g.row + u);
          d = __ldg(g.row + u + 1) - b;
          s_lb[i] = b;
          s_ld[i] = __ldcg(a.dist + u);
        }
        uint32_t tile = 0;
        const uint32_t ex = block_exclusive_scan(d, s_scan, &tile);
        if (i < cnt) s_lp[i] = carry + ex;
        carry += tile;
      }
      if (threadIdx.x == 0) s_lp[cnt] = carry;
      __syncthreads();
    };
    if (nbig <= kHubList) {
      // hubs: every CTA builds the same list; the team's threads share its edges
      build_list([&](uint32_t i) { return __ldcg(hin + i); }, nbig);
      sssp_relax_list(a, s_lp, s_lb, s_ld, nbig, team.tid(), team.nthreads(), sink, my_edges);
      __syncthreads();
    } else {
      expand_hubs(team, g, hin, nbig, relax);
    }
    {
      // regular queue: vertices of degree > kCtaDegree go to the CTA's list
      // (relaxed edge-balanced by the whole CTA below); degree > kWarpDegree
      // edge-parallel across the warp; the rest one lane each; every tier
      // keeps four edges per lane in flight
      __shared__ uint32_t s_cta_u[kCtaListCap];
      __shared__ uint32_t s_ncta;
      if (threadIdx.x == 0) s_ncta = 0;
      __syncthreads();
      const uint32_t lane = lane_id();
      const uint32_t gw = team.warp(), nwarps = team.nwarps();
      for (uint32_t base = gw * 32u; base < nreg; base += nwarps * 32u) {
        const uint32_t i = base + lane;
        uint32_t u = 0, b = 0, e = 0;
        int32_t du0 = 0;
        if (i < nreg) {
          u = __ldcg(qin + i);
          if (u != kHole) {
            // the distance is read alongside the row range (one round trip):
            // a later decrease in this round re-queues the vertex anyway
            b = __ldg(g.row + u);
            e = __ldg(g.row + u + 1);
            du0 = __ldcg(a.dist + u);
          }
        }
        const uint32_t deg = e - b;
        bool warp_tier = deg > kWarpDegree;
        if (deg > kCtaDegree) {
          const uint32_t slot = atomicAdd(&s_ncta, 1u);
          if (slot < kCtaListCap) {
            s_cta_u[slot] = u;
            warp_tier = false;
          }
        }
        uint32_t coop = __ballot_sync(0xffffffffu, warp_tier);
        while (coop) {
          const int src = __ffs(coop) - 1;
          coop &= coop - 1;
          const uint32_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
          const long long du = (long long)__shfl_sync(0xffffffffu, du0, src);
          for (uint32_t j0 = bb; j0 < ee; j0 += 128) sssp_relax4(a, du, j0 + lane, 32u, ee, sink, my_edges);
        }
        const uint32_t mine = deg <= kWarpDegree ? deg : 0u;
        const uint32_t kmax = warp_max_u32(mine);
        const long long du = mine ? (long long)du0 : 0;
        for (uint32_t k0 = 0; k0 < kmax; k0 += 4) sssp_relax4(a, du, b + k0, 1u, b + mine, sink, my_edges);
      }
      __syncthreads();
      const uint32_t ncta = min(s_ncta, kCtaListCap);
      if (ncta) {
        build_list([&](uint32_t i) { return s_cta_u[i]; }, ncta);
        sssp_relax_list(a, s_lp, s_lb, s_ld, ncta, threadIdx.x, blockDim.x, sink, my_edges);
      }
    }
    warp_res_close(qout, 2u * g.n, res, kHole);
    relaxed_edges += my_edges;
    ++step;
    ok = bar.sync();
  }
  // per-thread relaxed-edge counts -> one total
  const unsigned long long ws = warp_sum_u64(relaxed_edges);
  if (lane_id() == 0 && ws) atomicAdd(a.out_edges, ws);
  if (team.cta == 0 && threadIdx.x == 0) {
    a.out[0] = rounds;
    a.out[1] = buckets;
    a.out[3] = ok ? 0u : 1u;
  }
}

template <int V>
__global__ void __launch_bounds__(1024)
sssp_kernel(gsrb::GridBarrier gb, SsspArgs a) {
  __shared__ gsrb::BarrierShared bsh;
  gsrb::GridSync<V> bar;
  const bool ok = bar.init(gb, &bsh);
  sssp_run<V>(bar, ok, a, Team{blockIdx.x, gridDim.x});
  bar.finish();
}

// ------------------------------------------------------------------ batches ---
// Many traversals in one persistent launch: instance i owns CTAs
// [first_i, first_i + count_i) and a barrier slot of its own (sub-grid
// barriers carved from the same state block).  A CTA finds its instance in a
// table, copies the instance's descriptor and runs the same traversal body as
// the single-instance kernels.  Only barrier variants whose verdict does not
// involve hardware cluster barriers are used (instances of one CTA are allowed).
struct BatchDesc {
  gsrb::GridBarrier gb;
  uint32_t first;
  uint32_t count;
  uint32_t kind;  // 0 BFS, 1 SSSP
  uint32_t pad;
  BfsArgs bfs;
  SsspArgs sssp;
};

template <int V>
__global__ void __launch_bounds__(kGraphMaxThreads)
batch_kernel(const BatchDesc* __restrict__ descs, const uint16_t* __restrict__ cta_inst) {
  __shared__ gsrb::BarrierShared bsh;
  const uint32_t i = cta_inst[blockIdx.x];
  const BatchDesc& d = descs[i];
  const Team team{blockIdx.x - d.first, d.count};
  gsrb::GridSync<V> bar;
  const bool ok = bar.init(d.gb, &bsh);
  if (d.kind == 0) bfs_run<V>(bar, ok, d.bfs, team);
  else sssp_run<V>(bar, ok, d.sssp, team);
  bar.finish();
}

// --------------------------------------------------------------- PageRank ---
struct PrArgs {
  DevCSR g;
  float alpha;
  int32_t iters;
  float* rank;            // output x (FP32)
  float* contrib[2];      // x / deg, double-buffered by iteration parity
  const uint32_t* hubs;   // vertices of degree > kPrHubDegree, ascending
  const uint32_t* hub_c0; // [nhubs + 1] first chunk of each hub
  const uint32_t* chunk_hub;  // [nchunks] hub index of each chunk
  uint32_t nhubs, nchunks;
  double* part;           // [nchunks] chunk sums
  uint32_t* hub_done;     // [nhubs] finished chunks (monotonic over iterations)
  unsigned long long* ticket;  // block tickets (monotonic over iterations)
  uint32_t* out;
  int32_t gather_l1;      // 1: x/deg gathers through L1 (ld.ca), 0: L2 only (ld.cg)
};

// One x/deg gather.  Through L1 the hubs' entries (read by many rows of a
// power-law graph) hit in the SM: an edge-parallel pass over RMAT-22 with
// nothing but these gathers runs at 340 G edges/s through L1 against 224
// through L2 only.  The buffer a gather reads was last written two iterations
// earlier, before the grid barrier whose acquire orders those writes before
// every later load of the CTA (the acquire invalidates the SM's L1).
__device__ __forceinline__ float pr_gather(const float* cin, uint32_t d, int l1) {
  return l1 ? __ldca(cin + d) : __ldcg(cin + d);
}

// Sum of cin[dst[j]] over j in [j0, j1) by one warp: lanes stride the range,
// 4 independent gathers in flight per lane, FP64 per lane, fixed-order
// butterfly at the end (the same bits on every run).  The destinations of the
// next 128 edges are loaded while this step's gathers are in flight, so a
// step costs one dependent round trip (the gather), not two.
__device__ __forceinline__ double warp_gather_sum(const uint32_t* __restrict__ dst, const float* cin, uint32_t j0,
                                                  uint32_t j1, uint32_t lane, int l1) {
  double s = 0.0;
  uint32_t j = j0 + lane;
  uint32_t d0 = 0, d1 = 0, d2 = 0, d3 = 0;
  if (j + 96 < j1) {
    d0 = __ldg(dst + j);
    d1 = __ldg(dst + j + 32);
    d2 = __ldg(dst + j + 64);
    d3 = __ldg(dst + j + 96);
  }
  for (; j + 96 < j1; j += 128) {
    const float c0 = pr_gather(cin, d0, l1), c1 = pr_gather(cin, d1, l1), c2 = pr_gather(cin, d2, l1),
                c3 = pr_gather(cin, d3, l1);
    if (j + 224 < j1) {
      d0 = __ldg(dst + j + 128);
      d1 = __ldg(dst + j + 160);
      d2 = __ldg(dst + j + 192);
      d3 = __ldg(dst + j + 224);
    }
    s += (double)c0;
    s += (double)c1;
    s += (double)c2;
    s += (double)c3;
  }
  for (; j < j1; j += 32) s += (double)pr_gather(cin, __ldg(dst + j), l1);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// Pull PageRank, one grid barrier per iteration.
//  * Hubs (degree > kPrHubDegree) are cut into chunks of kPrChunk edges; a warp
//    sums a chunk, stores it, and bumps the hub's counter (acq_rel); the warp
//    that finishes a hub's last chunk adds the chunk sums in chunk order and
//    writes the hub's rank and contribution.
//  * Every other vertex: a warp takes 32 consecutive vertices and walks their
//    concatenated edge lists 32 edges per round (coalesced dst loads); each
//    lane finds the owner of its edge by a binary search over the lanes'
//    exclusive degree prefix, and a segmented shuffle scan hands each owner its
//    segment's sum.  Per-vertex FP64 sums in a fixed order.
template <int V>
__global__ void __launch_bounds__(1024)
pagerank_kernel(gsrb::GridBarrier gb, PrArgs a) {
  __shared__ gsrb::BarrierShared bsh;
  gsrb::GridSync<V> bar;
  bool ok = bar.init(gb, &bsh);
  const DevCSR& g = a.g;
  const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
  const float base = 1.f - a.alpha;
  // x0 = 1 - alpha (apps/pr/kernel_gsrb.cu:311)
  for (uint32_t v = tid; v < g.n; v += nthreads) {
    const uint32_t d = __ldg(g.row + v + 1) - __ldg(g.row + v);
    a.rank[v] = base;
    a.contrib[0][v] = d ? base / (float)d : 0.f;
  }
  ok = bar.sync() && ok;
  const uint32_t lane = lane_id();
  const uint32_t gw = tid >> 5, nw = nthreads >> 5;
  int32_t it = 0;
  for (; ok && it < a.iters; ++it) {
    const float* cin = a.contrib[it & 1];
    float* cout = a.contrib[(it + 1) & 1];
    // ---- hub chunks
    for (uint32_t c = gw; c < a.nchunks; c += nw) {
      const uint32_t k = __ldg(a.chunk_hub + c);
      const uint32_t u = __ldg(a.hubs + k);
      const uint32_t c0 = __ldg(a.hub_c0 + k), c1 = __ldg(a.hub_c0 + k + 1);
      const uint32_t ub = __ldg(g.row + u), ue = __ldg(g.row + u + 1);
      const uint32_t j0 = ub + (c - c0) * kPrChunk;
      const uint32_t j1 = min(ue, j0 + kPrChunk);
      const double t = warp_gather_sum(g.dst, cin, j0, j1, lane, a.gather_l1);
      uint32_t last = 0;
      if (lane == 0) {
        a.part[c] = t;
        const uint32_t target = (c1 - c0) * (uint32_t)(it + 1);
        last = gsrb::ptx::atom_add_acq_rel_gpu(a.hub_done + k, 1u) + 1u == target;
      }
      last = __shfl_sync(0xffffffffu, last, 0);
      if (last) {
        // fixed order: lane-strided chunk sums, then the same butterfly
        double s = 0.0;
        for (uint32_t i = c0 + lane; i < c1; i += 32) s += __ldcg(a.part + i);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
          const float x = (float)((double)base + (double)a.alpha * s);
          a.rank[u] = x;
          cout[u] = x / (float)(ue - ub);
        }
      }
    }
    // ---- everything else: blocks of 32 consecutive vertices, taken by warps
    // from a ticket counter (block sizes vary by orders of magnitude)
    const uint32_t nblocks = (g.n + 31u) >> 5;
    const unsigned long long tbase = (unsigned long long)it * (nblocks + nw);
    for (;;) {
      unsigned long long t = 0;
      if (lane == 0) t = atomicAdd(a.ticket, 1ull);
      t = __shfl_sync(0xffffffffu, t, 0);
      const unsigned long long blk = t - tbase;
      if (blk >= nblocks) break;  // every warp draws exactly one ticket past the end
      const uint32_t v = (uint32_t)blk * 32u + lane;
      uint32_t b = 0, d = 0;
      bool mine = false;
      if (v < g.n) {
        b = __ldg(g.row + v);
        const uint32_t dd = __ldg(g.row + v + 1) - b;
        mine = dd <= kPrHubDegree;
        d = mine ? dd : 0u;
      }
      uint32_t inc = d;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if ((int)lane >= o) inc += y;
      }
      const uint32_t excl = inc - d;
      const uint32_t E = __shfl_sync(0xffffffffu, inc, 31);
      double acc = 0.0;
      // kRounds rounds of 32 edges per step: all gathers of a step in flight together
      constexpr int kRounds = 4;
      for (uint32_t f0 = 0; f0 < E; f0 += 32u * kRounds) {
        uint32_t own[kRounds], nbr[kRounds];
        double val[kRounds];
#pragma unroll
        for (int r = 0; r < kRounds; ++r) {
          const uint32_t f = f0 + 32u * r + lane;
          // owner = the last lane whose exclusive prefix is <= f; the search
          // carries that prefix along (lane 0's is 0), so it costs no shuffle
          uint32_t lo = 0, oe = 0;
#pragma unroll
          for (uint32_t step = 16; step > 0; step >>= 1) {
            const uint32_t x = __shfl_sync(0xffffffffu, excl, lo + step);
            if (x <= f) {
              lo += step;
              oe = x;
            }
          }
          // the lane (of this round) where the owner's segment begins: the
          // segmented scan below compares lanes against it instead of
          // shuffling owners
          own[r] = oe > f0 + 32u * r ? oe - (f0 + 32u * r) : 0u;
          const uint32_t ob = __shfl_sync(0xffffffffu, b, lo);
          nbr[r] = f < E ? __ldg(g.dst + ob + (f - oe)) : 0u;
        }
#pragma unroll
        for (int r = 0; r < kRounds; ++r) {
          const uint32_t f = f0 + 32u * r + lane;
          val[r] = f < E ? (double)pr_gather(cin, nbr[r], a.gather_l1) : 0.0;
        }
#pragma unroll
        for (int r = 0; r < kRounds; ++r) {
          const uint32_t rb = f0 + 32u * r;
          if (rb >= E) break;  // warp-uniform
          // segmented inclusive scan: lane l - o belongs to the same owner
          // as lane l exactly when l - o is not before the owner's first lane
          double x = val[r];
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, x, o);
            if ((int)lane - o >= (int)own[r]) x += y;
          }
          // this lane's vertex: its segment in this round ends at flat index
          // min(excl + d, rb + 32, E) - 1
          const uint32_t seg_b = excl > rb ? excl : rb;
          const uint32_t seg_e = min(min(excl + d, rb + 32u), E);
          const uint32_t endl = seg_e > seg_b ? seg_e - 1u - rb : 0u;
          const double t2 = __shfl_sync(0xffffffffu, x, endl);
          if (seg_e > seg_b) acc += t2;
        }
      }
      if (mine) {
        const float x = (float)((double)base + (double)a.alpha * acc);
        a.rank[v] = x;
        cout[v] = d ? x / (float)d : 0.f;
      }
    }
    ok = bar.sync();
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.out[0] = (uint32_t)it;
    a.out[3] = ok ? 0u : 1u;
  }
  bar.finish();
}

// ------------------------------------------------------ push-residual PR ---
// The reference's PageRank (apps/pr/kernel_gsrb.cu:298-508, restated):
//   init_1  p[v] = 1 - alpha; r[w] += 1 / outdeg(u) over every edge u -> w
//   init_2  r[v] *= (1 - alpha) * alpha; every vertex enters the worklist
//   round   for every u in the worklist: res = exchange(r[u], 0); p[u] += res;
//           for every edge u -> w: prev = r[w] += alpha * res / outdeg(u), and
//           w enters the next worklist when r[w] crosses epsilon from below
// until the worklist is empty or max_iters rounds ran; one grid barrier per
// round (+1 when hub vertices, degree > kBigDegree, are in the worklist: their
// residual is taken first and their edges are split across the grid).  FP32
// atomics in an order that changes from run to run, as in the reference;
// p[u] is updated atomically (the reference's plain += races when a vertex is
// in a worklist twice).
struct PrrArgs {
  DevCSR g;
  float alpha, eps;
  int32_t max_iters;
  float* p;             // output ranks
  float* r;             // residuals
  float* hub_upd;       // alpha * res / outdeg of the hubs of the current round, by vertex
  uint32_t* mark;       // round stamps: a vertex enters a worklist at most once
  uint32_t* q[2];
  uint32_t* hq[2];
  LevelCounters* cnt;   // [3]
  uint32_t* overflow;
  uint32_t* out;        // [0] rounds, [1] worklist pushes (low 32 bits), [3] failure
  unsigned long long* out_edges;
};

// Where a residual push step puts the vertices whose residual crossed epsilon.
struct PrrSink {
  uint32_t* qout;
  uint32_t* hout;
  unsigned long long* n_reg;
  unsigned long long* n_big;
  uint32_t stamp;  // a vertex enters the next worklist at most once per round
  WarpRes* res;    // the warp's worklist reservation (chunk 0: direct appends)
};

// Push residual along four edges per lane at once: edge r of the lane is j[r]
// (bit r of `act`), carrying upd[r].  The four destinations, then the four
// residual additions, then the four worklist stamps are issued together, and
// the warp reserves queue space once per step (apps/pr/kernel_gsrb.cu:430-470:
// r[dst] += alpha * res / outdeg, pushed when it crosses epsilon).
// Warp-synchronous.
__device__ __forceinline__ void prr_push4e(const PrrArgs& a, const float* upd, const uint32_t* j, uint32_t act,
                                           const PrrSink& s, unsigned long long& pushes) {
  const DevCSR& g = a.g;
  uint32_t w[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) w[r] = ((act >> r) & 1u) ? __ldg(g.dst + j[r]) : 0u;
  bool cross[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    cross[r] = false;
    if ((act >> r) & 1u) {
      const float prev = atomicAdd(a.r + w[r], upd[r]);
      cross[r] = prev + upd[r] > a.eps && prev < a.eps;
    }
  }
  // the row range of a candidate goes out with its stamp exchange (one round
  // trip instead of two; unused when the exchange finds it already queued)
  uint32_t rb[4], re[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    rb[r] = cross[r] ? __ldg(g.row + w[r]) : 0u;
    re[r] = cross[r] ? __ldg(g.row + w[r] + 1) : 0u;
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) cross[r] = cross[r] && atomicExch(a.mark + w[r], s.stamp) != s.stamp;
  bool reg[4], big[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const uint32_t d = cross[r] ? re[r] - rb[r] : 0u;
    reg[r] = cross[r] && d <= kBigDegree;
    big[r] = cross[r] && d > kBigDegree;
    pushes += cross[r] ? 1u : 0u;
  }
  if (s.res->chunk) warp_append_res<4>(reg, w, s.qout, s.n_reg, 2u * g.n, a.overflow, *s.res, kHole);
  else warp_append_k<4>(reg, w, s.qout, s.n_reg, g.n, a.overflow);
  warp_append_k<4>(big, w, s.hout, s.n_big, g.n, a.overflow);
}

// The same from one vertex: edge r is jbase + r * stride while below jend.
__device__ __forceinline__ void prr_push4(const PrrArgs& a, float upd, uint32_t jbase, uint32_t stride, uint32_t jend,
                                          const PrrSink& s, unsigned long long& pushes) {
  float u4[4];
  uint32_t j[4];
  uint32_t act = 0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    u4[r] = upd;
    j[r] = jbase + (uint32_t)r * stride;
    if (j[r] < jend) act |= 1u << r;
  }
  prr_push4e(a, u4, j, act, s, pushes);
}

// A list of vertices pushed edge-balanced: edge prefix p[0..cnt], first edges
// b[], updates (float bits) d[] in shared memory; thread x of nthr takes edges
// (x & ~31) + lane + k * nthr, four per step.  Warp-synchronous loops.
__device__ __forceinline__ void prr_push_list(const PrrArgs& a, const uint32_t* p, const uint32_t* b,
                                              const int32_t* d, uint32_t cnt, uint32_t x, uint32_t nthr,
                                              const PrrSink& s, unsigned long long& pushes) {
  const uint32_t total = p[cnt];
  for (uint32_t t0 = (x & ~31u) + lane_id(); t0 - lane_id() < total; t0 += 4u * nthr) {
    float upd[4];
    uint32_t j[4];
    uint32_t act = 0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint32_t t = t0 + (uint32_t)r * nthr;
      upd[r] = 0.f;
      j[r] = 0;
      if (t < total) {
        const uint32_t o = list_owner(p, cnt, t);
        j[r] = b[o] + (t - p[o]);
        upd[r] = __int_as_float(d[o]);
        act |= 1u << r;
      }
    }
    prr_push4e(a, upd, j, act, s, pushes);
  }
}

template <int V>
__global__ void __launch_bounds__(1024)
pr_residual_kernel(gsrb::GridBarrier gb, PrrArgs a) {
  __shared__ gsrb::BarrierShared bsh;
  gsrb::GridSync<V> bar;
  bool ok = bar.init(gb, &bsh);
  const DevCSR& g = a.g;
  const Team team{blockIdx.x, gridDim.x};
  const uint32_t tid = team.tid(), nthreads = team.nthreads();
  const uint32_t lane = lane_id();
  // init_1
  for (uint32_t v = tid; v < g.n; v += nthreads) {
    a.p[v] = 1.f - a.alpha;
    a.r[v] = 0.f;
    a.mark[v] = 0;
  }
  if (tid == 0)
    for (int k = 0; k < 3; ++k) a.cnt[k].n_reg = a.cnt[k].n_big = a.cnt[k].m_next = 0;
  ok = bar.sync() && ok;
  for (uint32_t gwarp = tid >> 5; gwarp * 32u < g.n; gwarp += nthreads >> 5) {
    const uint32_t u = gwarp * 32u + lane;
    uint32_t b = 0, e = 0;
    if (u < g.n) {
      b = __ldg(g.row + u);
      e = __ldg(g.row + u + 1);
    }
    const float upd = e > b ? 1.f / (float)(e - b) : 0.f;
    // warp-strided edges of the 32 vertices, one vertex at a time
    for (int src = 0; src < 32; ++src) {
      const uint32_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
      const float uu = __shfl_sync(0xffffffffu, upd, src);
      for (uint32_t j = bb + lane; j < ee; j += 32) atomicAdd(a.r + __ldg(g.dst + j), uu);
    }
  }
  ok = bar.sync() && ok;
  // init_2: scale, every vertex enters the worklist (hubs to the hub queue)
  for (uint32_t base = (tid >> 5) * 32u; base < g.n; base += nthreads) {
    const uint32_t v = base + lane;
    bool reg = false, big = false;
    if (v < g.n) {
      a.r[v] *= (1.f - a.alpha) * a.alpha;
      const uint32_t d = __ldg(g.row + v + 1) - __ldg(g.row + v);
      big = d > kBigDegree;
      reg = !big;
    }
    warp_append(reg, v, a.q[0], &a.cnt[0].n_reg, g.n, a.overflow);
    warp_append(big, v, a.hq[0], &a.cnt[0].n_big, g.n, a.overflow);
  }
  ok = bar.sync() && ok;
  uint32_t round = 0;
  unsigned long long pushes = 0;
  for (; ok && round < (uint32_t)a.max_iters; ++round) {
    const uint32_t nreg = (uint32_t)__ldcg(&a.cnt[round % 3].n_reg);
    const uint32_t nbig = (uint32_t)__ldcg(&a.cnt[round % 3].n_big);
    if (nreg + nbig == 0) break;
    if (tid == 0) {
      a.cnt[(round + 2) % 3].n_reg = 0;
      a.cnt[(round + 2) % 3].n_big = 0;
    }
    const uint32_t* qin = a.q[round & 1];
    const uint32_t* hin = a.hq[round & 1];
    uint32_t* qout = a.q[(round + 1) & 1];
    uint32_t* hout = a.hq[(round + 1) & 1];
    LevelCounters* c = &a.cnt[(round + 1) % 3];
    // a vertex whose residual crosses epsilon twice in one round (its own
    // exchange in this round restarted it from 0) enters the next list once
    const uint32_t stamp = round + 2u;
    auto push = [&](bool cross, uint32_t w) {
      uint32_t d = 0;
      if (cross) cross = atomicExch(a.mark + w, stamp) != stamp;
      if (cross) d = __ldg(g.row + w + 1) - __ldg(g.row + w);
      // (the worklist's slots may include reservation holes: 2n of them)
      warp_append(cross && d <= kBigDegree, w, qout, &c->n_reg, 2u * g.n, a.overflow);
      warp_append(cross && d > kBigDegree, w, hout, &c->n_big, g.n, a.overflow);
      pushes += cross ? 1u : 0u;
    };
    // worklist reservations in chunks of 64 slots when the queue (2n slots)
    // can hold the holes of every warp (see WarpRes)
    WarpRes wres{0ull, 0u, 63ull * (nthreads >> 5) <= g.n ? 64u : 0u};
    const PrrSink sink{qout, hout, &c->n_reg, &c->n_big, stamp, &wres};
    ListSmem& L_ = list_smem();
    // builds an edge-balanced list from vertex ids and their updates (CTA-wide)
    auto build_list = [&](auto id_of, auto upd_of, uint32_t cnt) {
      uint32_t carry = 0;
      for (uint32_t base = 0; base < cnt; base += blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        uint32_t d = 0;
        if (i < cnt) {
          const uint32_t u = id_of(i);
          const uint32_t b = __ldg(g.row + u);
          d = __ldg(g.row + u + 1) - b;
          L_.b[i] = b;
          L_.d[i] = __float_as_int(upd_of(i, u));
        }
        uint32_t tile = 0;
        const uint32_t ex = block_exclusive_scan(d, L_.scan, &tile);
        if (i < cnt) L_.p[i] = carry + ex;
        carry += tile;
      }
      if (threadIdx.x == 0) L_.p[cnt] = carry;
      __syncthreads();
    };
    if (nbig) {
      // hubs: take the residual once, then share the edges across the grid
      for (uint32_t k = tid; k < nbig; k += nthreads) {
        const uint32_t u = __ldcg(hin + k);
        const float res = atomicExch(a.r + u, 0.f);
        atomicAdd(a.p + u, res);
        a.hub_upd[u] = res * a.alpha / (float)(__ldg(g.row + u + 1) - __ldg(g.row + u));
      }
      ok = bar.sync();
      if (!ok) break;
      if (nbig <= kHubList) {
        build_list([&](uint32_t i) { return __ldcg(hin + i); },
                   [&](uint32_t, uint32_t u) { return __ldcg(a.hub_upd + u); }, nbig);
        prr_push_list(a, L_.p, L_.b, L_.d, nbig, tid, nthreads, sink, pushes);
        __syncthreads();
      } else {
        auto hub_edge = [&](uint32_t u, uint32_t j, bool active) {
          bool cross = false;
          uint32_t w = 0;
          if (active) {
            w = __ldg(g.dst + j);
            const float upd = __ldcg(a.hub_upd + u);
            const float prev = atomicAdd(a.r + w, upd);
            cross = prev + upd > a.eps && prev < a.eps;
          }
          push(cross, w);
        };
        expand_hubs(team, g, hin, nbig, hub_edge);
      }
    }
    // regular worklist: a lane per vertex exchanges its residual once; edges
    // of degree > kCtaDegree vertices go to the CTA's edge-balanced list,
    // degree > kWarpDegree across the warp, the rest per lane, four edges per
    // lane in flight
    __shared__ uint32_t s_cta_u[kCtaListCap];
    __shared__ float s_cta_upd[kCtaListCap];
    __shared__ uint32_t s_ncta;
    if (threadIdx.x == 0) s_ncta = 0;
    __syncthreads();
    for (uint32_t base = (tid >> 5) * 32u; base < nreg; base += nthreads) {
      const uint32_t i = base + lane;
      uint32_t u = 0, b = 0, e = 0;
      float upd = 0.f;
      if (i < nreg) u = __ldcg(qin + i);
      if (i < nreg && u != kHole) {
        b = __ldg(g.row + u);
        e = __ldg(g.row + u + 1);
        const float res = atomicExch(a.r + u, 0.f);
        atomicAdd(a.p + u, res);
        upd = e > b ? res * a.alpha / (float)(e - b) : 0.f;
      }
      const uint32_t deg = e - b;
      bool warp_tier = deg > kWarpDegree;
      if (deg > kCtaDegree) {
        const uint32_t slot = atomicAdd(&s_ncta, 1u);
        if (slot < kCtaListCap) {
          s_cta_u[slot] = u;
          s_cta_upd[slot] = upd;
          warp_tier = false;
        }
      }
      uint32_t coop = __ballot_sync(0xffffffffu, warp_tier);
      while (coop) {
        const int src = __ffs(coop) - 1;
        coop &= coop - 1;
        const uint32_t bb = __shfl_sync(0xffffffffu, b, src), ee = __shfl_sync(0xffffffffu, e, src);
        const float uu = __shfl_sync(0xffffffffu, upd, src);
        for (uint32_t j0 = bb; j0 < ee; j0 += 128) prr_push4(a, uu, j0 + lane, 32u, ee, sink, pushes);
      }
      const uint32_t mine = deg <= kWarpDegree ? deg : 0u;
      const uint32_t kmax = warp_max_u32(mine);
      for (uint32_t k0 = 0; k0 < kmax; k0 += 4) prr_push4(a, upd, b + k0, 1u, b + mine, sink, pushes);
    }
    __syncthreads();
    const uint32_t ncta = min(s_ncta, kCtaListCap);
    if (ncta) {
      build_list([&](uint32_t i) { return s_cta_u[i]; }, [&](uint32_t i, uint32_t) { return s_cta_upd[i]; }, ncta);
      prr_push_list(a, L_.p, L_.b, L_.d, ncta, threadIdx.x, blockDim.x, sink, pushes);
    }
    warp_res_close(qout, 2u * g.n, wres, kHole);
    ok = bar.sync();
  }
  const unsigned long long ws = warp_sum_u64(pushes);
  if (lane == 0 && ws) atomicAdd(a.out_edges, ws);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.out[0] = round;
    a.out[3] = ok ? 0u : 1u;
  }
  bar.finish();
}

template <template <int> class K>
struct Dummy {};

#define GSRB_GRAPH_FN(KERNEL)                                                    \
  [](int variant) -> const void* {                                              \
    switch (variant) {                                                          \
      case gsrb::V_CLUSTER: return (const void*)KERNEL<gsrb::V_CLUSTER>;         \
      case gsrb::V_DSMEM: return (const void*)KERNEL<gsrb::V_DSMEM>;             \
      case gsrb::V_SOFT2: return (const void*)KERNEL<gsrb::V_SOFT2>;             \
      case gsrb::V_FLAT: return (const void*)KERNEL<gsrb::V_FLAT>;               \
      case gsrb::V_TREE: return (const void*)KERNEL<gsrb::V_TREE>;               \
      case gsrb::V_CCG: return (const void*)KERNEL<gsrb::V_CCG>;                 \
      case gsrb::V_CLUSTER_RED: return (const void*)KERNEL<gsrb::V_CLUSTER_RED>; \
      case gsrb::V_FLIP: return (const void*)KERNEL<gsrb::V_FLIP>;               \
      case gsrb::V_FANOUT: return (const void*)KERNEL<gsrb::V_FANOUT>;           \
      case gsrb::V_HIER: return (const void*)KERNEL<gsrb::V_HIER>;               \
      default: return nullptr;                                                  \
    }                                                                           \
  }

const void* bfs_fn(int v) { return GSRB_GRAPH_FN(bfs_kernel)(v); }
const void* sssp_fn(int v) { return GSRB_GRAPH_FN(sssp_kernel)(v); }
const void* pr_fn(int v) { return GSRB_GRAPH_FN(pagerank_kernel)(v); }
const void* prr_fn(int v) { return GSRB_GRAPH_FN(pr_residual_kernel)(v); }
const void* batch_fn(int v) {
  switch (v) {  // variants without hardware cluster barriers (teams may be single CTAs)
    case gsrb::V_SOFT2: return (const void*)batch_kernel<gsrb::V_SOFT2>;
    case gsrb::V_FLAT: return (const void*)batch_kernel<gsrb::V_FLAT>;
    case gsrb::V_TREE: return (const void*)batch_kernel<gsrb::V_TREE>;
    case gsrb::V_FLIP: return (const void*)batch_kernel<gsrb::V_FLIP>;
    case gsrb::V_FANOUT: return (const void*)batch_kernel<gsrb::V_FANOUT>;
    case gsrb::V_HIER: return (const void*)batch_kernel<gsrb::V_HIER>;
    default: return nullptr;
  }
}

}  // namespace

const void* gsrb_graph_kernel_for(int variant) { return bfs_fn(variant); }

// ------------------------------------------------------------ host side ----
struct gsrb_graph {
  gsrb_ctx* ctx = nullptr;
  uint32_t n = 0;
  uint32_t m = 0;
  bool owns = false;
  uint32_t* row = nullptr;
  uint32_t* dst = nullptr;
  int32_t* w = nullptr;
  // scratch
  uint32_t* q[2] = {};
  uint32_t* hq[2] = {};
  uint32_t* far[2] = {};
  uint32_t* mark = nullptr;
  uint32_t* fmark = nullptr;
  LevelCounters* cnt = nullptr;
  unsigned long long* fcnt = nullptr;
  uint32_t* flags = nullptr;  // [0] overflow, [4..8) out, [8..16) BFS single-CTA state, edges at byte 64, PageRank tickets at byte 96
  LevelTrace* trace = nullptr;
  uint32_t trace_cap = 0;
  float* contrib[2] = {};
  uint32_t* hubs = nullptr;       // PageRank hubs (degree > kPrHubDegree)
  uint32_t nhubs = 0;
  uint32_t* hub_c0 = nullptr;     // [nhubs + 1] first chunk of each hub
  uint32_t* chunk_hub = nullptr;  // [nchunks] hub of each chunk
  uint32_t nchunks = 0;
  double* hub_part = nullptr;     // [nchunks] chunk sums
  uint32_t* hub_done = nullptr;   // [nhubs] chunk counters
  MLPWeights* mlp = nullptr;
  bool mlp_set = false;
  MLPWeights mlp_host{};        // host copy of the policy weights (the launch choice runs on the host)
  gsrb_cfg_t launch[2]{};       // the two launch configurations head 3 chooses between
  bool launch_set = false;
  uint32_t* lb_pre = nullptr;   // [n] load-balanced BFS: edge offset of each queue entry
  uint32_t* lb_own = nullptr;   // [m / kLbChunk + 2] queue entry owning each chunk's first edge
  uint32_t* lb_part = nullptr;  // [kLbMaxCtas] per-CTA edge totals
  bool symmetric = false;       // every edge (u, v) has its reverse (v, u)
  // graph statistics of the SSSP policy's features (taken when the graph is created)
  uint32_t max_degree = 0;
  std::vector<uint32_t> h_row;  // host copy of row_start (source degrees for the host-side policy heads)
  int32_t w_min = 0, w_max = 0;
  double w_mean = 0.0;
  MLPWeights sssp_host{};       // SSSP policy weights (evaluated on the host, once per traversal)
  bool sssp_set = false;
  int32_t last_delta = 0;       // bucket width of the last SSSP launched on this graph (0: none)
};

namespace {

template <class T>
cudaError_t dalloc(T** p, size_t count) {
  return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

DevCSR dev_csr(const gsrb_graph* G) {
  DevCSR d;
  d.n = G->n;
  d.m = G->m;
  d.row = G->row;
  d.dst = G->dst;
  d.w = G->w;
  return d;
}

// splitmix64's output mix (Steele, Lea, Flood, OOPSLA'14), as a hash of an edge.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Symmetry test of a CSR: sums (mod 2^64) of two hashes of every edge (u, v)
// and of its reverse (v, u).  The edge multiset equals its reverse exactly
// when the graph is symmetric; then both pairs of sums agree, and otherwise
// they differ except with probability about 2^-128.  One warp per row.
__global__ void __launch_bounds__(256) edge_hash_kernel(DevCSR g, unsigned long long* sums) {
  const uint32_t lane = lane_id();
  const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  unsigned long long f1 = 0, r1 = 0, f2 = 0, r2 = 0;
  for (uint32_t u = w0; u < g.n; u += nw) {
    const uint32_t b = g.row[u], e = g.row[u + 1];
    for (uint32_t j = b + lane; j < e; j += 32) {
      const uint32_t v = g.dst[j];
      const unsigned long long fw = ((unsigned long long)u << 32) | v, rv = ((unsigned long long)v << 32) | u;
      f1 += mix64(fw);
      r1 += mix64(rv);
      f2 += mix64(fw ^ 0x5851f42d4c957f2dull);
      r2 += mix64(rv ^ 0x5851f42d4c957f2dull);
    }
  }
  f1 = warp_sum_u64(f1);
  r1 = warp_sum_u64(r1);
  f2 = warp_sum_u64(f2);
  r2 = warp_sum_u64(r2);
  if (lane == 0) {
    atomicAdd(sums + 0, f1);
    atomicAdd(sums + 1, r1);
    atomicAdd(sums + 2, f2);
    atomicAdd(sums + 3, r2);
  }
}

// Edge-weight statistics: minimum, maximum (as order-preserving unsigned keys)
// and the int64 sum.  Grid-stride over the weights.
__global__ void __launch_bounds__(256) edge_weight_stats_kernel(const int32_t* __restrict__ w, uint64_t m,
                                                                unsigned long long* out) {
  uint32_t lo = 0xffffffffu, hi = 0;
  long long sum = 0;
  for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < m; j += (uint64_t)gridDim.x * blockDim.x) {
    const int32_t x = w[j];
    const uint32_t key = (uint32_t)x ^ 0x80000000u;  // signed order as unsigned order
    lo = min(lo, key);
    hi = max(hi, key);
    sum += x;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
  }
  if (lane_id() == 0) {
    atomicMin(out + 0, (unsigned long long)lo);
    atomicMax(out + 1, (unsigned long long)hi);
    atomicAdd(out + 2, (unsigned long long)sum);
  }
}

// The gather floor of a pull pass: every edge's x/deg[dst[j]] gathered
// edge-parallel (grid-stride, eight loads in flight per thread, no per-vertex
// bookkeeping), through L1 (L1 != 0) or L2 only.  Measures what the random
// gathers alone cost on this graph (gsrb_probe_gather).
template <int L1>
__global__ void __launch_bounds__(512) gather_probe_kernel(const uint32_t* __restrict__ dst, uint64_t m,
                                                           const float* cin, double* sink) {
  double s = 0.0;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
  for (; j + 7 * stride < m; j += 8 * stride) {
    uint32_t d[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) d[k] = __ldg(dst + j + k * stride);
    float c[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) c[k] = L1 ? __ldca(cin + d[k]) : __ldcg(cin + d[k]);
#pragma unroll
    for (int k = 0; k < 8; ++k) s += (double)c[k];
  }
  for (; j < m; j += stride) s += (double)(L1 ? __ldca(cin + dst[j]) : __ldcg(cin + dst[j]));
  if (s == -1.0) *sink = s;  // keeps the loads; never true for non-negative inputs
}

gsrb_status_t graph_scratch(gsrb_graph* G) {
  const size_t n = G->n;
  cudaError_t e = cudaSuccess;
  for (int k = 0; k < 2 && !e; ++k) {
    // 4n words: BFS keeps an edge range (two words) per queue slot, and up to
    // 2n slots (entries plus reservation holes)
    e = dalloc(&G->q[k], 4 * n);
    if (!e) e = dalloc(&G->hq[k], 2 * n);
    if (!e) e = dalloc(&G->far[k], n);
    if (!e) e = dalloc(&G->contrib[k], n);
  }
  if (!e) e = dalloc(&G->mark, n);
  if (!e) e = dalloc(&G->fmark, n);
  if (!e) e = dalloc(&G->cnt, 3);
  if (!e) e = dalloc(&G->fcnt, 2);
  if (!e) e = dalloc(&G->flags, 32);
  G->trace_cap = 1u << 16;
  if (!e) e = dalloc(&G->trace, G->trace_cap);
  if (!e) e = dalloc(&G->mlp, 1);
  if (!e) e = cudaMemset(G->mlp, 0, sizeof(MLPWeights));
  if (!e) e = dalloc(&G->lb_pre, 2 * n);  // one per queue slot (holes included)
  if (!e) e = dalloc(&G->lb_own, (size_t)G->m / kLbChunk + 2);
  if (!e) e = dalloc(&G->lb_part, kLbMaxCtas);
  // PageRank hub chunks (degree > kPrHubDegree), built on the host from row_start
  if (!e) {
    std::vector<uint32_t>& hrow = G->h_row;
    hrow.assign(n + 1, 0u);
    e = cudaMemcpy(hrow.data(), G->row, sizeof(uint32_t) * (n + 1), cudaMemcpyDeviceToHost);
    std::vector<uint32_t> hl, c0, ch;
    for (size_t v = 0; !e && v < n; ++v) {
      const uint32_t d = hrow[v + 1] - hrow[v];
      if (d > G->max_degree) G->max_degree = d;
      if (d <= kPrHubDegree) continue;
      c0.push_back((uint32_t)ch.size());
      for (uint32_t j = 0; j < d; j += kPrChunk) ch.push_back((uint32_t)hl.size());
      hl.push_back((uint32_t)v);
    }
    c0.push_back((uint32_t)ch.size());
    G->nhubs = (uint32_t)hl.size();
    G->nchunks = (uint32_t)ch.size();
    if (!e) e = dalloc(&G->hubs, hl.size());
    if (!e) e = dalloc(&G->hub_c0, c0.size());
    if (!e) e = dalloc(&G->chunk_hub, ch.size());
    if (!e) e = dalloc(&G->hub_part, ch.size());
    if (!e) e = dalloc(&G->hub_done, hl.size());
    if (!e && !hl.empty()) e = cudaMemcpy(G->hubs, hl.data(), sizeof(uint32_t) * hl.size(), cudaMemcpyHostToDevice);
    if (!e) e = cudaMemcpy(G->hub_c0, c0.data(), sizeof(uint32_t) * c0.size(), cudaMemcpyHostToDevice);
    if (!e && !ch.empty())
      e = cudaMemcpy(G->chunk_hub, ch.data(), sizeof(uint32_t) * ch.size(), cudaMemcpyHostToDevice);
  }
  // symmetric? (pull directions and pull PageRank read a row as in-edges)
  if (!e) {
    unsigned long long* sums = reinterpret_cast<unsigned long long*>(G->lb_part);
    e = cudaMemset(sums, 0, 4 * sizeof(unsigned long long));
    if (!e) {
      edge_hash_kernel<<<1184, 256>>>(dev_csr(G), sums);
      e = cudaGetLastError();
    }
    unsigned long long h[4] = {0, 0, 0, 0};
    if (!e) e = cudaMemcpy(h, sums, sizeof h, cudaMemcpyDeviceToHost);
    G->symmetric = h[0] == h[1] && h[2] == h[3];
  }
  // edge weights: minimum, maximum, mean
  if (!e && G->w && G->m) {
    unsigned long long* st = reinterpret_cast<unsigned long long*>(G->lb_part);
    const unsigned long long init[3] = {0xffffffffull, 0ull, 0ull};
    e = cudaMemcpy(st, init, sizeof init, cudaMemcpyHostToDevice);
    if (!e) {
      edge_weight_stats_kernel<<<1184, 256>>>(G->w, G->m, st);
      e = cudaGetLastError();
    }
    unsigned long long h[3] = {0, 0, 0};
    if (!e) e = cudaMemcpy(h, st, sizeof h, cudaMemcpyDeviceToHost);
    G->w_min = (int32_t)((uint32_t)h[0] ^ 0x80000000u);
    G->w_max = (int32_t)((uint32_t)h[1] ^ 0x80000000u);
    G->w_mean = (double)(long long)h[2] / (double)G->m;
  }
  if (!e) e = cudaDeviceSynchronize();
  if (e) return cuda_err(e, "graph scratch");
  return GSRB_OK;
}

void graph_free(gsrb_graph* G) {
  if (G->owns) {
    cudaFree(G->row);
    cudaFree(G->dst);
    cudaFree(G->w);
  }
  for (int k = 0; k < 2; ++k) {
    cudaFree(G->q[k]);
    cudaFree(G->hq[k]);
    cudaFree(G->far[k]);
    cudaFree(G->contrib[k]);
  }
  cudaFree(G->mark);
  cudaFree(G->fmark);
  cudaFree(G->cnt);
  cudaFree(G->fcnt);
  cudaFree(G->flags);
  cudaFree(G->trace);
  cudaFree(G->hubs);
  cudaFree(G->hub_c0);
  cudaFree(G->chunk_hub);
  cudaFree(G->hub_part);
  cudaFree(G->hub_done);
  cudaFree(G->mlp);
  cudaFree(G->lb_pre);
  cudaFree(G->lb_own);
  cudaFree(G->lb_part);
}


gsrb_cfg_t graph_cfg(gsrb_ctx* ctx, const gsrb_cfg_t* in) {
  gsrb_cfg_t c = resolve_cfg(ctx, in);
  if (!in) {
    c.ctas_per_sm = 2;
    c.threads = 512;
    c.cluster = 2;
  }
  return c;
}

gsrb_status_t finish_stats(gsrb_graph* G, gsrb_traversal_stats_t* st, float ms) {
  uint32_t h[32];
  unsigned long long edges = 0;
  GSRB_CUDA(cudaStreamSynchronize(G->ctx->stream));
  GSRB_CUDA(cudaMemcpy(h, G->flags, sizeof(h), cudaMemcpyDeviceToHost));
  GSRB_CUDA(cudaMemcpy(&edges, (char*)G->flags + 64, sizeof(edges), cudaMemcpyDeviceToHost));
  if (st) {
    st->levels = h[4];
    st->aux = h[5];
    st->decisions = h[6];
    st->edges = edges;
    st->kernel_ms = ms;
    st->trace_records = h[4] < G->trace_cap ? h[4] : G->trace_cap;
    st->launch = 0;
    st->delta = G->last_delta;
  }
  if (h[0]) return GSRB_ERR_OVERFLOW;
  if (h[7]) return GSRB_ERR_TIMEOUT;
  return GSRB_OK;
}

}  // namespace

extern "C" {

gsrb_status_t gsrb_graph_upload(gsrb_ctx_t ctx, const gsrb_host_csr_t* h, gsrb_graph_t* out) {
  if (!ctx || !h || !out || !h->row_start || (h->nedges && !h->edge_dst) || h->nedges >= (1ull << 32))
    return GSRB_ERR_ARG;
  gsrb_graph* G = new gsrb_graph();
  G->ctx = ctx;
  G->n = h->nnodes;
  G->m = (uint32_t)h->nedges;
  G->owns = true;
  cudaError_t e = dalloc(&G->row, (size_t)G->n + 1);
  if (!e) e = dalloc(&G->dst, G->m);
  if (!e) e = dalloc(&G->w, G->m);
  if (!e) e = cudaMemcpy(G->row, h->row_start, sizeof(uint32_t) * ((size_t)G->n + 1), cudaMemcpyHostToDevice);
  if (!e && G->m) e = cudaMemcpy(G->dst, h->edge_dst, sizeof(uint32_t) * G->m, cudaMemcpyHostToDevice);
  if (!e && G->m && h->edge_data) e = cudaMemcpy(G->w, h->edge_data, sizeof(int32_t) * G->m, cudaMemcpyHostToDevice);
  gsrb_status_t st = e ? cuda_err(e, "graph upload") : graph_scratch(G);
  if (st) {
    graph_free(G);
    delete G;
    return st;
  }
  *out = G;
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_wrap(gsrb_ctx_t ctx, uint32_t n, uint64_t m, const uint32_t* d_row, const uint32_t* d_dst,
                              const int32_t* d_w, gsrb_graph_t* out) {
  if (!ctx || !out || !d_row || (m && !d_dst) || m >= (1ull << 32)) return GSRB_ERR_ARG;
  gsrb_graph* G = new gsrb_graph();
  G->ctx = ctx;
  G->n = n;
  G->m = (uint32_t)m;
  G->owns = false;
  G->row = const_cast<uint32_t*>(d_row);
  G->dst = const_cast<uint32_t*>(d_dst);
  G->w = const_cast<int32_t*>(d_w);
  gsrb_status_t st = graph_scratch(G);
  if (st) {
    graph_free(G);
    delete G;
    return st;
  }
  *out = G;
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_free(gsrb_graph_t G) {
  if (!G) return GSRB_ERR_ARG;
  cudaStreamSynchronize(G->ctx->stream);
  graph_free(G);
  delete G;
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_info(gsrb_graph_t G, uint32_t* n, uint64_t* m, uint32_t* nhubs) {
  if (!G) return GSRB_ERR_ARG;
  if (n) *n = G->n;
  if (m) *m = G->m;
  if (nhubs) *nhubs = G->nhubs;
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_is_symmetric(gsrb_graph_t G, int32_t* symmetric) {
  if (!G || !symmetric) return GSRB_ERR_ARG;
  *symmetric = G->symmetric ? 1 : 0;
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_set_policy(gsrb_graph_t G, const float* h_weights, size_t count) {
  if (!G || !h_weights || count != sizeof(MLPWeights) / sizeof(float)) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaMemcpy(G->mlp, h_weights, sizeof(MLPWeights), cudaMemcpyHostToDevice));
  memcpy(&G->mlp_host, h_weights, sizeof(MLPWeights));
  G->mlp_set = true;
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_set_launch_choices(gsrb_graph_t G, const gsrb_cfg_t* cfg0, const gsrb_cfg_t* cfg1) {
  if (!G) return GSRB_ERR_ARG;
  if (!cfg0 && !cfg1) {
    G->launch_set = false;
    return GSRB_OK;
  }
  if (!cfg0 || !cfg1) return GSRB_ERR_ARG;
  const gsrb_cfg_t* in[2] = {cfg0, cfg1};
  for (int k = 0; k < 2; ++k) {
    const gsrb_cfg_t c = graph_cfg(G->ctx, in[k]);
    if (!bfs_fn(c.variant)) return GSRB_ERR_UNSUPPORTED;
    const int grid = grid_of(G->ctx, c);
    if (grid <= 0 || grid % c.cluster || c.threads % 32 || c.threads > kGraphMaxThreads) return GSRB_ERR_ARG;
    G->launch[k] = c;
  }
  G->launch_set = true;
  return GSRB_OK;
}

namespace {

// Host forward pass of the policy network (the layout of MLPWeights; ReLU on
// the two hidden layers).  Used for the per-traversal launch choice, which is
// taken before the launch.
void mlp_forward_host(const MLPWeights& W, const float* x, float* out) {
  float h1[kHid], h2[kHid];
  for (int j = 0; j < kHid; ++j) {
    float z = W.b1[j];
    for (int i = 0; i < kFeat; ++i) z += W.w1[j][i] * x[i];
    h1[j] = z > 0.f ? z : 0.f;
  }
  for (int j = 0; j < kHid; ++j) {
    float z = W.b2[j];
    for (int k = 0; k < kHid; ++k) z += W.w2[j][k] * h1[k];
    h2[j] = z > 0.f ? z : 0.f;
  }
  for (int o = 0; o < kOut; ++o) {
    float z = W.b3[o];
    for (int k = 0; k < kHid; ++k) z += W.w3[o][k] * h2[k];
    out[o] = z;
  }
}

}  // namespace

gsrb_status_t gsrb_graph_policy_launch(gsrb_graph_t G, uint32_t src, int32_t* choice, float* score) {
  if (!G || !choice || src >= G->n) return GSRB_ERR_ARG;
  if (!G->mlp_set) return GSRB_ERR_STATE;
  // the first level's features, as the traversal computes them: the frontier
  // is the source, every other vertex and edge is unvisited
  const uint32_t dsrc = G->h_row[src + 1] - G->h_row[src];
  float feat[kFeat], out[kOut];
  level_features(feat, G->n, G->m, 1, 1, dsrc, G->n - 1, (unsigned long long)G->m - dsrc, 1, DIR_PUSH);
  mlp_forward_host(G->mlp_host, feat, out);
  *choice = out[3] > 0.f ? 1 : 0;
  if (score) *score = out[3];
  return GSRB_OK;
}

// The SSSP policy's 12 features of a traversal from a source: graph size,
// degree distribution, edge-weight range and the source's degree (log-scaled).
static void sssp_features_of(uint32_t n, uint64_t m, uint32_t max_degree, uint32_t src_degree, double w_mean,
                             int32_t w_min, int32_t w_max, int32_t symmetric, float* f) {
  const double nn = n ? (double)n : 1.0;
  const double md = (double)m / nn;
  f[0] = (float)log2(nn);
  f[1] = (float)log2(1.0 + (double)m);
  f[2] = (float)log2(1.0 + md);
  f[3] = (float)log2(1.0 + (double)max_degree);
  f[4] = (float)log2(1.0 + (double)src_degree);
  f[5] = (float)log2(1.0 + (w_mean > 0 ? w_mean : 0.0));
  f[6] = (float)log2(1.0 + (w_max > 0 ? (double)w_max : 0.0));
  f[7] = (float)log2(1.0 + (w_min > 0 ? (double)w_min : 0.0));
  f[8] = symmetric ? 1.f : 0.f;
  f[9] = f[3] - f[2];            // degree skew
  f[10] = f[6] - f[5];           // weight spread
  f[11] = f[0] - 2.f * f[2];     // size against mean degree (high for meshes)
}

void gsrb_sssp_features(uint32_t n, uint64_t m, uint32_t max_degree, uint32_t src_degree, double w_mean,
                        int32_t w_min, int32_t w_max, int32_t symmetric, float* h_out12) {
  sssp_features_of(n, m, max_degree, src_degree, w_mean, w_min, w_max, symmetric, h_out12);
}

gsrb_status_t gsrb_graph_sssp_features(gsrb_graph_t G, uint32_t src, float* h_out12) {
  if (!G || !h_out12 || src >= G->n) return GSRB_ERR_ARG;
  sssp_features_of(G->n, G->m, G->max_degree, G->h_row[src + 1] - G->h_row[src], G->w_mean, G->w_min, G->w_max,
                   G->symmetric ? 1 : 0, h_out12);
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_set_sssp_policy(gsrb_graph_t G, const float* h_weights, size_t count) {
  if (!G) return GSRB_ERR_ARG;
  if (!h_weights) {
    G->sssp_set = false;
    return GSRB_OK;
  }
  if (count != sizeof(MLPWeights) / sizeof(float)) return GSRB_ERR_ARG;
  memcpy(&G->sssp_host, h_weights, sizeof(MLPWeights));
  G->sssp_set = true;
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_sssp_plan(gsrb_graph_t G, uint32_t src, int32_t* delta, int32_t* choice, float* scores) {
  if (!G || src >= G->n) return GSRB_ERR_ARG;
  if (!G->sssp_set) return GSRB_ERR_STATE;
  float feat[kFeat], out[kOut];
  gsrb_status_t st = gsrb_graph_sssp_features(G, src, feat);
  if (st) return st;
  mlp_forward_host(G->sssp_host, feat, out);
  // head 2: log2(bucket width / mean edge weight)
  const double wm = G->w_mean >= 1.0 ? G->w_mean : 1.0;
  double d = exp2((double)(out[2] < -30.f ? -30.f : (out[2] > 30.f ? 30.f : out[2]))) * wm;
  if (!(d >= 1.0)) d = 1.0;
  if (d > 1073741824.0) d = 1073741824.0;
  if (delta) *delta = (int32_t)llround(d);
  if (choice) *choice = out[3] > 0.f ? 1 : 0;
  if (scores) {
    scores[0] = out[2];
    scores[1] = out[3];
  }
  return GSRB_OK;
}

gsrb_status_t gsrb_probe_gather(gsrb_ctx_t ctx, gsrb_graph_t G, int32_t l1, float* ms) {
  if (!ctx || !G || !ms) return GSRB_ERR_ARG;
  if (!G->m) {
    *ms = 0.f;
    return GSRB_OK;
  }
  std::lock_guard<std::mutex> g(ctx->mu);
  // x/deg of the first PageRank buffer (any FP32 values do; zeroed here)
  GSRB_CUDA(cudaMemsetAsync(G->contrib[0], 0, sizeof(float) * G->n, ctx->stream));
  double* sink = reinterpret_cast<double*>((char*)G->flags + 64);
  const dim3 grid((unsigned)ctx->num_sms * 2u), block(512);
  auto launch = [&]() -> cudaError_t {
    if (l1) gather_probe_kernel<1><<<grid, block, 0, ctx->stream>>>(G->dst, G->m, G->contrib[0], sink);
    else gather_probe_kernel<0><<<grid, block, 0, ctx->stream>>>(G->dst, G->m, G->contrib[0], sink);
    return cudaGetLastError();
  };
  if (!ctx->events[62]) GSRB_CUDA(cudaEventCreate(&ctx->events[62]));
  if (!ctx->events[63]) GSRB_CUDA(cudaEventCreate(&ctx->events[63]));
  for (int i = 0; i < 3; ++i) GSRB_CUDA(launch());
  constexpr int kReps = 10;
  GSRB_CUDA(cudaEventRecord(ctx->events[62], ctx->stream));
  for (int i = 0; i < kReps; ++i) GSRB_CUDA(launch());
  GSRB_CUDA(cudaEventRecord(ctx->events[63], ctx->stream));
  GSRB_CUDA(cudaEventSynchronize(ctx->events[63]));
  float t = 0;
  GSRB_CUDA(cudaEventElapsedTime(&t, ctx->events[62], ctx->events[63]));
  *ms = t / kReps;
  gsrbrt::g_launches.fetch_add(3 + kReps, std::memory_order_relaxed);
  return GSRB_OK;
}

gsrb_status_t gsrb_graph_trace(gsrb_graph_t G, void* h_out, uint32_t max_records, uint32_t* records) {
  if (!G || !h_out) return GSRB_ERR_ARG;
  uint32_t h[32];
  GSRB_CUDA(cudaStreamSynchronize(G->ctx->stream));
  GSRB_CUDA(cudaMemcpy(h, G->flags, sizeof(h), cudaMemcpyDeviceToHost));
  uint32_t r = h[4] < G->trace_cap ? h[4] : G->trace_cap;
  if (r > max_records) r = max_records;
  if (r) GSRB_CUDA(cudaMemcpy(h_out, G->trace, sizeof(LevelTrace) * r, cudaMemcpyDeviceToHost));
  if (records) *records = r;
  return GSRB_OK;
}

gsrb_status_t gsrb_bfs(gsrb_ctx_t ctx, gsrb_graph_t G, uint32_t src, int32_t* d_level, int32_t mode,
                       const gsrb_cfg_t* cfgin, gsrb_traversal_stats_t* stats) {
  const bool lb = (mode & GSRB_BFS_FLAG_LB) != 0;
  mode &= ~GSRB_BFS_FLAG_LB;
  if (!ctx || !G || !d_level || src >= G->n || mode < 0 || mode > GSRB_BFS_TOPO) return GSRB_ERR_ARG;
  if (mode == GSRB_BFS_LEARNED && !G->mlp_set) return GSRB_ERR_STATE;
  if (mode == GSRB_BFS_PULL && !G->symmetric) return GSRB_ERR_UNSUPPORTED;
  gsrb_cfg_t c = graph_cfg(ctx, cfgin);
  uint32_t launch = 0;
  if (mode == GSRB_BFS_LEARNED && !cfgin && G->launch_set) {
    // the policy's head 3 picks the launch configuration (barrier variant and
    // CTA shape) from the first level's features
    int32_t k = 0;
    gsrb_status_t st = gsrb_graph_policy_launch(G, src, &k, nullptr);
    if (st) return st;
    c = G->launch[k];
    launch = 1u + (uint32_t)k;
  }
  const void* fn = bfs_fn(c.variant);
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster || c.threads % 32 || c.threads > kGraphMaxThreads) return GSRB_ERR_ARG;
  if (lb && grid > (int)kLbMaxCtas) return GSRB_ERR_ARG;
  BfsArgs a;
  a.symmetric = G->symmetric;
  a.lb = lb;
  a.lb_pre = G->lb_pre;
  a.lb_own = G->lb_own;
  a.lb_part = G->lb_part;
  a.g = dev_csr(G);
  a.src = src;
  a.level = d_level;
  a.q[0] = G->q[0];
  a.q[1] = G->q[1];
  a.hq[0] = G->hq[0];
  a.hq[1] = G->hq[1];
  a.cnt = G->cnt;
  a.overflow = G->flags;
  a.trace = G->trace;
  a.trace_cap = G->trace_cap;
  a.mlp = G->mlp;
  a.mode = mode;
  a.alpha = 15.f;
  a.beta = 18.f;
  a.out = G->flags + 4;
  a.out_edges = (unsigned long long*)((char*)G->flags + 64);
  a.solo = G->flags + 8;
  G->last_delta = 0;
  std::lock_guard<std::mutex> g(ctx->mu);
  GSRB_CUDA(cudaMemsetAsync(G->flags, 0, 128, ctx->stream));
  gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)grid, 0, 0);
  void* args[] = {&gb, &a};
  if (!ctx->events[62]) GSRB_CUDA(cudaEventCreate(&ctx->events[62]));
  if (!ctx->events[63]) GSRB_CUDA(cudaEventCreate(&ctx->events[63]));
  GSRB_CUDA(cudaEventRecord(ctx->events[62], ctx->stream));
  gsrb_status_t st = launch_persistent(ctx, fn, grid, c.threads, 0, c.cluster, coop_of(c), args);
  if (st) return st;
  GSRB_CUDA(cudaEventRecord(ctx->events[63], ctx->stream));
  GSRB_CUDA(cudaEventSynchronize(ctx->events[63]));
  float ms = 0;
  GSRB_CUDA(cudaEventElapsedTime(&ms, ctx->events[62], ctx->events[63]));
  st = finish_stats(G, stats, ms);
  if (stats) stats->launch = launch;
  return st;
}

gsrb_status_t gsrb_sssp(gsrb_ctx_t ctx, gsrb_graph_t G, uint32_t src, int32_t* d_dist, int32_t delta,
                        const gsrb_cfg_t* cfgin, gsrb_traversal_stats_t* stats) {
  if (!ctx || !G || !d_dist || src >= G->n || delta < 0) return GSRB_ERR_ARG;
  gsrb_cfg_t c = graph_cfg(ctx, cfgin);
  uint32_t launch = 0;
  if (delta == GSRB_SSSP_DELTA_LEARNED) {
    // the SSSP policy picks the bucket width and, without a cfg, the launch
    // configuration; both change the schedule, never the distances
    int32_t k = 0;
    gsrb_status_t st = gsrb_graph_sssp_plan(G, src, &delta, &k, nullptr);
    if (st) return st;
    if (!cfgin && G->launch_set) {
      c = G->launch[k];
      launch = 1u + (uint32_t)k;
    }
  }
  const void* fn = sssp_fn(c.variant);
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster || c.threads % 32) return GSRB_ERR_ARG;
  SsspArgs a;
  a.g = dev_csr(G);
  a.src = src;
  a.dist = d_dist;
  for (int k = 0; k < 2; ++k) {
    a.q[k] = G->q[k];
    a.hq[k] = G->hq[k];
    a.far[k] = G->far[k];
  }
  a.mark = G->mark;
  a.fmark = G->fmark;
  a.cnt = G->cnt;
  a.fcnt = G->fcnt;
  a.overflow = G->flags;
  a.trace = G->trace;
  a.trace_cap = G->trace_cap;
  a.delta = delta;
  a.out = G->flags + 4;
  a.out_edges = (unsigned long long*)((char*)G->flags + 64);
  G->last_delta = delta;
  std::lock_guard<std::mutex> g(ctx->mu);
  GSRB_CUDA(cudaMemsetAsync(G->flags, 0, 128, ctx->stream));
  gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)grid, 0, 0);
  void* args[] = {&gb, &a};
  if (!ctx->events[62]) GSRB_CUDA(cudaEventCreate(&ctx->events[62]));
  if (!ctx->events[63]) GSRB_CUDA(cudaEventCreate(&ctx->events[63]));
  GSRB_CUDA(cudaEventRecord(ctx->events[62], ctx->stream));
  gsrb_status_t st = launch_persistent(ctx, fn, grid, c.threads, 0, c.cluster, coop_of(c), args);
  if (st) return st;
  GSRB_CUDA(cudaEventRecord(ctx->events[63], ctx->stream));
  GSRB_CUDA(cudaEventSynchronize(ctx->events[63]));
  float ms = 0;
  GSRB_CUDA(cudaEventElapsedTime(&ms, ctx->events[62], ctx->events[63]));
  st = finish_stats(G, stats, ms);
  if (stats) stats->launch = launch;
  return st;
}

gsrb_status_t gsrb_pagerank(gsrb_ctx_t ctx, gsrb_graph_t G, float alpha, int32_t iters, float* d_rank,
                            const gsrb_cfg_t* cfgin, gsrb_traversal_stats_t* stats) {
  if (!ctx || !G || !d_rank || iters < 0 || !(alpha >= 0.f && alpha < 1.f)) return GSRB_ERR_ARG;
  if (!G->symmetric) return GSRB_ERR_UNSUPPORTED;  // a row is summed as the vertex's in-edges
  gsrb_cfg_t c = graph_cfg(ctx, cfgin);
  const void* fn = pr_fn(c.variant);
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster || c.threads % 32 || grid > 148 * 32) return GSRB_ERR_ARG;
  PrArgs a;
  a.g = dev_csr(G);
  a.alpha = alpha;
  a.iters = iters;
  a.rank = d_rank;
  a.contrib[0] = G->contrib[0];
  a.contrib[1] = G->contrib[1];
  a.hubs = G->hubs;
  a.hub_c0 = G->hub_c0;
  a.chunk_hub = G->chunk_hub;
  a.nhubs = G->nhubs;
  a.nchunks = G->nchunks;
  a.part = G->hub_part;
  a.hub_done = G->hub_done;
  a.ticket = reinterpret_cast<unsigned long long*>(G->flags + 24);
  a.out = G->flags + 4;
  a.gather_l1 = c.form == GSRB_FORM_L2 ? 0 : 1;
  G->last_delta = 0;
  std::lock_guard<std::mutex> g(ctx->mu);
  GSRB_CUDA(cudaMemsetAsync(G->flags, 0, 128, ctx->stream));
  if (G->nhubs) GSRB_CUDA(cudaMemsetAsync(G->hub_done, 0, sizeof(uint32_t) * G->nhubs, ctx->stream));
  gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)grid, 0, 0);
  void* args[] = {&gb, &a};
  if (!ctx->events[62]) GSRB_CUDA(cudaEventCreate(&ctx->events[62]));
  if (!ctx->events[63]) GSRB_CUDA(cudaEventCreate(&ctx->events[63]));
  GSRB_CUDA(cudaEventRecord(ctx->events[62], ctx->stream));
  gsrb_status_t st = launch_persistent(ctx, fn, grid, c.threads, 0, c.cluster, coop_of(c), args);
  if (st) return st;
  GSRB_CUDA(cudaEventRecord(ctx->events[63], ctx->stream));
  GSRB_CUDA(cudaEventSynchronize(ctx->events[63]));
  float ms = 0;
  GSRB_CUDA(cudaEventElapsedTime(&ms, ctx->events[62], ctx->events[63]));
  return finish_stats(G, stats, ms);
}

gsrb_status_t gsrb_pagerank_residual(gsrb_ctx_t ctx, gsrb_graph_t G, float alpha, float epsilon, int32_t max_iters,
                                     float* d_rank, const gsrb_cfg_t* cfgin, gsrb_traversal_stats_t* stats) {
  if (!ctx || !G || !d_rank || max_iters < 0 || !(alpha >= 0.f && alpha < 1.f) || !(epsilon > 0.f))
    return GSRB_ERR_ARG;
  gsrb_cfg_t c = graph_cfg(ctx, cfgin);
  const void* fn = prr_fn(c.variant);
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  const int grid = grid_of(ctx, c);
  if (grid % c.cluster || c.threads % 32) return GSRB_ERR_ARG;
  PrrArgs a;
  a.g = dev_csr(G);
  a.alpha = alpha;
  a.eps = epsilon;
  a.max_iters = max_iters;
  a.p = d_rank;
  a.r = G->contrib[0];
  a.hub_upd = G->contrib[1];
  a.mark = G->mark;
  a.q[0] = G->q[0];
  a.q[1] = G->q[1];
  a.hq[0] = G->hq[0];
  a.hq[1] = G->hq[1];
  a.cnt = G->cnt;
  a.overflow = G->flags;
  a.out = G->flags + 4;
  a.out_edges = (unsigned long long*)((char*)G->flags + 64);
  G->last_delta = 0;
  std::lock_guard<std::mutex> g(ctx->mu);
  GSRB_CUDA(cudaMemsetAsync(G->flags, 0, 128, ctx->stream));
  gsrb::GridBarrier gb = make_barrier(ctx, c, 0, (uint32_t)grid, 0, 0);
  void* args[] = {&gb, &a};
  if (!ctx->events[62]) GSRB_CUDA(cudaEventCreate(&ctx->events[62]));
  if (!ctx->events[63]) GSRB_CUDA(cudaEventCreate(&ctx->events[63]));
  GSRB_CUDA(cudaEventRecord(ctx->events[62], ctx->stream));
  gsrb_status_t st = launch_persistent(ctx, fn, grid, c.threads, 0, c.cluster, coop_of(c), args);
  if (st) return st;
  GSRB_CUDA(cudaEventRecord(ctx->events[63], ctx->stream));
  GSRB_CUDA(cudaEventSynchronize(ctx->events[63]));
  float ms = 0;
  GSRB_CUDA(cudaEventElapsedTime(&ms, ctx->events[62], ctx->events[63]));
  return finish_stats(G, stats, ms);
}

}  // extern "C"

// ---------------------------------------------------------------- batches ----
struct gsrb_batch {
  gsrb_ctx* ctx = nullptr;
  std::vector<gsrb_graph*> graphs;
  gsrb_cfg_t cfg;
  int grid = 0;
  std::vector<uint32_t> first, count;
  BatchDesc* h_desc = nullptr;  // pinned
  BatchDesc* d_desc = nullptr;
  uint16_t* d_cta_inst = nullptr;
};

namespace {

BfsArgs bfs_args(gsrb_graph* G, uint32_t src, int32_t* level, int32_t mode) {
  BfsArgs a;
  a.g = dev_csr(G);
  a.src = src;
  a.level = level;
  a.q[0] = G->q[0];
  a.q[1] = G->q[1];
  a.hq[0] = G->hq[0];
  a.hq[1] = G->hq[1];
  a.cnt = G->cnt;
  a.overflow = G->flags;
  a.trace = G->trace;
  a.trace_cap = G->trace_cap;
  a.mlp = G->mlp;
  a.mode = mode;
  a.alpha = 15.f;
  a.beta = 18.f;
  a.out = G->flags + 4;
  a.out_edges = (unsigned long long*)((char*)G->flags + 64);
  a.solo = G->flags + 8;
  a.symmetric = G->symmetric;
  a.lb = false;
  a.lb_pre = G->lb_pre;
  a.lb_own = G->lb_own;
  a.lb_part = G->lb_part;
  return a;
}

SsspArgs sssp_args(gsrb_graph* G, uint32_t src, int32_t* dist, int32_t delta) {
  SsspArgs a;
  a.g = dev_csr(G);
  a.src = src;
  a.dist = dist;
  for (int k = 0; k < 2; ++k) {
    a.q[k] = G->q[k];
    a.hq[k] = G->hq[k];
    a.far[k] = G->far[k];
  }
  a.mark = G->mark;
  a.fmark = G->fmark;
  a.cnt = G->cnt;
  a.fcnt = G->fcnt;
  a.overflow = G->flags;
  a.trace = G->trace;
  a.trace_cap = G->trace_cap;
  a.delta = delta;
  a.out = G->flags + 4;
  a.out_edges = (unsigned long long*)((char*)G->flags + 64);
  return a;
}

gsrb_status_t batch_launch(gsrb_batch* B, const uint32_t* srcs, int32_t* const* outs, int kind, int32_t param) {
  if (!B || !srcs || !outs) return GSRB_ERR_ARG;
  const int k = (int)B->graphs.size();
  for (int i = 0; i < k; ++i)
    if (!outs[i] || srcs[i] >= B->graphs[i]->n) return GSRB_ERR_ARG;
  if (kind == 0 && param == GSRB_BFS_LEARNED)
    for (int i = 0; i < k; ++i)
      if (!B->graphs[i]->mlp_set) return GSRB_ERR_STATE;
  // SSSP with the learned bucket width: every instance its own (host-side
  // plan from the graph's statistics; nothing is read from the device)
  std::vector<int32_t> deltas((size_t)k, param);
  if (kind == 1 && param == GSRB_SSSP_DELTA_LEARNED)
    for (int i = 0; i < k; ++i) {
      gsrb_status_t st = gsrb_graph_sssp_plan(B->graphs[i], srcs[i], &deltas[i], nullptr, nullptr);
      if (st) return st;
    }
  gsrb_ctx* ctx = B->ctx;
  const void* fn = batch_fn(B->cfg.variant);
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> g(ctx->mu);
  for (int i = 0; i < k; ++i) {
    BatchDesc& d = B->h_desc[i];
    memset(&d, 0, sizeof(d));
    // slot 1 + i and, for the group-counter variants, groups starting at the
    // instance's first CTA (an instance never has more groups than CTAs)
    d.gb = make_barrier(ctx, B->cfg, 1 + i, B->count[i], B->first[i], B->first[i]);
    d.first = B->first[i];
    d.count = B->count[i];
    d.kind = (uint32_t)kind;
    if (kind == 0) {
      d.bfs = bfs_args(B->graphs[i], srcs[i], outs[i], param);
      B->graphs[i]->last_delta = 0;
    }
    else {
      d.sssp = sssp_args(B->graphs[i], srcs[i], outs[i], deltas[i]);
      B->graphs[i]->last_delta = deltas[i];
    }
    GSRB_CUDA(cudaMemsetAsync(B->graphs[i]->flags, 0, 128, ctx->stream));
  }
  GSRB_CUDA(cudaMemcpyAsync(B->d_desc, B->h_desc, sizeof(BatchDesc) * k, cudaMemcpyHostToDevice, ctx->stream));
  const BatchDesc* dd = B->d_desc;
  const uint16_t* ci = B->d_cta_inst;
  void* args[] = {(void*)&dd, (void*)&ci};
  return launch_persistent(ctx, fn, B->grid, B->cfg.threads, 0, 1, coop_of(B->cfg), args);
}

}  // namespace

extern "C" {

gsrb_status_t gsrb_batch_create(gsrb_ctx_t ctx, const gsrb_graph_t* graphs, int32_t k, const gsrb_cfg_t* cfgin,
                                gsrb_batch_t* out) {
  if (!ctx || !graphs || !out || k <= 0 || k > kSlots - 1) return GSRB_ERR_ARG;
  gsrb_cfg_t c = resolve_cfg(ctx, cfgin);
  if (!cfgin) {
    c.variant = gsrb::V_FANOUT;
    c.ctas_per_sm = 2;
    c.threads = 512;
  }
  c.cluster = 1;
  if (!batch_fn(c.variant)) return GSRB_ERR_UNSUPPORTED;
  if (c.threads % 32 || c.threads > kGraphMaxThreads) return GSRB_ERR_ARG;
  const int grid = grid_of(ctx, c);
  if (grid < k || grid > 65535) return GSRB_ERR_ARG;
  gsrb_batch* B = new gsrb_batch();
  B->ctx = ctx;
  B->cfg = c;
  B->grid = grid;
  for (int i = 0; i < k; ++i) {
    if (!graphs[i]) {
      delete B;
      return GSRB_ERR_ARG;
    }
    B->graphs.push_back(graphs[i]);
  }
  // CTAs in proportion to each instance's edges (+ vertices), at least one each
  std::vector<double> w(k);
  double W = 0;
  for (int i = 0; i < k; ++i) {
    w[i] = (double)graphs[i]->m + (double)graphs[i]->n;
    W += w[i];
  }
  std::vector<uint32_t> cnt(k, 1);
  int left = grid - k;
  std::vector<std::pair<double, int>> rem;
  for (int i = 0; i < k; ++i) {
    const double share = W > 0 ? left * w[i] / W : 0.0;
    const uint32_t extra = (uint32_t)share;
    cnt[i] += extra;
    rem.push_back({share - extra, i});
  }
  int used = 0;
  for (int i = 0; i < k; ++i) used += (int)cnt[i];
  std::sort(rem.begin(), rem.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
    return a.first > b.first || (a.first == b.first && a.second < b.second);
  });
  for (size_t j = 0; used < grid && j < rem.size(); ++j, ++used) cnt[rem[j].second] += 1;
  std::vector<uint16_t> inst(grid);
  uint32_t f = 0;
  for (int i = 0; i < k; ++i) {
    B->first.push_back(f);
    B->count.push_back(cnt[i]);
    for (uint32_t j = 0; j < cnt[i]; ++j) inst[f + j] = (uint16_t)i;
    f += cnt[i];
  }
  cudaError_t e = cudaMallocHost(&B->h_desc, sizeof(BatchDesc) * k);
  if (!e) e = cudaMalloc(&B->d_desc, sizeof(BatchDesc) * k);
  if (!e) e = cudaMalloc(&B->d_cta_inst, sizeof(uint16_t) * grid);
  if (!e) e = cudaMemcpy(B->d_cta_inst, inst.data(), sizeof(uint16_t) * grid, cudaMemcpyHostToDevice);
  if (e) {
    gsrb_batch_free(B);
    return cuda_err(e, "batch_create");
  }
  *out = B;
  return GSRB_OK;
}

gsrb_status_t gsrb_batch_free(gsrb_batch_t B) {
  if (!B) return GSRB_ERR_ARG;
  if (B->ctx) cudaStreamSynchronize(B->ctx->stream);
  if (B->h_desc) cudaFreeHost(B->h_desc);
  if (B->d_desc) cudaFree(B->d_desc);
  if (B->d_cta_inst) cudaFree(B->d_cta_inst);
  delete B;
  return GSRB_OK;
}

gsrb_status_t gsrb_batch_layout(gsrb_batch_t B, uint32_t* first, uint32_t* count) {
  if (!B) return GSRB_ERR_ARG;
  for (size_t i = 0; i < B->graphs.size(); ++i) {
    if (first) first[i] = B->first[i];
    if (count) count[i] = B->count[i];
  }
  return GSRB_OK;
}

gsrb_status_t gsrb_batch_bfs(gsrb_batch_t B, const uint32_t* srcs, int32_t* const* d_levels, int32_t mode) {
  if (mode < 0 || mode > GSRB_BFS_TOPO) return GSRB_ERR_ARG;
  return batch_launch(B, srcs, d_levels, 0, mode);
}

gsrb_status_t gsrb_batch_sssp(gsrb_batch_t B, const uint32_t* srcs, int32_t* const* d_dists, int32_t delta) {
  if (delta < 0) return GSRB_ERR_ARG;
  return batch_launch(B, srcs, d_dists, 1, delta);
}

gsrb_status_t gsrb_batch_stats(gsrb_batch_t B, gsrb_traversal_stats_t* stats) {
  if (!B) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaStreamSynchronize(B->ctx->stream));
  gsrb_status_t worst = GSRB_OK;
  for (size_t i = 0; i < B->graphs.size(); ++i) {
    gsrb_status_t st = finish_stats(B->graphs[i], stats ? &stats[i] : nullptr, 0.f);
    if (st && !worst) worst = st;
  }
  return worst;
}

// ---- CUDA graphs: capture the context stream's work once, replay it ----------
gsrb_status_t gsrb_capture_begin(gsrb_ctx_t ctx) {
  if (!ctx) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  return GSRB_OK;
}

gsrb_status_t gsrb_capture_end(gsrb_ctx_t ctx, gsrb_exec_t* out) {
  if (!ctx || !out) return GSRB_ERR_ARG;
  cudaGraph_t graph = nullptr;
  GSRB_CUDA(cudaStreamEndCapture(ctx->stream, &graph));
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e) return cuda_err(e, "cudaGraphInstantiate");
  *out = (gsrb_exec_t)exec;
  return GSRB_OK;
}

gsrb_status_t gsrb_exec_launch(gsrb_ctx_t ctx, gsrb_exec_t exec) {
  if (!ctx || !exec) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaGraphLaunch((cudaGraphExec_t)exec, ctx->stream));
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return GSRB_OK;
}

gsrb_status_t gsrb_exec_free(gsrb_exec_t exec) {
  if (exec) GSRB_CUDA(cudaGraphExecDestroy((cudaGraphExec_t)exec));
  return GSRB_OK;
}

}  // extern "C"
