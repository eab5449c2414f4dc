// gsrb/barrier.cuh -- grid barriers for persistent kernels on sm_100a.
//
// Reference algorithms restated here (behaviour, not code):
//   * GSRB, the two-level sense-reversing barrier of the TPDS'22 artifact:
//     Heterosync/cudaLocksBarrierAtomicSRB.cu:63-236 and its application copy
//     Reduce/reduce_gsrb.cu:198-269 (group = blockIdx % min(grid, NUM_SM); the
//     last arriver of a group joins the global counter; everyone waits for the
//     global sense to flip).
//   * GCPUSRB, the one-level "CPU style" sense-reversing barrier:
//     Heterosync/cudaLocksBarrierAtomicSRB.cu:17-61 (naive = true in the apps,
//     e.g. Reduce/reduce_gcpusrb.cu).
//   * the HeteroSync atomic tree barrier used as the paper's baseline:
//     Heterosync/cudaLocksBarrierAtomic.cu:6-170 (two counters per level, no sense).
//   * CUDA cooperative groups grid.sync(): Heterosync/main.cu:127-133.
//
// The B200-native barrier (GSRB_CLUSTER and its siblings) has three levels:
//   CTA      -> __syncthreads (implied by the cluster barrier, which every thread joins)
//   cluster  -> hardware `barrier.cluster.arrive.release / wait.acquire`, or a
//               distributed-shared-memory arrival counter in the cluster leader
//   global   -> one arriving thread per cluster does `atom.acq_rel.gpu.add` (or
//               `red.release.gpu.add`) on an L2-resident counter, optionally
//               through a layer of sub-group counters (fan-in), and the barrier
//               completes when the generation word ("sense", kept as an epoch
//               counter so it never needs resetting) is bumped with a
//               `st.release.gpu`; waiters poll it with `ld.acquire.gpu`.
//
// Every wait is bounded by a %globaltimer deadline.  A wait that runs out records
// GSRB_DEV_TIMEOUT in the slot's status word (first error wins) and returns
// false; every other waiter notices the status word within 32 polls and returns
// false too, so all CTAs leave the kernel and the host reads the error.  Nothing
// traps, nothing spins forever.
#pragma once
#include <stdint.h>
#include <cooperative_groups.h>
#include "gsrb/ptx.cuh"

namespace gsrb {

// Device status codes written into BarrierSlot::status.
enum : uint32_t {
  GSRB_DEV_OK = 0,
  GSRB_DEV_TIMEOUT = 1,        // a bounded wait ran out
  GSRB_DEV_BAD_CONFIG = 2,     // kernel saw a launch shape it cannot serve
  GSRB_DEV_OVERFLOW = 3,       // a worklist or scratch area would overflow
  GSRB_DEV_LOCK_TIMEOUT = 4,   // mutex / semaphore wait ran out
  GSRB_DEV_INVARIANT = 5,      // a checked invariant failed (e.g. semaphore over-post)
};

// Barrier variants.  The numeric values are part of the C ABI (include/gsrb.h).
enum Variant : int {
  V_CLUSTER = 0,         // HW cluster barrier -> leader global -> HW cluster barrier release
  V_CLUSTER_ALLPOLL = 1, // HW cluster barrier -> leader global arrive; every CTA polls
  V_DSMEM = 2,           // DSMEM arrival counter -> leader global -> DSMEM release flags
  V_SOFT2 = 3,           // reference GSRB: software group counters -> global; all poll
  V_FLAT = 4,            // reference GCPUSRB: every CTA arrives at one counter; all poll
  V_TREE = 5,            // HeteroSync atomic tree barrier (two counters per level)
  V_CCG = 6,             // cooperative_groups::this_grid().sync()
  V_CLUSTER_RED = 7,     // HW cluster barrier -> red.release arrivals, master polls count
  V_FLIP = 8,            // no cluster level: every CTA arrives on the split flip words
  V_FANOUT = 9,          // one arrival counter, generation published to R wake-up lines
  V_CLUSTER_FANOUT = 10, // HW cluster arrival -> leader on the counter -> every CTA polls its wake-up line
  V_HIER = 11,           // group counters on separate lines -> root counter -> wake-up lines
  V_LOCKFREE = 12,       // HeteroSync lock-free tree barrier: in/out flag arrays, master CTA scans
  V_COUNT = 13
};

// One global barrier slot: four 128-byte lines so that the arrival counter, the
// generation word and the status word never share an L2 line.
struct __align__(128) BarrierSlot {
  uint32_t count;      // arrivals at the global level (reset by the completer)
  uint32_t _p0[31];
  uint32_t epoch;      // generation; bumped once per completed episode
  uint32_t _p1[31];
  uint32_t status;     // GSRB_DEV_* (first error wins)
  uint32_t where;      // episode index of the first error
  uint32_t who;        // block index that recorded it
  uint32_t _p2[29];
  uint32_t count2;     // second counter for the tree barrier
  uint32_t _p3[31];
};
static_assert(sizeof(BarrierSlot) == 512, "slot layout");

// A sub-group counter for fan-in combining (and for the per-SM level of the
// reference-style barriers).  Two lines: counter and a private generation.
struct __align__(128) GroupSlot {
  uint32_t count;
  uint32_t _p0[31];
  uint32_t count2;     // second counter (tree barrier local level)
  uint32_t _p1[31];
};
static_assert(sizeof(GroupSlot) == 256, "group layout");

// Launch-time parameters of one grid barrier (passed by value to kernels).
struct GridBarrier {
  BarrierSlot* slot;
  GroupSlot* groups;      // >= ngroups entries when ngroups > 0
  uint32_t nparticipants; // CTAs taking part (gridDim.x for whole-grid barriers)
  uint32_t first_cta;     // first participating block index (sub-grid barriers)
  uint32_t ngroups;       // global fan-in groups (0 = arrive directly at the root)
  uint32_t spin_ns;       // __nanosleep between polls (0 = hot spin)
  uint64_t timeout_ns;    // per-wait deadline
  uint32_t* flip;         // flip words of the native variants (word r at flip[32 r])
  uint32_t nflip;         // number of flip words in use (0 or 1 = one word)
  uint32_t _pad;
};

// Shared-memory words a CTA needs for the cluster / DSMEM levels.
struct BarrierShared {
  uint32_t arrive;   // DSMEM arrival counter (used in the cluster leader)
  uint32_t release;  // DSMEM release flag (epoch broadcast into every CTA)
  uint32_t ok;       // result broadcast
  uint32_t pad;
};

namespace detail {

__device__ __forceinline__ void record_error(const GridBarrier& gb, uint32_t code,
                                             uint32_t episode) {
  if (ptx::atom_cas_acq_rel_gpu(&gb.slot->status, 0u, code) == 0u) {
    ptx::st_relaxed_gpu(&gb.slot->where, episode);
    ptx::st_relaxed_gpu(&gb.slot->who, blockIdx.x);
  }
}

// Poll `*word` until it differs from `old`.  Bounded: returns false after the
// deadline (recording a timeout) or when another CTA has recorded an error.
__device__ __forceinline__ bool wait_ne(const uint32_t* word, uint32_t old,
                                        const GridBarrier& gb, uint32_t episode) {
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    if (ptx::ld_acquire_gpu(word) != old) return true;
    if ((it & 31u) == 31u) {
      if (ptx::ld_relaxed_gpu(&gb.slot->status) != 0u) return false;
      const uint64_t now = ptx::globaltimer_ns();
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > gb.timeout_ns) {
        record_error(gb, GSRB_DEV_TIMEOUT, episode);
        return false;
      }
    }
    if (gb.spin_ns) __nanosleep(gb.spin_ns);
  }
}

// Poll until `*word == want` (used by the red-arrival master and the tree barrier).
__device__ __forceinline__ bool wait_eq(const uint32_t* word, uint32_t want,
                                        const GridBarrier& gb, uint32_t episode) {
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    if (ptx::ld_acquire_gpu(word) == want) return true;
    if ((it & 31u) == 31u) {
      if (ptx::ld_relaxed_gpu(&gb.slot->status) != 0u) return false;
      const uint64_t now = ptx::globaltimer_ns();
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > gb.timeout_ns) {
        record_error(gb, GSRB_DEV_TIMEOUT, episode);
        return false;
      }
    }
    if (gb.spin_ns) __nanosleep(gb.spin_ns);
  }
}

// Number of arrivals (among `n` participants numbered 0..n-1) that land in
// fan-in group g when participant i belongs to group i % ngroups.
__device__ __forceinline__ uint32_t group_size(uint32_t n, uint32_t ngroups, uint32_t g) {
  return n / ngroups + (g < n % ngroups ? 1u : 0u);
}

// Global level, atom flavour: participant `idx` of `n` arrives; the completing
// arrival resets the counter(s) and bumps the epoch.  Returns true if this
// caller completed the episode (it need not wait).
__device__ __forceinline__ bool global_arrive_atom(const GridBarrier& gb, uint32_t idx,
                                                   uint32_t n, uint32_t epoch) {
  if (gb.ngroups > 1 && n > gb.ngroups) {
    const uint32_t g = idx % gb.ngroups;
    uint32_t* gc = &gb.groups[g].count;
    const uint32_t gs = group_size(n, gb.ngroups, g);
    if (ptx::atom_add_acq_rel_gpu(gc, 1u) != gs - 1u) return false;
    ptx::st_relaxed_gpu(gc, 0u);
    n = gb.ngroups;  // the root counts groups
  }
  if (ptx::atom_add_acq_rel_gpu(&gb.slot->count, 1u) != n - 1u) return false;
  ptx::st_relaxed_gpu(&gb.slot->count, 0u);
  ptx::st_release_gpu(&gb.slot->epoch, epoch + 1u);
  return true;
}

// ---- split "sum-to-flip" global level (the native variants) -----------------
// R flip words (R = min(nflip, n), nflip <= kFlipLines), each on its own
// 128-byte line in the first half of the slot's flip area (separate from the
// counters of the other protocols).  Arrival unit idx of n adds to word
// r = idx % R: the first unit of each word adds 0x80000000 - (count_r - 1),
// every other unit adds 1, so the word's top bit toggles exactly when its last
// arrival lands and its low bits return to their old value -- no completer, no
// reset store, and the arrivals are fire-and-forget `red.release.gpu.add`.
// Splitting the arrivals over R words divides the same-address serialisation
// at the L2 by R.  Each waiter keeps the top bit it expects of every word (a
// word's parity depends on how many episodes it has seen over earlier
// launches, so the words are tracked separately) and polls the words that have
// not flipped yet with `ld.acquire.gpu`.
constexpr uint32_t kFlipLines = 8;    // lines 0..7: flip words
constexpr uint32_t kFanoutBase = 8;   // lines 8..15: wake-up lines of the fan-out protocol
constexpr uint32_t kFanoutLines = 8;

__device__ __forceinline__ uint32_t* flip_word(const GridBarrier& gb, uint32_t r) { return gb.flip + r * 32u; }
__device__ __forceinline__ uint32_t flip_count(const GridBarrier& gb, uint32_t n) {
  uint32_t R = gb.nflip ? gb.nflip : 1u;
  if (R > kFlipLines) R = kFlipLines;
  return R < n ? R : n;
}

__device__ __forceinline__ void flip_arrive(const GridBarrier& gb, uint32_t idx, uint32_t n) {
  const uint32_t R = flip_count(gb, n);
  const uint32_t r = idx % R;
  const uint32_t cnt = group_size(n, R, r);
  const uint32_t inc = (idx == r) ? (0x80000000u - (cnt - 1u)) : 1u;
  ptx::red_add_release_gpu(flip_word(gb, r), inc);
}

// Bit r of the returned mask = the top bit word r will show after the next flip.
__device__ __forceinline__ uint32_t flip_expect_init(const GridBarrier& gb, uint32_t n) {
  const uint32_t R = flip_count(gb, n);
  uint32_t m = 0;
  for (uint32_t r = 0; r < R; ++r) m |= ((ptx::ld_acquire_gpu(flip_word(gb, r)) >> 31) ^ 1u) << r;
  return m;
}
__device__ __forceinline__ uint32_t flip_all(const GridBarrier& gb, uint32_t n) {
  return (1u << flip_count(gb, n)) - 1u;
}

// Wait until every word r in use shows top bit == bit r of `expect`.  Bounded.
__device__ __forceinline__ bool flip_wait(const GridBarrier& gb, uint32_t n, uint32_t expect, uint32_t episode) {
  const uint32_t R = flip_count(gb, n);
  uint64_t t0 = 0;
  uint32_t next = 0;  // words below `next` have flipped
  for (uint32_t it = 0;; ++it) {
    while (next < R && (ptx::ld_acquire_gpu(flip_word(gb, next)) >> 31) == ((expect >> next) & 1u)) ++next;
    if (next == R) return true;
    if ((it & 31u) == 31u) {
      if (ptx::ld_relaxed_gpu(&gb.slot->status) != 0u) return false;
      const uint64_t now = ptx::globaltimer_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > gb.timeout_ns) {
        record_error(gb, GSRB_DEV_TIMEOUT, episode);
        return false;
      }
    }
    if (gb.spin_ns) __nanosleep(gb.spin_ns);
  }
}

// ---- counter + fan-out wake-up lines (V_FANOUT, V_CLUSTER_FANOUT) -------------
// Arrivals (one per unit) go to the counter line slot->count with a release
// RMW (fence.acq_rel + relaxed atom); the unit whose arrival completes the
// episode resets the counter, then one fence.acq_rel acquires the other
// arrivals and orders the reset before the new generation, which it writes
// into all kFanoutLines wake-up lines (second half of the flip
// area; all of them, so they always hold the same value whatever R a later
// launch uses); unit u polls line u % R with ld.acquire.  Keeping the polled
// lines apart from the counter line means the polling loads never queue in
// front of the arrival atomics, and R lines divide the polling load per L2
// slice by R.  Returns true when this unit completed the episode.
__device__ __forceinline__ uint32_t* fanout_line(const GridBarrier& gb, uint32_t r) {
  return gb.flip + (kFanoutBase + r) * 32u;
}
__device__ __forceinline__ uint32_t fanout_count(const GridBarrier& gb) {
  uint32_t R = gb.nflip ? gb.nflip : 1u;
  return R > kFanoutLines ? kFanoutLines : R;
}
__device__ __forceinline__ bool fanout_arrive(const GridBarrier& gb, uint32_t n, uint32_t epoch) {
  ptx::fence_acq_rel_gpu();
  if (ptx::atom_add_relaxed_gpu(&gb.slot->count, 1u) != n - 1u) return false;
  // reset before the fence, so that the fence orders it before the generation
  // stores (a CTA that sees the new generation arrives on a reset counter)
  ptx::st_relaxed_gpu(&gb.slot->count, 0u);
  ptx::fence_acq_rel_gpu();
  for (uint32_t r = 0; r < kFanoutLines; ++r) ptx::st_relaxed_gpu(fanout_line(gb, r), epoch + 1u);
  return true;
}
__device__ __forceinline__ bool fanout_wait(const GridBarrier& gb, uint32_t unit, uint32_t epoch, uint32_t episode) {
  return wait_ne(fanout_line(gb, unit % fanout_count(gb)), epoch, gb, episode);
}

// ---- lock-free flag barrier (V_LOCKFREE) -------------------------------------
// The HeteroSync "lock-free" tree barrier (Heterosync/cudaLocksBarrierFast.cu:
// 182-330, after Xiao and Feng): member j sets in[j] = 1; the group's master
// (member 0) has its threads scan all in flags, then resets in[i] = 0 and sets
// out[i] = 1 (released); member j waits for out[j] = 1 and clears it.  Flags
// return to 0 after every episode, so the protocol is stateless across
// launches.  Restated with scoped ordering (the reference's plain volatile
// stores in=0 / out=1 are not ordered against each other) and bounded waits.
// `inner` runs in the whole master CTA after every member arrived and before
// any is released (the global level of the two-level form).
__device__ __forceinline__ bool lf_wait_eq(const uint32_t* word, uint32_t want, const GridBarrier& gb,
                                           uint32_t episode) {
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    if (ptx::ld_acquire_gpu(word) == want) return true;
    if ((it & 31u) == 31u) {
      if (ptx::ld_relaxed_gpu(&gb.slot->status) != 0u) return false;
      const uint64_t now = ptx::globaltimer_ns();
      if (t0 == 0) {
        t0 = now;
      } else if (now - t0 > gb.timeout_ns) {
        record_error(gb, GSRB_DEV_TIMEOUT, episode);
        return false;
      }
    }
  }
}
template <class Inner>
__device__ __forceinline__ bool lf_episode(uint32_t* in, uint32_t* out, uint32_t members, uint32_t j,
                                           const GridBarrier& gb, uint32_t episode, Inner inner) {
  __syncthreads();
  if (threadIdx.x == 0) {
    ptx::fence_acq_rel_gpu();
    ptx::st_relaxed_gpu(in + j, 1u);
  }
  bool ok = true;
  if (j == 0) {
    for (uint32_t i = threadIdx.x; i < members; i += blockDim.x) ok = lf_wait_eq(in + i, 1u, gb, episode) && ok;
    ok = __syncthreads_and(ok) != 0;
    if (ok) ok = inner();
    for (uint32_t i = threadIdx.x; i < members; i += blockDim.x) {
      ptx::st_relaxed_gpu(in + i, 0u);
      ptx::st_release_gpu(out + i, 1u);
    }
  }
  if (threadIdx.x == 0) {
    ok = lf_wait_eq(out + j, 1u, gb, episode) && ok;
    ptx::st_relaxed_gpu(out + j, 0u);
  }
  return __syncthreads_and(ok) != 0;
}
// Flag area layout (gb.flip points at it): global in / out arrays of
// kLfGlobal words, then per-group local in / out arrays of kLfLocal words.
constexpr uint32_t kLfGlobal = 8192, kLfGroups = 256, kLfLocal = 64;
constexpr size_t kLfWords = 2 * (size_t)kLfGlobal + 2 * (size_t)kLfGroups * kLfLocal;

// ---- two-level counters + wake-up lines (V_HIER) --------------------------------
// Unit u arrives on group counter u % G (each group counter on its own 256-byte
// line, so G groups spread the same-address serialisation over G L2 lines);
// the group's last arrival acquires and arrives on the root counter for the
// group; the root's last arrival resets the counters it completed and publishes
// the generation to every wake-up line.  Every RMW is a release (fence.acq_rel
// before a relaxed atom); a completer resets its counter and then fences, which
// acquires the arrivals it completed and orders the reset before its next
// arrival or the generation stores.
__device__ __forceinline__ bool hier_arrive(const GridBarrier& gb, uint32_t idx, uint32_t n, uint32_t epoch) {
  const uint32_t G = gb.ngroups;
  ptx::fence_acq_rel_gpu();
  if (G > 1 && n > G) {
    const uint32_t g = idx % G;
    uint32_t* gc = &gb.groups[g].count;
    if (ptx::atom_add_relaxed_gpu(gc, 1u) != group_size(n, G, g) - 1u) return false;
    // reset before the fence: the fence orders it before the root arrival
    ptx::st_relaxed_gpu(gc, 0u);
    ptx::fence_acq_rel_gpu();
    n = G;
  }
  if (ptx::atom_add_relaxed_gpu(&gb.slot->count, 1u) != n - 1u) return false;
  ptx::st_relaxed_gpu(&gb.slot->count, 0u);
  ptx::fence_acq_rel_gpu();
  for (uint32_t r = 0; r < kFanoutLines; ++r) ptx::st_relaxed_gpu(fanout_line(gb, r), epoch + 1u);
  return true;
}

// Global level, red flavour: arrivals are fire-and-forget `red.release.gpu.add`;
// participant 0 polls the counter, resets it and bumps the epoch.
__device__ __forceinline__ bool global_arrive_red(const GridBarrier& gb, uint32_t idx,
                                                  uint32_t n, uint32_t epoch,
                                                  uint32_t episode) {
  ptx::red_add_release_gpu(&gb.slot->count, 1u);
  if (idx != 0) return true;
  if (!wait_eq(&gb.slot->count, n, gb, episode)) return false;
  ptx::st_relaxed_gpu(&gb.slot->count, 0u);
  ptx::st_release_gpu(&gb.slot->epoch, epoch + 1u);
  return true;
}

}  // namespace detail

// Per-CTA barrier handle.  All member functions are whole-CTA collectives:
// every thread of the CTA (and, for the cluster variants, of its cluster) must
// call them in the same order.
template <int V>
struct GridSync {
  GridBarrier gb;
  BarrierShared* sh;
  uint32_t epoch;    // meaningful in thread 0
  uint32_t episode;  // meaningful in thread 0
  uint32_t sense;    // flip variants: per-word top bits the next episode waits for (thread 0)

  static constexpr bool kCluster = V == V_CLUSTER || V == V_CLUSTER_ALLPOLL || V == V_DSMEM ||
                                   V == V_CLUSTER_RED || V == V_CLUSTER_FANOUT;
  static constexpr bool kFlip = V == V_CLUSTER || V == V_CLUSTER_ALLPOLL || V == V_DSMEM || V == V_FLIP;
  static constexpr bool kFanout = V == V_FANOUT || V == V_CLUSTER_FANOUT || V == V_HIER;
  // arrive() and wait() are split (a CTA may arrive and leave without waiting)
  static constexpr bool kSplit = V == V_FANOUT || V == V_HIER || V == V_FLIP;
  // arrive() tells thread 0 (arrived_done) whether its arrival completed the
  // episode; the completer has then acquired every other CTA's arrival
  static constexpr bool kCompleter = V == V_FANOUT || V == V_HIER;

  // Index of this CTA among the participants and of its arrival unit.
  __device__ __forceinline__ uint32_t my_index() const { return blockIdx.x - gb.first_cta; }
  // Arrival units at the global level (clusters for the cluster variants).
  __device__ __forceinline__ uint32_t units() const {
    return (V == V_FLIP || V == V_FANOUT) ? gb.nparticipants : gb.nparticipants / ptx::cluster_nctarank();
  }

  // Reads the current generation and refuses to start after a recorded error.
  // For the cluster variants the verdict is taken by the cluster leader and
  // broadcast, so that every CTA of a cluster takes the same path (a hardware
  // cluster barrier must see the same number of arrivals from all of them).
  __device__ bool init(const GridBarrier& g, BarrierShared* s) {
    gb = g;
    sh = s;
    episode = 0;
    if (threadIdx.x == 0) {
      // the generation word each protocol waits on (read before this CTA
      // arrives anywhere, so it cannot have moved past this launch's first episode)
      epoch = kFanout ? ptx::ld_acquire_gpu(detail::fanout_line(gb, 0)) : ptx::ld_acquire_gpu(&gb.slot->epoch);
      sense = kFlip ? detail::flip_expect_init(gb, units()) : 0u;
      sh->arrive = 0;
      sh->release = 0;
      sh->ok = 0;
    }
    if (kCluster) {
      ptx::cluster_sync();  // peers' shared words are initialised
      if (threadIdx.x == 0 && ptx::cluster_ctarank() == 0) {
        const uint32_t ok = (ptx::ld_relaxed_gpu(&gb.slot->status) == 0u) ? 1u : 0u;
        const uint32_t n = ptx::cluster_nctarank();
        const uint32_t sa = ptx::smem_u32(&sh->ok);
        for (uint32_t r = 0; r < n; ++r) ptx::st_cluster_relaxed_u32(ptx::mapa_shared(sa, r), ok);
      }
      ptx::cluster_sync();
    } else {
      if (threadIdx.x == 0) sh->ok = (ptx::ld_relaxed_gpu(&gb.slot->status) == 0u) ? 1u : 0u;
      __syncthreads();
    }
    return sh->ok != 0u;
  }

  // Cluster variants must not leave while a peer may still touch their shared
  // memory; every CTA calls finish() once, on every exit path.
  __device__ void finish() {
    if (kCluster) ptx::cluster_sync();
  }

  __device__ bool sync();

  // Split phase: arrive() then, after work that neither depends on this
  // episode nor changes what other CTAs read through it, wait().  Both are
  // whole-CTA collectives; every arrive() is followed by exactly one wait()
  // before the next arrive() or sync().  Variants without a split form arrive
  // and wait inside wait() (correct, no overlap).
  __device__ __forceinline__ void arrive() { arrived_done = 0u; }
  __device__ __forceinline__ bool wait() { return sync(); }

  uint32_t arrived_done;  // thread 0: this CTA's arrival completed the episode
};

// ---------------------------------------------------------------------------
// V_CLUSTER: level 2 = hardware cluster barrier; level 3 = the cluster leader's
// thread 0 arrives on the split flip words and waits for them; the cluster is
// released by a second hardware cluster barrier.  The leader writes the verdict
// into every peer's shared memory before releasing them.
template <>
__device__ __forceinline__ bool GridSync<V_CLUSTER>::sync() {
  ptx::cluster_sync();
  if (ptx::cluster_ctarank() == 0 && threadIdx.x == 0) {
    const uint32_t n = ptx::cluster_nctarank();
    const uint32_t ncl = gb.nparticipants / n;
    detail::flip_arrive(gb, my_index() / n, ncl);
    const bool ok = detail::flip_wait(gb, ncl, sense, episode);
    const uint32_t sa = ptx::smem_u32(&sh->ok);
    for (uint32_t r = 0; r < n; ++r) ptx::st_cluster_relaxed_u32(ptx::mapa_shared(sa, r), ok ? 1u : 0u);
  }
  ptx::cluster_sync();
  if (threadIdx.x == 0) { sense ^= detail::flip_all(gb, units()); ++episode; }
  return sh->ok != 0u;
}

// V_CLUSTER_RED: the completer-publishes protocol with clusters: hardware
// cluster barrier, `red.release.gpu.add` arrivals on one counter, the leader of
// cluster 0 polls the counter, resets it and bumps the epoch; a second hardware
// cluster barrier releases the clusters.
template <>
__device__ __forceinline__ bool GridSync<V_CLUSTER_RED>::sync() {
  ptx::cluster_sync();
  const uint32_t crank = ptx::cluster_ctarank();
  if (crank == 0 && threadIdx.x == 0) {
    const uint32_t ncl = gb.nparticipants / ptx::cluster_nctarank();
    const uint32_t cid = my_index() / ptx::cluster_nctarank();
    bool ok = detail::global_arrive_red(gb, cid, ncl, epoch, episode);
    if (ok && cid != 0) ok = detail::wait_ne(&gb.slot->epoch, epoch, gb, episode);
    const uint32_t n = ptx::cluster_nctarank();
    const uint32_t sa = ptx::smem_u32(&sh->ok);
    for (uint32_t r = 0; r < n; ++r) ptx::st_cluster_relaxed_u32(ptx::mapa_shared(sa, r), ok ? 1u : 0u);
  }
  ptx::cluster_sync();
  if (threadIdx.x == 0) { ++epoch; ++episode; }
  return sh->ok != 0u;
}

// V_CLUSTER_ALLPOLL: one hardware cluster barrier for arrival; the leader
// arrives on the flip words; every CTA's thread 0 then polls them itself.  The
// verdict is per CTA (not cluster-uniform), so a kernel using this variant must
// keep calling sync() the same number of times on every CTA even after a
// failure (the library's kernels only use it in fixed-count loops).
template <>
__device__ __forceinline__ bool GridSync<V_CLUSTER_ALLPOLL>::sync() {
  ptx::cluster_sync();
  if (threadIdx.x == 0) {
    const uint32_t n = ptx::cluster_nctarank();
    const uint32_t ncl = gb.nparticipants / n;
    if (ptx::cluster_ctarank() == 0) detail::flip_arrive(gb, my_index() / n, ncl);
    sh->ok = detail::flip_wait(gb, ncl, sense, episode) ? 1u : 0u;
    sense ^= detail::flip_all(gb, ncl);
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

// V_DSMEM: no hardware cluster barrier per episode.  Every non-leader CTA's
// thread 0 adds one to the leader's shared-memory arrival counter
// (red.release.cluster); the leader polls its own shared memory, arrives on the
// flip words, waits, and stores (episode + 1, top bit = failure) into every
// peer's release word (st.release.cluster); peers poll their own shared memory.
template <>
__device__ __forceinline__ bool GridSync<V_DSMEM>::sync() {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t n = ptx::cluster_nctarank();
    const uint32_t msg_ok = (episode + 1u) & 0x7fffffffu;
    bool ok = true;
    if (ptx::cluster_ctarank() == 0) {
      uint64_t t0 = 0;
      for (uint32_t it = 0;; ++it) {  // the n-1 peers (bounded shared-memory poll)
        if (ptx::ld_shared_acquire_cluster_u32(&sh->arrive) == n - 1u) break;
        if ((it & 255u) == 255u) {
          if (ptx::ld_relaxed_gpu(&gb.slot->status) != 0u) { ok = false; break; }
          const uint64_t now = ptx::globaltimer_ns();
          if (t0 == 0) t0 = now;
          else if (now - t0 > gb.timeout_ns) {
            detail::record_error(gb, GSRB_DEV_TIMEOUT, episode);
            ok = false;
            break;
          }
        }
      }
      sh->arrive = 0;
      const uint32_t ncl = gb.nparticipants / n;
      if (ok) {
        detail::flip_arrive(gb, my_index() / n, ncl);
        ok = detail::flip_wait(gb, ncl, sense, episode);
      }
      const uint32_t msg = ok ? msg_ok : (msg_ok | 0x80000000u);
      const uint32_t sa = ptx::smem_u32(&sh->release);
      for (uint32_t r = 1; r < n; ++r) ptx::st_cluster_release_u32(ptx::mapa_shared(sa, r), msg);
    } else {
      ptx::red_cluster_release_add_u32(ptx::mapa_shared(ptx::smem_u32(&sh->arrive), 0), 1u);
      uint64_t t0 = 0;
      for (uint32_t it = 0;; ++it) {
        const uint32_t v = ptx::ld_shared_acquire_cluster_u32(&sh->release);
        if ((v & 0x7fffffffu) == msg_ok) { ok = (v & 0x80000000u) == 0u; break; }
        if ((it & 255u) == 255u) {
          const uint64_t now = ptx::globaltimer_ns();
          if (t0 == 0) t0 = now;
          // the leader always answers (its own waits are bounded by the same
          // deadline), so allow it twice the time before giving up here
          else if (now - t0 > 2 * gb.timeout_ns + 1000000ull) {
            detail::record_error(gb, GSRB_DEV_TIMEOUT, episode);
            ok = false;
            break;
          }
        }
      }
    }
    sh->ok = ok ? 1u : 0u;
    sense ^= detail::flip_all(gb, gb.nparticipants / n);
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

// V_FANOUT: __syncthreads, every CTA's thread 0 arrives on the counter and the
// completer publishes the generation to the wake-up lines; CTA b polls line b % R.
template <>
__device__ __forceinline__ bool GridSync<V_FANOUT>::sync() {
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = true;
    if (!detail::fanout_arrive(gb, gb.nparticipants, epoch))
      ok = detail::fanout_wait(gb, my_index(), epoch, episode);
    sh->ok = ok ? 1u : 0u;
    ++epoch;
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

// V_CLUSTER_FANOUT: one hardware cluster barrier for arrival; the cluster
// leader arrives on the counter; every CTA's thread 0 polls its wake-up line.
// Per-CTA verdict (see V_CLUSTER_ALLPOLL): fixed-count loops only.
template <>
__device__ __forceinline__ bool GridSync<V_CLUSTER_FANOUT>::sync() {
  ptx::cluster_sync();
  if (threadIdx.x == 0) {
    bool done = false;
    if (ptx::cluster_ctarank() == 0) done = detail::fanout_arrive(gb, gb.nparticipants / ptx::cluster_nctarank(), epoch);
    sh->ok = (done || detail::fanout_wait(gb, my_index(), epoch, episode)) ? 1u : 0u;
    ++epoch;
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

// V_HIER: __syncthreads; thread 0 arrives on its group counter (groups =
// fanin_groups); group completers arrive on the root; the root completer
// publishes to the wake-up lines (R = nflip, at most 8); CTA b polls line b % R.
template <>
__device__ __forceinline__ bool GridSync<V_HIER>::sync() {
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = true;
    if (!detail::hier_arrive(gb, my_index(), gb.nparticipants, epoch))
      ok = detail::fanout_wait(gb, my_index(), epoch, episode);
    sh->ok = ok ? 1u : 0u;
    ++epoch;
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

template <>
__device__ __forceinline__ void GridSync<V_FANOUT>::arrive() {
  __syncthreads();
  if (threadIdx.x == 0) arrived_done = detail::fanout_arrive(gb, gb.nparticipants, epoch) ? 1u : 0u;
}
template <>
__device__ __forceinline__ bool GridSync<V_FANOUT>::wait() {
  if (threadIdx.x == 0) {
    const bool ok = arrived_done || detail::fanout_wait(gb, my_index(), epoch, episode);
    sh->ok = ok ? 1u : 0u;
    ++epoch;
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}
template <>
__device__ __forceinline__ void GridSync<V_HIER>::arrive() {
  __syncthreads();
  if (threadIdx.x == 0) arrived_done = detail::hier_arrive(gb, my_index(), gb.nparticipants, epoch) ? 1u : 0u;
}
template <>
__device__ __forceinline__ bool GridSync<V_HIER>::wait() {
  if (threadIdx.x == 0) {
    const bool ok = arrived_done || detail::fanout_wait(gb, my_index(), epoch, episode);
    sh->ok = ok ? 1u : 0u;
    ++epoch;
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

// V_FLIP: two levels without clusters: __syncthreads, then every CTA's thread 0
// arrives on the split flip words and polls them.
template <>
__device__ __forceinline__ bool GridSync<V_FLIP>::sync() {
  __syncthreads();
  if (threadIdx.x == 0) {
    detail::flip_arrive(gb, my_index(), gb.nparticipants);
    sh->ok = detail::flip_wait(gb, gb.nparticipants, sense, episode) ? 1u : 0u;
    sense ^= detail::flip_all(gb, gb.nparticipants);
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}
template <>
__device__ __forceinline__ void GridSync<V_FLIP>::arrive() {
  __syncthreads();
  if (threadIdx.x == 0) detail::flip_arrive(gb, my_index(), gb.nparticipants);
}
template <>
__device__ __forceinline__ bool GridSync<V_FLIP>::wait() {
  if (threadIdx.x == 0) {
    sh->ok = detail::flip_wait(gb, gb.nparticipants, sense, episode) ? 1u : 0u;
    sense ^= detail::flip_all(gb, gb.nparticipants);
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

// V_LOCKFREE: flat (ngroups <= 1: every CTA is a member of one flag barrier,
// CTA 0 the master) or two-level (ngroups = G: group g = index % G with its
// first member as local master, as the reference's per-SM local barrier;
// the local masters form the global barrier, master = group 0's master).
template <>
__device__ __forceinline__ bool GridSync<V_LOCKFREE>::sync() {
  uint32_t* gin = gb.flip;
  uint32_t* gout = gb.flip + detail::kLfGlobal;
  const uint32_t n = gb.nparticipants, p = my_index(), G = gb.ngroups;
  const uint32_t ep = episode++;
  bool ok;
  if (G <= 1 || n <= G) {
    ok = detail::lf_episode(gin, gout, n, p, gb, ep, [] { return true; });
  } else {
    const uint32_t g = p % G, j = p / G;
    uint32_t* lin = gb.flip + 2 * detail::kLfGlobal + (size_t)g * 2 * detail::kLfLocal;
    uint32_t* lout = lin + detail::kLfLocal;
    const uint32_t m = detail::group_size(n, G, g);
    ok = detail::lf_episode(lin, lout, m, j, gb, ep, [&] {
      return detail::lf_episode(gin, gout, G, g, gb, ep, [] { return true; });
    });
  }
  return ok;
}

// V_SOFT2: the reference GSRB two-level structure with software groups
// (group g = participant % ngroups, ngroups = min(participants, #SMs) by
// default).  The last arriver of a group arrives at the root; all CTAs poll.
template <>
__device__ __forceinline__ bool GridSync<V_SOFT2>::sync() {
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = true;
    if (!detail::global_arrive_atom(gb, my_index(), gb.nparticipants, epoch))
      ok = detail::wait_ne(&gb.slot->epoch, epoch, gb, episode);
    sh->ok = ok ? 1u : 0u;
    ++epoch;
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

// V_FLAT: the reference GCPUSRB: one counter, every CTA arrives and polls.
template <>
__device__ __forceinline__ bool GridSync<V_FLAT>::sync() {
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = true;
    GridBarrier flat = gb;
    flat.ngroups = 0;
    if (!detail::global_arrive_atom(flat, my_index(), gb.nparticipants, epoch))
      ok = detail::wait_ne(&gb.slot->epoch, epoch, gb, episode);
    sh->ok = ok ? 1u : 0u;
    ++epoch;
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

namespace detail {
// One sub-barrier of the HeteroSync atomic tree barrier
// (Heterosync/cudaLocksBarrierAtomic.cu:6-57): arrive with an increment, then
// try compare-and-swap(count: n -> 0); the barrier is passed once the counter is
// seen at zero.  Bounded.
__device__ __forceinline__ bool tree_sub(uint32_t* cnt, uint32_t n, const GridBarrier& gb,
                                         uint32_t episode) {
  ptx::atom_add_acq_rel_gpu(cnt, 1u);
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    if (ptx::atom_cas_acq_rel_gpu(cnt, n, 0u) == 0u) return true;
    if ((it & 31u) == 31u) {
      if (ptx::ld_relaxed_gpu(&gb.slot->status) != 0u) return false;
      const uint64_t now = ptx::globaltimer_ns();
      if (t0 == 0) t0 = now;
      else if (now - t0 > gb.timeout_ns) {
        record_error(gb, GSRB_DEV_TIMEOUT, episode);
        return false;
      }
    }
    if (gb.spin_ns) __nanosleep(gb.spin_ns);
  }
}
}  // namespace detail

// V_TREE: HeteroSync atomic tree barrier (joinBarrier_helper,
// Heterosync/cudaLocksBarrierAtomic.cu:145-170): when a group holds more than
// one CTA, a local two-counter barrier, then group member 0 does the global
// two-counter barrier, then the local barrier again.
template <>
__device__ __forceinline__ bool GridSync<V_TREE>::sync() {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t idx = my_index();
    const uint32_t G = gb.ngroups ? gb.ngroups : 1u;
    const uint32_t g = idx % G;
    const uint32_t member = idx / G;
    const uint32_t gsz = detail::group_size(gb.nparticipants, G, g);
    bool ok = true;
    if (gsz > 1) {
      ok = detail::tree_sub(&gb.groups[g].count, gsz, gb, episode) &&
           detail::tree_sub(&gb.groups[g].count2, gsz, gb, episode);
      if (ok && member == 0)
        ok = detail::tree_sub(&gb.slot->count, G, gb, episode) &&
             detail::tree_sub(&gb.slot->count2, G, gb, episode);
      if (ok)
        ok = detail::tree_sub(&gb.groups[g].count, gsz, gb, episode) &&
             detail::tree_sub(&gb.groups[g].count2, gsz, gb, episode);
    } else {
      ok = detail::tree_sub(&gb.slot->count, gb.nparticipants < G ? gb.nparticipants : G, gb, episode) &&
           detail::tree_sub(&gb.slot->count2, gb.nparticipants < G ? gb.nparticipants : G, gb, episode);
    }
    sh->ok = ok ? 1u : 0u;
    ++episode;
  }
  __syncthreads();
  return sh->ok != 0u;
}

// V_CCG: the library barrier.  Only valid under a cooperative launch, which the
// host side always uses for this variant (it refuses a grid that is not
// co-resident instead of hanging).
template <>
__device__ __forceinline__ bool GridSync<V_CCG>::sync() {
  cooperative_groups::this_grid().sync();
  return true;
}

}  // namespace gsrb
