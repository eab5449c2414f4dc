// gsrb/cudaLocks.cuh -- drop-in device API of the Heterosync cudaLocks layer.
//
// Same names and parameters as the reference device functions (all whole-CTA
// collectives), implemented on the sm_100a primitives of gsrb/barrier.cuh and
// gsrb/locks.cuh.  Differences a caller can observe:
//   * every wait is bounded (GSRB_LOCKS_TIMEOUT_NS, default 2 s); a wait that
//     runs out records a status code in the buffer's header (read it on the host
//     with gsrb_cudalocks_status()) and the call returns without the lock, so the
//     kernel finishes instead of hanging;
//   * ordering uses gpu-scope acquire/release also in the *Local variants (the
//     reference orders those with __threadfence_block although its "SM" groups
//     are logical, blockIdx % NUM_SM, so their CTAs can sit on different SMs);
//   * the priority semaphore functions run the B200-native protocol on the
//     reference record (gsrb::PrioritySem); the plain spin / EBO semaphores keep
//     the reference protocol, with its record stride fixed to 5 words (the
//     reference indexes them with stride 4, Heterosync/cudaLocksSemaphoreSpin.cu:44,
//     against the stride-5 layout of the create function, :18);
//   * the grid barriers keep no state between calls in registers: thread 0 reads
//     the generation word on entry (one extra L2 read per episode compared with
//     gsrb::GridSync, which is the fast path for new code).
// Include in exactly the translation units that launch the kernels (like the
// reference's #include "cudaLocks*.cu"), and link libgsrb.so for the host API.
#pragma once
#include <cstddef>

#include "gsrb/barrier.cuh"
#include "gsrb/cudaLocks.h"
#include "gsrb/locks.cuh"

#ifndef GSRB_LOCKS_TIMEOUT_NS
#define GSRB_LOCKS_TIMEOUT_NS 2000000000ull
#endif

// ------------------------------------------------------------------ mutexes --
// Heterosync/cudaLocksMutexSpin.cu:13-50 (+ Local :53-96)
inline __device__ void cudaMutexSpinLock(const cudaMutex_t mutex, unsigned int* mutexBufferHeads, const int NUM_SM) {
  gsrb::mutex_spin_lock(mutexBufferHeads + mutex * NUM_SM, mutexBufferHeads, GSRB_LOCKS_TIMEOUT_NS, false);
}
inline __device__ void cudaMutexSpinUnlock(const cudaMutex_t mutex, unsigned int* mutexBufferHeads, const int NUM_SM) {
  gsrb::mutex_spin_unlock(mutexBufferHeads + mutex * NUM_SM);
}
inline __device__ void cudaMutexSpinLockLocal(const cudaMutex_t mutex, const unsigned int smID,
                                              unsigned int* mutexBufferHeads, const int NUM_SM) {
  gsrb::mutex_spin_lock(mutexBufferHeads + mutex * NUM_SM + smID, mutexBufferHeads, GSRB_LOCKS_TIMEOUT_NS, false);
}
inline __device__ void cudaMutexSpinUnlockLocal(const cudaMutex_t mutex, const unsigned int smID,
                                                unsigned int* mutexBufferHeads, const int NUM_SM) {
  gsrb::mutex_spin_unlock(mutexBufferHeads + mutex * NUM_SM + smID);
}
// Heterosync/cudaLocksMutexEBO.cu:13-65 (+ Local)
inline __device__ void cudaMutexEBOLock(const cudaMutex_t mutex, unsigned int* mutexBufferHeads, const int NUM_SM) {
  gsrb::mutex_spin_lock(mutexBufferHeads + mutex * NUM_SM, mutexBufferHeads, GSRB_LOCKS_TIMEOUT_NS, true);
}
inline __device__ void cudaMutexEBOUnlock(const cudaMutex_t mutex, unsigned int* mutexBufferHeads, const int NUM_SM) {
  gsrb::mutex_spin_unlock(mutexBufferHeads + mutex * NUM_SM);
}
inline __device__ void cudaMutexEBOLockLocal(const cudaMutex_t mutex, const unsigned int smID,
                                             unsigned int* mutexBufferHeads, const int NUM_SM) {
  gsrb::mutex_spin_lock(mutexBufferHeads + mutex * NUM_SM + smID, mutexBufferHeads, GSRB_LOCKS_TIMEOUT_NS, true);
}
inline __device__ void cudaMutexEBOUnlockLocal(const cudaMutex_t mutex, const unsigned int smID,
                                               unsigned int* mutexBufferHeads, const int NUM_SM) {
  gsrb::mutex_spin_unlock(mutexBufferHeads + mutex * NUM_SM + smID);
}
// Heterosync/cudaLocksMutexFA.cu:13-69 (+ Local :72-140)
inline __device__ void cudaMutexFALock(const cudaMutex_t mutex, unsigned int* mutexBufferHeads,
                                       unsigned int* mutexBufferTails, const int NUM_SM) {
  gsrb::mutex_fa_lock(mutexBufferHeads + mutex * NUM_SM, mutexBufferTails + mutex * NUM_SM, mutexBufferHeads,
                      GSRB_LOCKS_TIMEOUT_NS);
}
inline __device__ void cudaMutexFAUnlock(const cudaMutex_t mutex, unsigned int* mutexBufferTails, const int NUM_SM) {
  gsrb::mutex_fa_unlock(mutexBufferTails + mutex * NUM_SM);
}
inline __device__ void cudaMutexFALockLocal(const cudaMutex_t mutex, const unsigned int smID,
                                            unsigned int* mutexBufferHeads, unsigned int* mutexBufferTails,
                                            const int NUM_SM) {
  gsrb::mutex_fa_lock(mutexBufferHeads + mutex * NUM_SM + smID, mutexBufferTails + mutex * NUM_SM + smID,
                      mutexBufferHeads, GSRB_LOCKS_TIMEOUT_NS);
}
inline __device__ void cudaMutexFAUnlockLocal(const cudaMutex_t mutex, const unsigned int smID,
                                              unsigned int* mutexBufferTails, const int NUM_SM) {
  gsrb::mutex_fa_unlock(mutexBufferTails + mutex * NUM_SM + smID);
}
// Heterosync/cudaLocksMutexSleep.cu:20-108 (+ Local)
inline __device__ unsigned int cudaMutexSleepLock(const cudaMutex_t mutex, int* mutexBuffers,
                                                  unsigned int* mutexBufferTails, const int maxRingBufferSize,
                                                  const int arrayStride, const int NUM_SM) {
  uint32_t slot = 0;
  gsrb::mutex_sleep_lock(mutexBuffers + (size_t)(mutex * NUM_SM) * arrayStride, mutexBufferTails + mutex * NUM_SM,
                         (uint32_t)maxRingBufferSize, mutexBuffers, GSRB_LOCKS_TIMEOUT_NS, &slot);
  return slot;
}
inline __device__ void cudaMutexSleepUnlock(const cudaMutex_t mutex, int* mutexBuffers, unsigned int myBufferLoc,
                                            const int maxRingBufferSize, const int arrayStride, const int NUM_SM) {
  gsrb::mutex_sleep_unlock(mutexBuffers + (size_t)(mutex * NUM_SM) * arrayStride, myBufferLoc,
                           (uint32_t)maxRingBufferSize);
}
inline __device__ unsigned int cudaMutexSleepLockLocal(const cudaMutex_t mutex, const unsigned int smID,
                                                       int* mutexBuffers, unsigned int* mutexBufferTails,
                                                       const int maxRingBufferSize, const int arrayStride,
                                                       const int NUM_SM) {
  uint32_t slot = 0;
  gsrb::mutex_sleep_lock(mutexBuffers + (size_t)(mutex * NUM_SM + smID) * arrayStride,
                         mutexBufferTails + mutex * NUM_SM + smID, (uint32_t)maxRingBufferSize, mutexBuffers,
                         GSRB_LOCKS_TIMEOUT_NS, &slot);
  return slot;
}
inline __device__ void cudaMutexSleepUnlockLocal(const cudaMutex_t mutex, const unsigned int smID, int* mutexBuffers,
                                                 unsigned int myBufferLoc, const int maxRingBufferSize,
                                                 const int arrayStride, const int NUM_SM) {
  gsrb::mutex_sleep_unlock(mutexBuffers + (size_t)(mutex * NUM_SM + smID) * arrayStride, myBufferLoc,
                           (uint32_t)maxRingBufferSize);
}

// --------------------------------------------------------------- semaphores --
// Record of semaphore `sem` for SM id `id` (5 words per record).
inline __device__ unsigned int* gsrb_sem_rec(const cudaSemaphore_t sem, unsigned int* semaphoreBuffers,
                                             const int NUM_SM, const unsigned int id) {
  return semaphoreBuffers + (size_t)sem * 5 * NUM_SM + (size_t)id * 5;
}
// Heterosync/cudaLocksSemaphoreSpin.cu:31-218 (+ Local :221-409)
inline __device__ void cudaSemaphoreSpinWait(const cudaSemaphore_t sem, const bool isWriter,
                                             const unsigned int maxSemCount, unsigned int* semaphoreBuffers,
                                             const int NUM_SM) {
  gsrb::refsem_wait(gsrb::RefSem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, 0)}, isWriter, maxSemCount, false,
                    false, semaphoreBuffers, GSRB_LOCKS_TIMEOUT_NS);
}
inline __device__ void cudaSemaphoreSpinPost(const cudaSemaphore_t sem, const bool isWriter,
                                             const unsigned int maxSemCount, unsigned int* semaphoreBuffers,
                                             const int NUM_SM) {
  gsrb::refsem_post(gsrb::RefSem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, 0)}, isWriter, maxSemCount, false,
                    semaphoreBuffers, GSRB_LOCKS_TIMEOUT_NS);
}
inline __device__ void cudaSemaphoreSpinWaitLocal(const cudaSemaphore_t sem, const unsigned int smID,
                                                  const bool isWriter, const unsigned int maxSemCount,
                                                  unsigned int* semaphoreBuffers, const int NUM_SM) {
  gsrb::refsem_wait(gsrb::RefSem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, smID)}, isWriter, maxSemCount, false,
                    false, semaphoreBuffers, GSRB_LOCKS_TIMEOUT_NS);
}
inline __device__ void cudaSemaphoreSpinPostLocal(const cudaSemaphore_t sem, const unsigned int smID,
                                                  const bool isWriter, const unsigned int maxSemCount,
                                                  unsigned int* semaphoreBuffers, const int NUM_SM) {
  gsrb::refsem_post(gsrb::RefSem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, smID)}, isWriter, maxSemCount, false,
                    semaphoreBuffers, GSRB_LOCKS_TIMEOUT_NS);
}
// Heterosync/cudaLocksSemaphoreEBO.cu:30-244 (+ Local)
inline __device__ void cudaSemaphoreEBOWait(const cudaSemaphore_t sem, const bool isWriter,
                                            const unsigned int maxSemCount, unsigned int* semaphoreBuffers,
                                            const int NUM_SM) {
  gsrb::refsem_wait(gsrb::RefSem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, 0)}, isWriter, maxSemCount, false, true,
                    semaphoreBuffers, GSRB_LOCKS_TIMEOUT_NS);
}
inline __device__ void cudaSemaphoreEBOPost(const cudaSemaphore_t sem, const bool isWriter,
                                            const unsigned int maxSemCount, unsigned int* semaphoreBuffers,
                                            const int NUM_SM) {
  gsrb::refsem_post(gsrb::RefSem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, 0)}, isWriter, maxSemCount, false,
                    semaphoreBuffers, GSRB_LOCKS_TIMEOUT_NS);
}
inline __device__ void cudaSemaphoreEBOWaitLocal(const cudaSemaphore_t sem, const unsigned int smID,
                                                 const bool isWriter, const unsigned int maxSemCount,
                                                 unsigned int* semaphoreBuffers, const int NUM_SM) {
  gsrb::refsem_wait(gsrb::RefSem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, smID)}, isWriter, maxSemCount, false,
                    true, semaphoreBuffers, GSRB_LOCKS_TIMEOUT_NS);
}
inline __device__ void cudaSemaphoreEBOPostLocal(const cudaSemaphore_t sem, const unsigned int smID,
                                                 const bool isWriter, const unsigned int maxSemCount,
                                                 unsigned int* semaphoreBuffers, const int NUM_SM) {
  gsrb::refsem_post(gsrb::RefSem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, smID)}, isWriter, maxSemCount, false,
                    semaphoreBuffers, GSRB_LOCKS_TIMEOUT_NS);
}
// Priority semaphores (Heterosync/cudaLocksSemaphoreSpin.cu:411-837,
// cudaLocksSemaphoreEBO.cu:456-930): the B200-native protocol on the same record.
inline __device__ void cudaSemaphoreSpinWaitPriority(const cudaSemaphore_t sem, const bool isWriter,
                                                     const unsigned int maxSemCount, unsigned int* semaphoreBuffers,
                                                     const int NUM_SM) {
  (void)maxSemCount;
  gsrb::psem_wait(gsrb::PrioritySem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, 0)}, isWriter, semaphoreBuffers,
                  GSRB_LOCKS_TIMEOUT_NS, 0);
}
inline __device__ void cudaSemaphoreSpinPostPriority(const cudaSemaphore_t sem, const bool isWriter,
                                                     const unsigned int maxSemCount, unsigned int* semaphoreBuffers,
                                                     const int NUM_SM) {
  (void)maxSemCount;
  gsrb::psem_post(gsrb::PrioritySem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, 0)}, isWriter);
}
inline __device__ void cudaSemaphoreSpinWaitLocalPriority(const cudaSemaphore_t sem, const unsigned int smID,
                                                          const bool isWriter, const unsigned int maxSemCount,
                                                          unsigned int* semaphoreBuffers, const int NUM_SM) {
  (void)maxSemCount;
  gsrb::psem_wait(gsrb::PrioritySem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, smID)}, isWriter, semaphoreBuffers,
                  GSRB_LOCKS_TIMEOUT_NS, 0);
}
inline __device__ void cudaSemaphoreSpinPostLocalPriority(const cudaSemaphore_t sem, const unsigned int smID,
                                                          const bool isWriter, const unsigned int maxSemCount,
                                                          unsigned int* semaphoreBuffers, const int NUM_SM) {
  (void)maxSemCount;
  gsrb::psem_post(gsrb::PrioritySem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, smID)}, isWriter);
}
inline __device__ void cudaSemaphoreEBOWaitPriority(const cudaSemaphore_t sem, const bool isWriter,
                                                    const unsigned int maxSemCount, unsigned int* semaphoreBuffers,
                                                    const int NUM_SM) {
  (void)maxSemCount;
  gsrb::psem_wait(gsrb::PrioritySem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, 0)}, isWriter, semaphoreBuffers,
                  GSRB_LOCKS_TIMEOUT_NS, 64);
}
inline __device__ void cudaSemaphoreEBOPostPriority(const cudaSemaphore_t sem, const bool isWriter,
                                                    const unsigned int maxSemCount, unsigned int* semaphoreBuffers,
                                                    const int NUM_SM) {
  (void)maxSemCount;
  gsrb::psem_post(gsrb::PrioritySem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, 0)}, isWriter);
}
inline __device__ void cudaSemaphoreEBOWaitLocalPriority(const cudaSemaphore_t sem, const unsigned int smID,
                                                         const bool isWriter, const unsigned int maxSemCount,
                                                         unsigned int* semaphoreBuffers, const int NUM_SM) {
  (void)maxSemCount;
  gsrb::psem_wait(gsrb::PrioritySem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, smID)}, isWriter, semaphoreBuffers,
                  GSRB_LOCKS_TIMEOUT_NS, 64);
}
inline __device__ void cudaSemaphoreEBOPostLocalPriority(const cudaSemaphore_t sem, const unsigned int smID,
                                                         const bool isWriter, const unsigned int maxSemCount,
                                                         unsigned int* semaphoreBuffers, const int NUM_SM) {
  (void)maxSemCount;
  gsrb::psem_post(gsrb::PrioritySem{gsrb_sem_rec(sem, semaphoreBuffers, NUM_SM, smID)}, isWriter);
}

// ------------------------------------------------------------------ barriers --
// Stateless wrappers over the native barriers: `barrierBuffers` (allocated by
// cudaLocksInit with room for one gsrb::BarrierSlot) holds the global level;
// `perSMBarrierBuffers` (the harness's per-SM area, zero-initialised,
// Heterosync/main.cu:2556) holds the group counters.
inline __device__ gsrb::GridBarrier gsrb_compat_barrier(unsigned int* barrierBuffers,
                                                        unsigned int* perSMBarrierBuffers, unsigned int groups,
                                                        unsigned int participants) {
  gsrb::GridBarrier gb;
  gb.slot = reinterpret_cast<gsrb::BarrierSlot*>(barrierBuffers);
  gb.groups = reinterpret_cast<gsrb::GroupSlot*>(perSMBarrierBuffers);
  gb.nparticipants = participants;
  gb.first_cta = 0;
  gb.ngroups = groups;
  gb.spin_ns = 0;
  gb.timeout_ns = GSRB_LOCKS_TIMEOUT_NS;
  gb.flip = nullptr;
  gb.nflip = 0;
  gb._pad = 0;
  return gb;
}

// Two-level sense-reversing barrier (Heterosync/cudaLocksBarrierAtomicSRB.cu:196-236):
// groups = numBlocksAtBarr (the number of "SM" groups), participants = gridDim.x.
inline __device__ void joinBarrier_helperSRB(unsigned int* barrierBuffers, unsigned int* perSMBarrierBuffers,
                                             const unsigned int numBlocksAtBarr, const int smID,
                                             const int perSM_blockID, const int numTBs_perSM,
                                             const bool isMasterThread, const int MAX_BLOCKS) {
  (void)smID; (void)perSM_blockID; (void)numTBs_perSM; (void)isMasterThread; (void)MAX_BLOCKS;
  __shared__ gsrb::BarrierShared s_bar;
  gsrb::GridSync<gsrb::V_SOFT2> b;
  const gsrb::GridBarrier gb = gsrb_compat_barrier(barrierBuffers, perSMBarrierBuffers, numBlocksAtBarr, gridDim.x);
  if (b.init(gb, &s_bar)) b.sync();
}
// One-level (GCPUSRB) barrier (Heterosync/cudaLocksBarrierAtomicSRB.cu:258-269).
inline __device__ void joinBarrier_helperNaiveSRB(unsigned int* barrierBuffers, const unsigned int numBlocksAtBarr,
                                                  const int smID, const bool isMasterThread, const int MAX_BLOCKS) {
  (void)smID; (void)isMasterThread; (void)MAX_BLOCKS;
  __shared__ gsrb::BarrierShared s_bar;
  gsrb::GridSync<gsrb::V_FLAT> b;
  const gsrb::GridBarrier gb = gsrb_compat_barrier(barrierBuffers, nullptr, 0, numBlocksAtBarr);
  if (b.init(gb, &s_bar)) b.sync();
}
// HeteroSync lock-free tree barrier (Heterosync/cudaLocksBarrierFast.cu:182-330):
// the reference's flag layout -- global in/out flags at barrierBuffers and
// barrierBuffers + arrayStride indexed by blockIdx (the per-SM masters are
// CTAs 0 .. numBlocksAtBarr-1), per-SM in/out flags at perSMBarrierBuffers +
// 2 * MAX_BLOCKS * smID indexed by perSM_blockID -- with scoped ordering and
// bounded waits (gsrb::detail::lf_episode).
inline __device__ void joinLFBarrier_helper(unsigned int* barrierBuffers, unsigned int* perSMBarrierBuffers,
                                            const unsigned int numBlocksAtBarr, const int smID,
                                            const int perSM_blockID, const int numTBs_perSM,
                                            const int arrayStride, const int MAX_BLOCKS) {
  const gsrb::GridBarrier gb = gsrb_compat_barrier(barrierBuffers + 2 * arrayStride, nullptr, 0, gridDim.x);
  unsigned int* gin = barrierBuffers;
  unsigned int* gout = barrierBuffers + arrayStride;
  if (numTBs_perSM > 1) {
    unsigned int* lin = perSMBarrierBuffers + (size_t)MAX_BLOCKS * smID * 2;
    unsigned int* lout = lin + MAX_BLOCKS;
    gsrb::detail::lf_episode(lin, lout, (uint32_t)numTBs_perSM, (uint32_t)perSM_blockID, gb, 0u, [&] {
      return gsrb::detail::lf_episode(gin, gout, numBlocksAtBarr, (uint32_t)smID, gb, 0u, [] { return true; });
    });
  } else {
    gsrb::detail::lf_episode(gin, gout, numBlocksAtBarr, blockIdx.x, gb, 0u, [] { return true; });
  }
}
// HeteroSync atomic tree barrier (Heterosync/cudaLocksBarrierAtomic.cu:145-170).
inline __device__ void joinBarrier_helper(unsigned int* barrierBuffers, unsigned int* perSMBarrierBuffers,
                                          const unsigned int numBlocksAtBarr, const int smID,
                                          const int perSM_blockID, const int numTBs_perSM,
                                          const bool isMasterThread, const int MAX_BLOCKS) {
  (void)smID; (void)perSM_blockID; (void)numTBs_perSM; (void)isMasterThread; (void)MAX_BLOCKS;
  __shared__ gsrb::BarrierShared s_bar;
  gsrb::GridSync<gsrb::V_TREE> b;
  const gsrb::GridBarrier gb = gsrb_compat_barrier(barrierBuffers, perSMBarrierBuffers, numBlocksAtBarr, gridDim.x);
  if (b.init(gb, &s_bar)) b.sync();
}

// Flat lock-free flag barrier (Heterosync/cudaLocksBarrierFast.cu:182-224): CTA
// 0 collects the in flags of CTAs 0 .. numBlocksAtBarr-1 and releases their out
// flags; the global flags sit where joinLFBarrier_helper keeps them.
inline __device__ void cudaBarrier(unsigned int* barrierBuffers, const int arrayStride,
                                   const unsigned int numBlocksAtBarr) {
  const gsrb::GridBarrier gb = gsrb_compat_barrier(barrierBuffers + 2 * arrayStride, nullptr, 0, gridDim.x);
  gsrb::detail::lf_episode(barrierBuffers, barrierBuffers + arrayStride, numBlocksAtBarr, blockIdx.x, gb, 0u,
                           [] { return true; });
}
// Per-SM lock-free flag barrier (Heterosync/cudaLocksBarrierFast.cu:226-293):
// the numTBs_perSM CTAs of group smID meet on the group's in/out flags; with
// isLocalGlobalBarr the group's first CTA joins the flat barrier in between.
inline __device__ void cudaBarrierLocal(unsigned int* barrierBuffers, const unsigned int numBlocksAtBarr,
                                        const int arrayStride, unsigned int* perSMBarrierBuffers,
                                        const unsigned int smID, const unsigned int numTBs_perSM,
                                        const unsigned int perSM_blockID, const bool isLocalGlobalBarr,
                                        const int MAX_BLOCKS) {
  const gsrb::GridBarrier gb = gsrb_compat_barrier(barrierBuffers + 2 * arrayStride, nullptr, 0, gridDim.x);
  unsigned int* lin = perSMBarrierBuffers + (size_t)MAX_BLOCKS * smID * 2;
  gsrb::detail::lf_episode(lin, lin + MAX_BLOCKS, numTBs_perSM, perSM_blockID, gb, 0u, [&] {
    if (!isLocalGlobalBarr) return true;
    return gsrb::detail::lf_episode(barrierBuffers, barrierBuffers + arrayStride, numBlocksAtBarr, smID, gb, 0u,
                                    [] { return true; });
  });
}
// Heterosync/cudaLocksBarrierFast.cu:295-313.
inline __device__ void cudaBarrierLocalGlobal(unsigned int* barrierBuffers, const unsigned int numBlocksAtBarr,
                                              const int arrayStride, unsigned int* perSMBarrierBuffers,
                                              const unsigned int smID, const unsigned int numTBs_perSM,
                                              const unsigned int perSM_blockID, const int MAX_BLOCKS) {
  cudaBarrierLocal(barrierBuffers, numBlocksAtBarr, arrayStride, perSMBarrierBuffers, smID, numTBs_perSM,
                   perSM_blockID, true, MAX_BLOCKS);
}

// Every thread of every CTA arrives (Heterosync/cudaLocksBarrierAtomicSRB.cu:242-256,
// numThreadsAtBarr = gridDim.x * blockDim.x): each thread adds one to the global
// counter; the last arrival resets it and bumps the generation word, which
// every thread polls (bounded).
inline __device__ void joinBarrier_helperNaiveAllSRB(unsigned int* barrierBuffers, unsigned int* perSMBarrierBuffers,
                                                     const unsigned int numThreadsAtBarr, const int smID,
                                                     const int MAX_BLOCKS) {
  (void)perSMBarrierBuffers; (void)smID; (void)MAX_BLOCKS;
  const gsrb::GridBarrier gb = gsrb_compat_barrier(barrierBuffers, nullptr, 0, gridDim.x);
  __syncthreads();
  const uint32_t gen = gsrb::ptx::ld_relaxed_gpu(&gb.slot->epoch);
  gsrb::ptx::fence_acq_rel_gpu();
  if (gsrb::ptx::atom_add_relaxed_gpu(&gb.slot->count, 1u) == numThreadsAtBarr - 1u) {
    gsrb::ptx::fence_acq_rel_gpu();
    gsrb::ptx::st_relaxed_gpu(&gb.slot->count, 0u);
    gsrb::ptx::st_release_gpu(&gb.slot->epoch, gen + 1u);
  } else {
    gsrb::detail::wait_ne(&gb.slot->epoch, gen, gb, 0u);
  }
  __syncthreads();
}

// ------------------------------------------------------------ local barriers --
// Status of the barriers that get no lock buffer (the per-SM local barriers
// below): one slot per translation unit, read and cleared on the host with
// gsrb_cudalocks_local_status().
static __device__ gsrb::BarrierSlot gsrb_local_status_slot;

// Per-group counter barrier of the local-exchange steps
// (Heterosync/cudaLocksBarrierAtomic.cu:82-140, cudaLocksBarrierAtomicSRB.cu:133-190):
// the numTBs_thisSM CTAs of group smID meet on a counter and a generation word
// of their own.  Group smID's record is the gsrb::GroupSlot at index
// MAX_BLOCKS + smID of the per-SM area (count = arrivals, count2 = generation):
// past the group slots of the two-level grid barriers (fewer than NUM_SM <=
// MAX_BLOCKS of them), and inside the harness's NUM_SM * MAX_BLOCKS * 2 words
// whenever NUM_SM >= 64 and MAX_BLOCKS >= 64.
inline __device__ void gsrb_compat_local_barrier(unsigned int* perSMBarrierBuffers, const unsigned int smID,
                                                 const unsigned int numTBs_thisSM, const int MAX_BLOCKS) {
  gsrb::GroupSlot* rec = reinterpret_cast<gsrb::GroupSlot*>(perSMBarrierBuffers) + (size_t)MAX_BLOCKS + smID;
  __syncthreads();
  if (threadIdx.x == 0) {
    const gsrb::GridBarrier gb =
        gsrb_compat_barrier(reinterpret_cast<unsigned int*>(&gsrb_local_status_slot), nullptr, 0, numTBs_thisSM);
    const uint32_t gen = gsrb::ptx::ld_relaxed_gpu(&rec->count2);
    gsrb::ptx::fence_acq_rel_gpu();
    if (gsrb::ptx::atom_add_relaxed_gpu(&rec->count, 1u) == numTBs_thisSM - 1u) {
      gsrb::ptx::fence_acq_rel_gpu();
      gsrb::ptx::st_relaxed_gpu(&rec->count, 0u);
      gsrb::ptx::st_release_gpu(&rec->count2, gen + 1u);
    } else {
      gsrb::detail::wait_ne(&rec->count2, gen, gb, smID);
    }
  }
  __syncthreads();
}
// Heterosync/cudaLocksBarrierAtomic.cu:125-140.
inline __device__ void cudaBarrierAtomicLocal(unsigned int* perSMBarrierBuffers, const unsigned int smID,
                                              const unsigned int numTBs_thisSM, const bool isMasterThread,
                                              const int MAX_BLOCKS) {
  (void)isMasterThread;
  gsrb_compat_local_barrier(perSMBarrierBuffers, smID, numTBs_thisSM, MAX_BLOCKS);
}
// Heterosync/cudaLocksBarrierAtomicSRB.cu:179-190.
inline __device__ void cudaBarrierAtomicLocalSRB(unsigned int* perSMBarrierBuffers, const unsigned int smID,
                                                 const unsigned int numTBs_thisSM, const bool isMasterThread,
                                                 const int MAX_BLOCKS) {
  (void)isMasterThread;
  gsrb_compat_local_barrier(perSMBarrierBuffers, smID, numTBs_thisSM, MAX_BLOCKS);
}
// Synchronous: the first status code a local barrier of this translation unit
// recorded (0 = none; ~0u if the slot could not be read), then cleared.
static inline unsigned int gsrb_cudalocks_local_status() {
  unsigned int st = 0;
  const unsigned int zero = 0;
  const size_t off = offsetof(gsrb::BarrierSlot, status);
  if (cudaMemcpyFromSymbol(&st, gsrb_local_status_slot, sizeof st, off) != cudaSuccess) return ~0u;
  if (st != 0 && cudaMemcpyToSymbol(gsrb_local_status_slot, &zero, sizeof zero, off) != cudaSuccess) return ~0u;
  return st;
}
