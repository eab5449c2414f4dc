// allSyncPrims-1kernel: the Heterosync microbenchmark program (Heterosync/main.cu)
// on the drop-in cudaLocks API (gsrb/cudaLocks.h, gsrb/cudaLocks.cuh).
//
// Command line as the reference (main.cu:2470-2540):
//   allSyncPrims-1kernel <syncPrim> <numLdSt> <numTBs> <numCSIters> [-r repeats] [-o storage.bin]
// Each syncPrim runs the reference's access pattern: CTAs of 32 threads shift
// their columns of NUM_LDST+1 cache lines down by one line (main.cu:68-80)
// inside a critical section, or between grid barriers with the CTA -> data
// mapping rotated after every barrier; the program times NUM_REPEATS launches
// (10, or -r), replays the same shifts on the host (main.cu:2987-3146) and prints
// PASSED! or the mismatches, with the reference's output lines and exit codes.
// -o writes the final storage array (float32) for external checking.
//
// Differences from the reference program:
//   * the lock data is passed to the kernels by value (the reference reads it
//     from pinned host memory on every use);
//   * every barrier kernel is launched cooperatively, so a grid that cannot be
//     co-resident fails at launch instead of hanging; mutex and semaphore grids
//     are checked against the occupancy limit first;
//   * the local-exchange kernels and the lock-free tree barrier need numTBs to be
//     a multiple of min(numTBs, NUM_SM) (otherwise the reference waits forever
//     for CTAs that do not exist); the program refuses other sizes;
//   * every wait is bounded: a barrier, mutex or semaphore wait that runs out is
//     reported and makes the run fail;
//   * the PRspinSemEBO1/2/10/120 names select syncPrims 32-35 as the reference's
//     usage text lists them (the reference parser maps them nowhere, and reaches
//     32-35 only through duplicate spinSemEBO* entries that 12-15 shadow).
#include <cooperative_groups.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "gsrb/cudaLocks.cuh"

namespace cg = cooperative_groups;

#define CK(x)                                                                        \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess) {                                                         \
      fprintf(stderr, "ERROR: %s failed: %s\n", #x, cudaGetErrorString(e_));         \
      exit(-1);                                                                      \
    }                                                                                \
  } while (0)

namespace {

constexpr int kThreads = 32;   // NUM_THREADS_PER_BLOCK (main.cu:8)
constexpr int kWords = 16;     // NUM_WORDS_PER_CACHELINE (main.cu:11)
constexpr int kHalfWarp = 16;  // NUM_THREADS_PER_HALFWARP (main.cu:12)

struct Args {
  float* storage;
  cudaLockData_t d;
  unsigned int* perSM;
  unsigned int numAtBarr;  // arrivals at the global barrier (CTAs; threads for the all-threads barrier)
  int groups;              // "SM" groups of the barrier: smID = blockIdx % groups
  int numTBs_perSM;
  int exch;                // CTA-index stride of the local exchange
  int iters;
  int nldst;
  int NUM_SM;
  int MAX_BLOCKS;
};

// First line of the column of CTA `block`'s thread (main.cu:125).
__device__ __forceinline__ int column_of(int block, int nldst) {
  return ((block * kThreads + (int)threadIdx.x) / kWords) * (nldst + 1);
}

// The critical section (main.cu:68-80): line n+1 of the column takes line n,
// from the bottom up, so the column moves down by one line.
__device__ __forceinline__ void shift_column(float* s, int col, int nldst) {
  const int w = threadIdx.x % kWords;
  for (int n = nldst - 1; n >= 0; --n) s[(col + n + 1) * kWords + w] = s[(col + n) * kWords + w];
}

// ------------------------------------------------------------------ barriers --
enum BarKind { B_TREE, B_LF, B_SRB, B_NAIVE, B_NAIVEALL, B_CCG };

template <int K>
__device__ __forceinline__ void global_barrier(const Args& a, int smID, int perSM_blockID) {
  const bool master = threadIdx.x == 0;
  if constexpr (K == B_TREE)
    joinBarrier_helper(a.d.barrierBuffers, a.perSM, a.numAtBarr, smID, perSM_blockID, a.numTBs_perSM, master,
                       a.MAX_BLOCKS);
  else if constexpr (K == B_SRB)
    joinBarrier_helperSRB(a.d.barrierBuffers, a.perSM, a.numAtBarr, smID, perSM_blockID, a.numTBs_perSM, master,
                          a.MAX_BLOCKS);
  else if constexpr (K == B_LF)
    joinLFBarrier_helper(a.d.barrierBuffers, a.perSM, a.numAtBarr, smID, perSM_blockID, a.numTBs_perSM,
                         a.d.arrayStride, a.MAX_BLOCKS);
  else if constexpr (K == B_NAIVE)
    joinBarrier_helperNaiveSRB(a.d.barrierBuffers, a.numAtBarr, smID, master, a.MAX_BLOCKS);
  else if constexpr (K == B_NAIVEALL)
    joinBarrier_helperNaiveAllSRB(a.d.barrierBuffers, a.perSM, a.numAtBarr, smID, a.MAX_BLOCKS);
  else
    cg::this_grid().sync();
}

// The barrier among the CTAs of one group before the local exchange
// (main.cu:366-372, 432-434, 635-640; the naive and library kernels use their
// global barrier there, main.cu:496-498, 552-554, 330).
template <int K>
__device__ __forceinline__ void local_barrier(const Args& a, int smID, int perSM_blockID) {
  const bool master = threadIdx.x == 0;
  if constexpr (K == B_TREE)
    cudaBarrierAtomicLocal(a.perSM, smID, a.numTBs_perSM, master, a.MAX_BLOCKS);
  else if constexpr (K == B_SRB)
    cudaBarrierAtomicLocalSRB(a.perSM, smID, a.numTBs_perSM, master, a.MAX_BLOCKS);
  else if constexpr (K == B_LF)
    cudaBarrierLocal(a.d.barrierBuffers, a.numAtBarr, a.d.arrayStride, a.perSM, smID, a.numTBs_perSM,
                     perSM_blockID, false, a.MAX_BLOCKS);
  else
    global_barrier<K>(a, smID, perSM_blockID);
}

// main.cu:111-667: shift the current CTA's columns, (local barrier, exchange
// within the group, shift again,) grid barrier, move on to the next CTA's data.
template <int K, bool LX>
__global__ void __launch_bounds__(kThreads) barrier_kernel(Args a) {
  const int smID = blockIdx.x % a.groups, perSM_blockID = blockIdx.x / a.groups;
  int cur = blockIdx.x;
  for (int i = 0; i < a.iters; ++i) {
    shift_column(a.storage, column_of(cur, a.nldst), a.nldst);
    if (LX && a.numTBs_perSM > 1) {
      local_barrier<K>(a, smID, perSM_blockID);
      cur = (cur + a.exch) % gridDim.x;
      shift_column(a.storage, column_of(cur, a.nldst), a.nldst);
    }
    global_barrier<K>(a, smID, perSM_blockID);
    cur = (cur + 1) % gridDim.x;
  }
}

// ------------------------------------------------------------------- mutexes --
enum MutexKind { M_SPIN, M_EBO, M_SLEEP, M_FA };

// main.cu:669-883: every CTA shifts the same columns (U: the columns of its
// group smID) under the mutex (U: the group's mutex).
template <int K, bool U>
__global__ void __launch_bounds__(kThreads) mutex_kernel(Args a, cudaMutex_t m) {
  const unsigned int smID = blockIdx.x % a.NUM_SM;
  const int col = column_of(U ? (int)smID : 0, a.nldst);
  const cudaLockData_t& d = a.d;
  for (int i = 0; i < a.iters; ++i) {
    unsigned int ring = 0;
    if constexpr (K == M_SPIN) {
      if (U) cudaMutexSpinLockLocal(m, smID, d.mutexBufferHeads, a.NUM_SM);
      else cudaMutexSpinLock(m, d.mutexBufferHeads, a.NUM_SM);
    } else if constexpr (K == M_EBO) {
      if (U) cudaMutexEBOLockLocal(m, smID, d.mutexBufferHeads, a.NUM_SM);
      else cudaMutexEBOLock(m, d.mutexBufferHeads, a.NUM_SM);
    } else if constexpr (K == M_SLEEP) {
      ring = U ? cudaMutexSleepLockLocal(m, smID, d.mutexBuffers, d.mutexBufferTails, d.maxBufferSize,
                                         d.arrayStride, a.NUM_SM)
               : cudaMutexSleepLock(m, d.mutexBuffers, d.mutexBufferTails, d.maxBufferSize, d.arrayStride, a.NUM_SM);
    } else {
      if (U) cudaMutexFALockLocal(m, smID, d.mutexBufferHeads, d.mutexBufferTails, a.NUM_SM);
      else cudaMutexFALock(m, d.mutexBufferHeads, d.mutexBufferTails, a.NUM_SM);
    }
    shift_column(a.storage, col, a.nldst);
    if constexpr (K == M_SPIN) {
      if (U) cudaMutexSpinUnlockLocal(m, smID, d.mutexBufferHeads, a.NUM_SM);
      else cudaMutexSpinUnlock(m, d.mutexBufferHeads, a.NUM_SM);
    } else if constexpr (K == M_EBO) {
      if (U) cudaMutexEBOUnlockLocal(m, smID, d.mutexBufferHeads, a.NUM_SM);
      else cudaMutexEBOUnlock(m, d.mutexBufferHeads, a.NUM_SM);
    } else if constexpr (K == M_SLEEP) {
      if (U) cudaMutexSleepUnlockLocal(m, smID, d.mutexBuffers, ring, d.maxBufferSize, d.arrayStride, a.NUM_SM);
      else cudaMutexSleepUnlock(m, d.mutexBuffers, ring, d.maxBufferSize, d.arrayStride, a.NUM_SM);
    } else {
      if (U) cudaMutexFAUnlockLocal(m, smID, d.mutexBufferTails, a.NUM_SM);
      else cudaMutexFAUnlock(m, d.mutexBufferTails, a.NUM_SM);
    }
  }
}

// ---------------------------------------------------------------- semaphores --
enum SemKind { S_SPIN, S_EBO };

// main.cu:885-1493: one writer CTA per group (perSM_blockID == smID % numTBs_perSM)
// shifts the columns of all of the group's CTAs; the others read their own
// columns.  Without U every group works on the same columns under one global
// semaphore; with U each group has its own columns and semaphore record.
template <int K, bool P, bool U>
__global__ void __launch_bounds__(kThreads) semaphore_kernel(Args a, cudaSemaphore_t sem) {
  const cudaLockData_t& d = a.d;
  const unsigned int maxSemCount = d.semaphoreBuffers[(size_t)sem * 5 * a.NUM_SM + 3];
  const unsigned int numSM = gridDim.x < (unsigned)a.NUM_SM ? gridDim.x : (unsigned)a.NUM_SM;
  const unsigned int smID = U ? blockIdx.x % numSM : blockIdx.x % a.NUM_SM;
  const int numTBs_perSM = (int)((gridDim.x + numSM - 1) / numSM);
  const int perSM_blockID = (int)(blockIdx.x / numSM);
  const bool isWriter = perSM_blockID == (int)(smID % numTBs_perSM);
  const int own = U ? (int)blockIdx.x : perSM_blockID;
  __shared__ volatile float dummy[kThreads];
  dummy[threadIdx.x] = 0.0f;
  for (int i = 0; i < a.iters; ++i) {
    if constexpr (K == S_SPIN && P) {
      if (U) cudaSemaphoreSpinWaitLocalPriority(sem, smID, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
      else cudaSemaphoreSpinWaitPriority(sem, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
    } else if constexpr (K == S_SPIN) {
      if (U) cudaSemaphoreSpinWaitLocal(sem, smID, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
      else cudaSemaphoreSpinWait(sem, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
    } else if constexpr (P) {
      if (U) cudaSemaphoreEBOWaitLocalPriority(sem, smID, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
      else cudaSemaphoreEBOWaitPriority(sem, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
    } else {
      if (U) cudaSemaphoreEBOWaitLocal(sem, smID, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
      else cudaSemaphoreEBOWait(sem, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
    }
    if (isWriter) {
      int blk = own;
      for (int j = 0; j < numTBs_perSM; ++j) {
        shift_column(a.storage, column_of(U ? blk : j, a.nldst), a.nldst);
        blk = (blk + (int)numSM) % (int)gridDim.x;
      }
    } else {
      const int col = column_of(own, a.nldst), w = threadIdx.x % kWords;
      for (int n = a.nldst - 1; n >= 0; --n) {
        dummy[threadIdx.x] += a.storage[(col + n) * kWords + w];
        __syncthreads();
      }
    }
    if constexpr (K == S_SPIN && P) {
      if (U) cudaSemaphoreSpinPostLocalPriority(sem, smID, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
      else cudaSemaphoreSpinPostPriority(sem, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
    } else if constexpr (K == S_SPIN) {
      if (U) cudaSemaphoreSpinPostLocal(sem, smID, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
      else cudaSemaphoreSpinPost(sem, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
    } else if constexpr (P) {
      if (U) cudaSemaphoreEBOPostLocalPriority(sem, smID, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
      else cudaSemaphoreEBOPostPriority(sem, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
    } else {
      if (U) cudaSemaphoreEBOPostLocal(sem, smID, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
      else cudaSemaphoreEBOPost(sem, isWriter, maxSemCount, d.semaphoreBuffers, a.NUM_SM);
    }
  }
}

// ------------------------------------------------------------- the programs --
struct Prim {
  const char* name;      // command-line name (main.cu:2479-2527)
  int id;                // syncPrim number
  const char* banner;    // line printed before the runs (main.cu:2620-2800)
  int banner_arg;        // number printed after the banner, or 0: the
                         // semaphore size, except that the reference prints 2
                         // for the size-120 spin semaphores (main.cu:2670, 2702,
                         // 2734), kept so that output parsers see the same lines
};

const Prim kPrims[] = {
    {"atomicTreeBarrUniq", 0, "atomic_tree_barrier", 0},
    {"atomicTreeBarrUniqLocalExch", 1, "atomic_tree_barrier_localExch", 0},
    {"lfTreeBarrUniq", 2, "fbs_tree_barrier", 0},
    {"lfTreeBarrUniqLocalExch", 3, "fbs_tree_barrier_localExch", 0},
    {"spinMutex", 4, "spin_lock_mutex", 0},
    {"spinMutexEBO", 5, "ebo_mutex", 0},
    {"sleepMutex", 6, "sleeping_mutex", 0},
    {"faMutex", 7, "fetchadd_mutex", 0},
    {"spinSem1", 8, "spin_lock_sem", 1},
    {"spinSem2", 9, "spin_lock_sem", 2},
    {"spinSem10", 10, "spin_lock_sem", 10},
    {"spinSem120", 11, "spin_lock_sem", 2},
    {"spinSemEBO1", 12, "ebo_sem", 1},
    {"spinSemEBO2", 13, "ebo_sem", 2},
    {"spinSemEBO10", 14, "ebo_sem", 10},
    {"spinSemEBO120", 15, "ebo_sem", 120},
    {"PRspinSem1", 16, "spin_lock_sem", 1},
    {"PRspinSem2", 17, "spin_lock_sem", 2},
    {"PRspinSem10", 18, "spin_lock_sem", 10},
    {"PRspinSem120", 19, "spin_lock_sem", 2},
    {"spinMutexUniq", 20, "spin_lock_mutex_uniq", 0},
    {"spinMutexEBOUniq", 21, "ebo_mutex_uniq", 0},
    {"sleepMutexUniq", 22, "sleeping_mutex_uniq", 0},
    {"faMutexUniq", 23, "fetchadd_mutex_uniq", 0},
    {"spinSemUniq1", 24, "spin_lock_sem_uniq", 1},
    {"spinSemUniq2", 25, "spin_lock_sem_uniq", 2},
    {"spinSemUniq10", 26, "spin_lock_sem_uniq", 10},
    {"spinSemUniq120", 27, "spin_lock_sem_uniq", 2},
    {"spinSemEBOUniq1", 28, "ebo_sem_uniq", 1},
    {"spinSemEBOUniq2", 29, "ebo_sem_uniq", 2},
    {"spinSemEBOUniq10", 30, "ebo_sem_uniq", 10},
    {"spinSemEBOUniq120", 31, "ebo_sem_uniq", 120},
    {"PRspinSemEBO1", 32, "ebo_sem", 1},
    {"PRspinSemEBO2", 33, "ebo_sem", 2},
    {"PRspinSemEBO10", 34, "ebo_sem", 10},
    {"PRspinSemEBO120", 35, "ebo_sem", 120},
    {"atomicTreeBarrUniqSRB", 37, "atomic_tree_barrier_SRB", 0},
    {"atomicTreeBarrUniqLocalExchSRB", 38, "atomic_tree_barrier_localExch_SRB", 0},
    {"atomicTreeBarrUniqNaiveSRB", 39, "atomic_tree_barrier_NaiveSRB", 0},
    {"atomicTreeBarrUniqLocalExchNaiveSRB", 40, "atomic_tree_barrier_localExch_NaiveSRB", 0},
    {"atomicTreeBarrUniqNaiveAllSRB", 41, "atomic_tree_barrier_NaiveAllSRB", 0},
    {"atomicTreeBarrUniqLocalExchNaiveAllSRB", 42, "atomic_tree_barrier_localExch_NaiveAllSRB", 0},
    {"atomicTreeBarrUniqHybridSRB", 43, "atomic_tree_barrier_hybridSRB", 0},
    {"atomicTreeBarrUniqLocalExchHybridSRB", 44, "atomic_tree_barrier_localExch_hybridSRB", 0},
    {"atomicTreeBarrUniqCCG", 45, "atomic_tree_barrier_ccg", 0},
    {"atomicTreeBarrUniqLocalExchCCG", 46, "atomic_tree_barrier_localExch_ccg", 0},
};

bool is_barrier(int p) { return p < 4 || p >= 37; }
bool is_local_exch(int p) { return p == 1 || p == 3 || p == 38 || p == 40 || p == 42 || p == 44 || p == 46; }

// Storage words (main.cu:2561-2583).
int storage_locs(int p, int nldst, int numTBs, int NUM_SM) {
  const int perSM = (numTBs + NUM_SM - 1) / NUM_SM;
  int mult = 0;
  if (is_barrier(p) || (p >= 24 && p <= 35)) mult = numTBs;
  else if (p >= 4 && p <= 7) mult = 1;
  else if (p >= 8 && p <= 19) mult = perSM;
  else mult = numTBs < NUM_SM ? numTBs : NUM_SM;
  return mult * kThreads * (nldst + 1);
}

// The harness's host replay (main.cu:41-59, 2987-3146): the same shifts, one
// word at a time, visiting each column from the bottom up.
struct Golden {
  std::vector<float> s;
  int nldst;
  void at(int loc) {
    if (loc % (kHalfWarp * (nldst + 1)) >= kWords) s[loc] = s[loc - kWords];
  }
  void sweep(int count, int offset, int mod) {
    for (int i = count - 1; i >= 0; --i) at((i + offset) % mod);
  }
};

std::vector<float> golden(int p, int nldst, int numTBs, int iters, int repeats, int NUM_SM, int nlocs) {
  Golden g{std::vector<float>(nlocs), nldst};
  for (int i = 0; i < nlocs; ++i) g.s[i] = (float)i;
  const int uniq = kThreads * (nldst + 1);
  const int perSM = (numTBs + NUM_SM - 1) / NUM_SM;
  const int nsm = numTBs < NUM_SM ? numTBs : NUM_SM;
  for (int r = 0; r < repeats; ++r) {
    for (int j = 0; j < iters; ++j) {
      if (is_barrier(p)) {
        const int acc = numTBs * uniq;
        g.sweep(acc, j * uniq, acc);
        if (is_local_exch(p) && perSM > 1) g.sweep(acc, (perSM * uniq + j * uniq) % acc, acc);
      } else if (p >= 4 && p <= 7) {
        for (int b = 0; b < numTBs; ++b) g.sweep(uniq, 0, uniq);
      } else if ((p >= 8 && p <= 19) || (p >= 32 && p <= 35)) {
        for (int tb = 0; tb < numTBs; ++tb) {
          const int sm = tb % nsm, per = tb / nsm;
          if (per != sm % perSM) continue;
          for (int k = 0; k < perSM; ++k) g.sweep(uniq, k * uniq, nlocs);
        }
      } else if (p >= 20 && p <= 23) {
        const int acc = numTBs * uniq;
        for (int i = acc - 1; i >= 0; --i) g.at(i % (NUM_SM * uniq));
      } else {
        g.sweep(numTBs * uniq, 0, numTBs * uniq);
      }
    }
  }
  return g.s;
}

int usage(const char* prog) {
  fprintf(stderr, "usage: %s <syncPrim> <numLdSt> <numTBs> <numCSIters> [-r repeats] [-o storage.bin]\n", prog);
  fprintf(stderr, "\t<syncPrim>:");
  for (const Prim& p : kPrims) fprintf(stderr, " %s", p.name);
  fprintf(stderr, "\n");
  return -1;
}

template <class F>
void launch_timed(F&& launch, int repeats, float* total) {
  cudaEvent_t t0, t1;
  CK(cudaEventCreate(&t0));
  CK(cudaEventCreate(&t1));
  for (int r = 0; r < repeats; ++r) {
    CK(cudaEventRecord(t0));
    CK(launch());
    CK(cudaEventRecord(t1));
    CK(cudaEventSynchronize(t1));
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, t0, t1));
    *total += ms;
  }
  CK(cudaEventDestroy(t0));
  CK(cudaEventDestroy(t1));
}

template <int K, bool LX>
cudaError_t launch_barrier(Args a, int blocks) {
  void* params[] = {&a};
  return cudaLaunchCooperativeKernel((const void*)barrier_kernel<K, LX>, blocks, kThreads, params, 0, 0);
}

cudaError_t fits(const void* fn, int blocks, int NUM_SM) {
  int per = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, kThreads, 0);
  if (e != cudaSuccess) return e;
  return blocks <= per * NUM_SM ? cudaSuccess : cudaErrorCooperativeLaunchTooLarge;
}

template <int K, bool U>
cudaError_t launch_mutex(Args a, int blocks, cudaMutex_t m) {
  cudaError_t e = fits((const void*)mutex_kernel<K, U>, blocks, a.NUM_SM);
  if (e != cudaSuccess) return e;
  mutex_kernel<K, U><<<blocks, kThreads>>>(a, m);
  return cudaGetLastError();
}

template <int K, bool P, bool U>
cudaError_t launch_semaphore(Args a, int blocks, cudaSemaphore_t s) {
  cudaError_t e = fits((const void*)semaphore_kernel<K, P, U>, blocks, a.NUM_SM);
  if (e != cudaSuccess) return e;
  semaphore_kernel<K, P, U><<<blocks, kThreads>>>(a, s);
  return cudaGetLastError();
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 5) return usage(argv[0]);
  int repeats = 10;  // NUM_REPEATS (main.cu:24)
  const char* out_path = nullptr;
  for (int i = 5; i < argc; ++i) {
    if (!strcmp(argv[i], "-r") && i + 1 < argc) repeats = atoi(argv[++i]);
    else if (!strcmp(argv[i], "-o") && i + 1 < argc) out_path = argv[++i];
    else return usage(argv[0]);
  }
  const Prim* prim = nullptr;
  for (const Prim& p : kPrims)
    if (!strcmp(p.name, argv[1])) prim = &p;
  if (!prim) {
    fprintf(stderr, "ERROR: Unknown synchronization primitive: %s\n", argv[1]);
    return -1;
  }
  const int nldst = atoi(argv[2]), numTBs = atoi(argv[3]), iters = atoi(argv[4]);
  if (nldst <= 0 || numTBs <= 0 || iters < 0 || repeats <= 0) return usage(argv[0]);

  int dev = 0, deviceCount = 0;
  CK(cudaGetDeviceCount(&deviceCount));
  if (deviceCount == 0) {
    fprintf(stderr, "There is no device supporting CUDA\n");
    return -1;
  }
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  fprintf(stdout, "GPU Compute Capability: %d.%d\n", prop.major, prop.minor);
  const int NUM_SM = prop.multiProcessorCount;
  const int maxTBPerSM = prop.maxThreadsPerBlock / kThreads;
  const int MAX_BLOCKS = maxTBPerSM * NUM_SM;
  fprintf(stdout, "# SM: %d, Max Thrs/TB: %d, Max TB/SM: %d, Max # TB: %d\n", NUM_SM, prop.maxThreadsPerBlock,
          maxTBPerSM, MAX_BLOCKS);
  if (numTBs > MAX_BLOCKS) {
    fprintf(stderr, "ERROR: numTBs (%d) > MAX_BLOCKS (%d)\n", numTBs, MAX_BLOCKS);
    return -1;
  }
  const int p = prim->id;
  const int groups = numTBs < NUM_SM ? numTBs : NUM_SM;
  const int numTBs_perSM = (numTBs + groups - 1) / groups;
  if ((is_local_exch(p) || p == 2) && numTBs % groups != 0) {
    fprintf(stderr, "ERROR: %s needs numTBs to be a multiple of %d (every group the same size)\n", prim->name,
            groups);
    return -1;
  }

  CK(cudaLocksInit(MAX_BLOCKS, 8 * NUM_SM, 24 * NUM_SM, false, NUM_SM));
  const size_t perSM_words = (size_t)NUM_SM * MAX_BLOCKS * 2;
  unsigned int* perSM = nullptr;
  CK(cudaMalloc(&perSM, perSM_words * sizeof(unsigned int)));
  CK(cudaMemset(perSM, 0, perSM_words * sizeof(unsigned int)));

  const int nlocs = storage_locs(p, nldst, numTBs, NUM_SM);
  fprintf(stdout, "# TBs: %d, # Ld/St: %d, # Locs Mult: %d, # Uniq Locs/TB: %d, # Storage Locs: %d\n", numTBs, nldst,
          nlocs / (kThreads * (nldst + 1)), kThreads * (nldst + 1), nlocs);
  std::vector<float> host(nlocs);
  for (int i = 0; i < nlocs; ++i) host[i] = (float)i;
  float* storage = nullptr;
  CK(cudaMalloc(&storage, sizeof(float) * nlocs));
  CK(cudaMemcpy(storage, host.data(), sizeof(float) * nlocs, cudaMemcpyHostToDevice));

  if (prim->banner_arg) printf("%s_%03d_%03d\n", prim->banner, prim->banner_arg, iters);
  else printf("%s_%03d\n", prim->banner, iters);
  fflush(stdout);

  Args a{};
  a.storage = storage;
  a.d = *cpuLockData;
  a.perSM = perSM;
  a.numAtBarr = (unsigned)groups;
  a.groups = groups;
  a.numTBs_perSM = numTBs_perSM;
  a.exch = groups;
  a.iters = iters;
  a.nldst = nldst;
  a.NUM_SM = NUM_SM;
  a.MAX_BLOCKS = MAX_BLOCKS;

  float total = 0.0f;
  auto run = [&](auto&& fn) { launch_timed(fn, repeats, &total); };
  // the hybrid picks the library barrier for few CTAs per SM (main.cu:1595-1610)
  const bool hybrid_ccg = numTBs_perSM < (MAX_BLOCKS / NUM_SM) / 4;
  const int sem_size = p == 11 || p == 19 || p == 27 ? 120 : prim->banner_arg;
  cudaMutex_t mtx = 0;
  cudaSemaphore_t sem = 0;
  if (p >= 4 && p <= 7) mtx = p - 4;                  // main.cu:2633-2648
  if (p >= 20 && p <= 23) mtx = p - 16;
  if ((p >= 8 && p <= 19) || (p >= 32 && p <= 35)) sem = (p - 8) % 4 + ((p >= 12 && p <= 15) || p >= 32 ? 4 : 0);
  if (p >= 24 && p <= 31) sem = p - 12;
  if (p == 4 || p == 20) CK(cudaMutexCreateSpin(&mtx, mtx));
  if (p == 5 || p == 21) CK(cudaMutexCreateEBO(&mtx, mtx));
  if (p == 6 || p == 22) CK(cudaMutexCreateSleep(&mtx, mtx));
  if (p == 7 || p == 23) CK(cudaMutexCreateFA(&mtx, mtx));
  if ((p >= 8 && p <= 11) || (p >= 16 && p <= 19) || (p >= 24 && p <= 27))
    CK(cudaSemaphoreCreateSpin(&sem, sem, sem_size, NUM_SM));
  if ((p >= 12 && p <= 15) || (p >= 28 && p <= 35)) CK(cudaSemaphoreCreateEBO(&sem, sem, sem_size, NUM_SM));

  switch (p) {
    case 0: run([&] { return launch_barrier<B_TREE, false>(a, numTBs); }); break;
    case 1: run([&] { return launch_barrier<B_TREE, true>(a, numTBs); }); break;
    case 2: run([&] { return launch_barrier<B_LF, false>(a, numTBs); }); break;
    case 3: run([&] { return launch_barrier<B_LF, true>(a, numTBs); }); break;
    case 4: run([&] { return launch_mutex<M_SPIN, false>(a, numTBs, mtx); }); break;
    case 5: run([&] { return launch_mutex<M_EBO, false>(a, numTBs, mtx); }); break;
    case 6: run([&] { return launch_mutex<M_SLEEP, false>(a, numTBs, mtx); }); break;
    case 7: run([&] { return launch_mutex<M_FA, false>(a, numTBs, mtx); }); break;
    case 8: case 9: case 10: case 11:
      run([&] { return launch_semaphore<S_SPIN, false, false>(a, numTBs, sem); }); break;
    case 12: case 13: case 14: case 15:
      run([&] { return launch_semaphore<S_EBO, false, false>(a, numTBs, sem); }); break;
    case 16: case 17: case 18: case 19:
      run([&] { return launch_semaphore<S_SPIN, true, false>(a, numTBs, sem); }); break;
    case 20: run([&] { return launch_mutex<M_SPIN, true>(a, numTBs, mtx); }); break;
    case 21: run([&] { return launch_mutex<M_EBO, true>(a, numTBs, mtx); }); break;
    case 22: run([&] { return launch_mutex<M_SLEEP, true>(a, numTBs, mtx); }); break;
    case 23: run([&] { return launch_mutex<M_FA, true>(a, numTBs, mtx); }); break;
    case 24: case 25: case 26: case 27:
      run([&] { return launch_semaphore<S_SPIN, false, true>(a, numTBs, sem); }); break;
    case 28: case 29: case 30: case 31:
      run([&] { return launch_semaphore<S_EBO, false, true>(a, numTBs, sem); }); break;
    case 32: case 33: case 34: case 35:
      run([&] { return launch_semaphore<S_EBO, true, false>(a, numTBs, sem); }); break;
    case 37: run([&] { return launch_barrier<B_SRB, false>(a, numTBs); }); break;
    case 38: run([&] { return launch_barrier<B_SRB, true>(a, numTBs); }); break;
    case 39:
    case 40:
      // the naive barrier counts every CTA; its exchange stride is numTBs (main.cu:1612-1642, 1800-1834)
      a.numAtBarr = (unsigned)numTBs;
      a.exch = numTBs;
      if (p == 39) run([&] { return launch_barrier<B_NAIVE, false>(a, numTBs); });
      else run([&] { return launch_barrier<B_NAIVE, true>(a, numTBs); });
      break;
    case 41:
    case 42:
      a.numAtBarr = (unsigned)(numTBs * kThreads);  // main.cu:1650, 1842
      if (p == 41) run([&] { return launch_barrier<B_NAIVEALL, false>(a, numTBs); });
      else run([&] { return launch_barrier<B_NAIVEALL, true>(a, numTBs); });
      break;
    case 43:
      if (hybrid_ccg) run([&] { return launch_barrier<B_CCG, false>(a, numTBs); });
      else run([&] { return launch_barrier<B_SRB, false>(a, numTBs); });
      break;
    case 44:
      if (hybrid_ccg) run([&] { return launch_barrier<B_CCG, true>(a, numTBs); });
      else run([&] { return launch_barrier<B_SRB, true>(a, numTBs); });
      break;
    case 45: run([&] { return launch_barrier<B_CCG, false>(a, numTBs); }); break;
    case 46: run([&] { return launch_barrier<B_CCG, true>(a, numTBs); }); break;
    default:
      fprintf(stderr, "ERROR: Unknown syncPrim: %d\n", p);
      return -1;
  }
  printf("elapsed time: %f ms, average: %f ms\n", total, total / (float)repeats);
  fflush(stdout);

  const unsigned int st = gsrb_cudalocks_status(), lst = gsrb_cudalocks_local_status();
  CK(cudaMemcpy(host.data(), storage, sizeof(float) * nlocs, cudaMemcpyDeviceToHost));
  if (out_path) {
    FILE* f = fopen(out_path, "wb");
    if (!f || fwrite(host.data(), sizeof(float), nlocs, f) != (size_t)nlocs) {
      fprintf(stderr, "ERROR: cannot write %s\n", out_path);
      return -1;
    }
    fclose(f);
  }
  cudaFree(storage);
  cudaFree(perSM);
  CK(cudaLocksDestroy());
  if (st != 0 || lst != 0) {
    fprintf(stderr, "ERROR: %s: a wait ran out (lock status %u, local barrier status %u)\n", prim->name, st, lst);
    return -1;
  }

  const std::vector<float> want = golden(p, nldst, numTBs, iters, repeats, NUM_SM, nlocs);
  fprintf(stdout, "Comparing GPU results to golden results:\n");
  unsigned int errors = 0;
  for (int i = 0; i < nlocs; ++i) {
    if (std::fabs(host[i] - want[i]) > 1e-5f) {
      if (errors < 20) fprintf(stderr, "\tERROR: storage[%d] = %f, golden[%d] = %f\n", i, host[i], i, want[i]);
      ++errors;
    }
  }
  if (errors > 0) {
    fprintf(stderr, "ERROR: %s has %u output errors\n", prim->name, errors);
    return -1;
  }
  fprintf(stdout, "PASSED!\n");
  return 0;
}
