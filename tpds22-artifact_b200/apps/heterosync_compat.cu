// Heterosync-style program written against the drop-in API only: the
// reference-named host API (cudaLocksInit, cudaMutexCreate*, cudaSemaphoreCreate*,
// gsrb/cudaLocks.h) and device API (joinBarrier_helper*, joinLFBarrier_helper,
// cudaMutex*Lock/Unlock, cudaSemaphore*Wait/Post*, gsrb/cudaLocks.cuh), with
// the harness's own conventions (Heterosync/main.cu: smID = blockIdx % NUM_SM,
// perSM_blockID = blockIdx / NUM_SM, a zeroed per-SM barrier buffer of
// NUM_SM * MAX_BLOCKS * 2 words).  Each kernel checks its own result:
//   barriers   -- message passing through the barrier (every CTA writes its
//                 slot, barrier, reads its neighbour's slot, barrier): no stale reads
//   mutexes    -- non-atomic read-modify-write of one counter inside the lock:
//                 exact final count
//   semaphores -- holders inside at once never exceed the capacity; writers
//                 hold alone; exact counts
// Prints one PASS/FAIL line per case; the exit status is the number of failures.
// Grids are checked for co-residency before launch (a non-co-resident grid
// would make any grid barrier wait out its timeout).
#include <cstdio>
#include <cstdlib>

#include "gsrb/cudaLocks.cuh"

#define CK(x)                                                                         \
  do {                                                                                \
    cudaError_t e_ = (x);                                                             \
    if (e_ != cudaSuccess) {                                                          \
      fprintf(stderr, "%s failed: %s\n", #x, cudaGetErrorString(e_));                 \
      exit(100);                                                                      \
    }                                                                                 \
  } while (0)

namespace {

constexpr int kThreads = 64;
constexpr int kMaxBlocks = 2048;

enum BarKind { BAR_SRB = 0, BAR_NAIVE = 1, BAR_TREE = 2, BAR_LF = 3 };

template <int K>
__device__ void join(cudaLockData_t d, unsigned int* perSM, int NUM_SM) {
  const int smID = blockIdx.x % NUM_SM, perSM_blockID = blockIdx.x / NUM_SM;
  const int numTBs_perSM = (gridDim.x + NUM_SM - 1) / NUM_SM;
  const bool master = threadIdx.x == 0;
  if (K == BAR_SRB)
    joinBarrier_helperSRB(d.barrierBuffers, perSM, NUM_SM, smID, perSM_blockID, numTBs_perSM, master, kMaxBlocks);
  else if (K == BAR_NAIVE)
    joinBarrier_helperNaiveSRB(d.barrierBuffers, gridDim.x, smID, master, kMaxBlocks);
  else if (K == BAR_TREE)
    joinBarrier_helper(d.barrierBuffers, perSM, NUM_SM, smID, perSM_blockID, numTBs_perSM, master, kMaxBlocks);
  else
    joinLFBarrier_helper(d.barrierBuffers, perSM, NUM_SM, smID, perSM_blockID, numTBs_perSM, d.arrayStride,
                         kMaxBlocks);
}

template <int K>
__global__ void barrier_kernel(cudaLockData_t d, unsigned int* perSM, int NUM_SM, int iters, unsigned int* slots,
                               unsigned int* stale) {
  const unsigned int G = gridDim.x, b = blockIdx.x;
  for (int it = 1; it <= iters; ++it) {
    if (threadIdx.x == 0) slots[b] = (unsigned int)it * G + b;
    join<K>(d, perSM, NUM_SM);
    if (threadIdx.x == 0) {
      const unsigned int nb = (b + 1) % G;
      const unsigned int v = *(volatile unsigned int*)&slots[nb];
      if (v != (unsigned int)it * G + nb) atomicAdd(stale, 1u);
    }
    join<K>(d, perSM, NUM_SM);
  }
}

enum MutexKind { MUT_SPIN = 0, MUT_EBO = 1, MUT_FA = 2, MUT_SLEEP = 3 };

template <int K>
__global__ void mutex_kernel(cudaLockData_t d, cudaMutex_t m, int NUM_SM, int iters, unsigned int* counter) {
  for (int it = 0; it < iters; ++it) {
    unsigned int loc = 0;
    if (K == MUT_SPIN) cudaMutexSpinLock(m, d.mutexBufferHeads, NUM_SM);
    else if (K == MUT_EBO) cudaMutexEBOLock(m, d.mutexBufferHeads, NUM_SM);
    else if (K == MUT_FA) cudaMutexFALock(m, d.mutexBufferHeads, d.mutexBufferTails, NUM_SM);
    else loc = cudaMutexSleepLock(m, d.mutexBuffers, d.mutexBufferTails, kMaxBlocks, d.arrayStride, NUM_SM);
    if (threadIdx.x == 0) {
      // non-atomic read-modify-write: exact only under mutual exclusion
      volatile unsigned int* c = counter;
      const unsigned int v = *c;
      *c = v + 1;
      __threadfence();
    }
    __syncthreads();
    if (K == MUT_SPIN) cudaMutexSpinUnlock(m, d.mutexBufferHeads, NUM_SM);
    else if (K == MUT_EBO) cudaMutexEBOUnlock(m, d.mutexBufferHeads, NUM_SM);
    else if (K == MUT_FA) cudaMutexFAUnlock(m, d.mutexBufferTails, NUM_SM);
    else cudaMutexSleepUnlock(m, d.mutexBuffers, loc, kMaxBlocks, d.arrayStride, NUM_SM);
  }
}

// counters: [0] writers done, [1] readers done, [2] inside now, [3] max inside, [4] writer overlaps
__global__ void semaphore_kernel(cudaLockData_t d, cudaSemaphore_t s, unsigned int cap, int NUM_SM, int iters,
                                 unsigned int* counters) {
  const bool writer = blockIdx.x % 10 == 0;
  for (int it = 0; it < iters; ++it) {
    cudaSemaphoreSpinWaitPriority(s, writer, cap, d.semaphoreBuffers, NUM_SM);
    if (threadIdx.x == 0) {
      const unsigned int now = atomicAdd(&counters[2], writer ? 1000u : 1u) + (writer ? 1000u : 1u);
      if (writer && now != 1000u) atomicAdd(&counters[4], 1u);
      if (!writer && now >= 1000u) atomicAdd(&counters[4], 1u);
      atomicMax(&counters[3], now < 1000u ? now : 0u);
      atomicSub(&counters[2], writer ? 1000u : 1u);
      atomicAdd(&counters[writer ? 0 : 1], 1u);
    }
    __syncthreads();
    cudaSemaphoreSpinPostPriority(s, writer, cap, d.semaphoreBuffers, NUM_SM);
  }
}

int g_fail = 0;

void report(bool ok, const char* name, const char* detail) {
  printf("%s %s%s%s\n", ok ? "PASS" : "FAIL", name, detail[0] ? " " : "", detail);
  if (!ok) ++g_fail;
}

bool coresident(const void* fn, int grid) {
  int nb = 0, nsm = 0, dev = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, kThreads, 0));
  return grid <= nb * nsm;
}

template <int K>
void run_barrier(const char* name, int NUM_SM, int grid, unsigned int* perSM) {
  const void* fn = (const void*)barrier_kernel<K>;
  if (!coresident(fn, grid)) {
    report(false, name, "(grid not co-resident)");
    return;
  }
  unsigned int *slots, *stale;
  CK(cudaMalloc(&slots, sizeof(unsigned int) * grid));
  CK(cudaMalloc(&stale, sizeof(unsigned int)));
  CK(cudaMemset(slots, 0, sizeof(unsigned int) * grid));
  CK(cudaMemset(stale, 0, sizeof(unsigned int)));
  barrier_kernel<K><<<grid, kThreads>>>(*cpuLockData, perSM, NUM_SM, 50, slots, stale);
  CK(cudaDeviceSynchronize());
  unsigned int h = 0;
  CK(cudaMemcpy(&h, stale, 4, cudaMemcpyDeviceToHost));
  const unsigned int st = gsrb_cudalocks_status();
  char buf[96];
  snprintf(buf, sizeof buf, "stale=%u status=%u", h, st);
  report(h == 0 && st == 0, name, buf);
  cudaFree(slots);
  cudaFree(stale);
}

template <int K>
void run_mutex(const char* name, int NUM_SM, int grid, cudaMutex_t m) {
  const void* fn = (const void*)mutex_kernel<K>;
  if (!coresident(fn, grid)) {
    report(false, name, "(grid not co-resident)");
    return;
  }
  unsigned int* counter;
  CK(cudaMalloc(&counter, sizeof(unsigned int)));
  CK(cudaMemset(counter, 0, sizeof(unsigned int)));
  const int iters = 20;
  mutex_kernel<K><<<grid, kThreads>>>(*cpuLockData, m, NUM_SM, iters, counter);
  CK(cudaDeviceSynchronize());
  unsigned int h = 0;
  CK(cudaMemcpy(&h, counter, 4, cudaMemcpyDeviceToHost));
  const unsigned int st = gsrb_cudalocks_status();
  char buf[96];
  snprintf(buf, sizeof buf, "count=%u want=%u status=%u", h, (unsigned)(grid * iters), st);
  report(h == (unsigned)(grid * iters) && st == 0, name, buf);
  cudaFree(counter);
}

}  // namespace

int main() {
  int dev = 0, NUM_SM = 0;
  CK(cudaSetDevice(dev));
  CK(cudaDeviceGetAttribute(&NUM_SM, cudaDevAttrMultiProcessorCount, dev));
  const int grid = 2 * NUM_SM;
  // the harness's call shape (Heterosync/main.cu:2542): MAX_BLOCKS, 8 * NUM_SM mutexes, 24 * NUM_SM semaphores
  CK(cudaLocksInit(kMaxBlocks, 8 * NUM_SM, 24 * NUM_SM, false, NUM_SM));
  unsigned int* perSM = nullptr;
  CK(cudaMalloc(&perSM, sizeof(unsigned int) * (size_t)NUM_SM * kMaxBlocks * 2));
  CK(cudaMemset(perSM, 0, sizeof(unsigned int) * (size_t)NUM_SM * kMaxBlocks * 2));

  run_barrier<BAR_SRB>("joinBarrier_helperSRB", NUM_SM, grid, perSM);
  run_barrier<BAR_NAIVE>("joinBarrier_helperNaiveSRB", NUM_SM, grid, perSM);
  run_barrier<BAR_TREE>("joinBarrier_helper", NUM_SM, grid, perSM);
  run_barrier<BAR_LF>("joinLFBarrier_helper", NUM_SM, grid, perSM);
  run_barrier<BAR_LF>("joinLFBarrier_helper(1 CTA/SM)", NUM_SM, NUM_SM, perSM);

  cudaMutex_t ms, me, mf, msl;
  CK(cudaMutexCreateSpin(&ms, 0));
  CK(cudaMutexCreateEBO(&me, 1));
  CK(cudaMutexCreateFA(&mf, 2));
  CK(cudaMutexCreateSleep(&msl, 0));
  run_mutex<MUT_SPIN>("cudaMutexSpinLock", NUM_SM, grid, ms);
  run_mutex<MUT_EBO>("cudaMutexEBOLock", NUM_SM, grid, me);
  run_mutex<MUT_FA>("cudaMutexFALock", NUM_SM, grid, mf);
  run_mutex<MUT_SLEEP>("cudaMutexSleepLock", NUM_SM, grid, msl);

  for (unsigned int cap : {1u, 10u}) {
    cudaSemaphore_t s;
    CK(cudaSemaphoreCreateSpin(&s, cap == 1u ? 0 : 1, cap, NUM_SM));
    unsigned int* c;
    CK(cudaMalloc(&c, sizeof(unsigned int) * 8));
    CK(cudaMemset(c, 0, sizeof(unsigned int) * 8));
    const int iters = 10;
    if (!coresident((const void*)semaphore_kernel, grid)) {
      report(false, "cudaSemaphoreSpinWaitPriority", "(grid not co-resident)");
      continue;
    }
    semaphore_kernel<<<grid, kThreads>>>(*cpuLockData, s, cap, NUM_SM, iters, c);
    CK(cudaDeviceSynchronize());
    unsigned int h[8];
    CK(cudaMemcpy(h, c, sizeof h, cudaMemcpyDeviceToHost));
    unsigned int writers = 0;
    for (int b = 0; b < grid; ++b) writers += (b % 10 == 0);
    const unsigned int st = gsrb_cudalocks_status();
    const bool ok = h[0] == writers * iters && h[1] == (grid - writers) * iters && h[3] <= cap && h[4] == 0 && st == 0;
    char buf[160];
    snprintf(buf, sizeof buf, "S=%u writers=%u readers=%u max_inside=%u overlaps=%u status=%u", cap, h[0], h[1], h[3],
             h[4], st);
    report(ok, "cudaSemaphoreSpinWaitPriority", buf);
    cudaFree(c);
  }
  cudaFree(perSM);
  CK(cudaLocksDestroy());
  return g_fail;
}
