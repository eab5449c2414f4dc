// Lock state (the cudaLocks host API) and the mutex / semaphore
// microbenchmarks.
//
// Reference host API: Heterosync/cudaLocks.cu:3-102 (cudaLocksInit /
// cudaLocksDestroy), the *Create* functions of cudaLocksMutex*.cu and
// cudaLocksSemaphore{Spin,EBO}.cu.  Reference microbenchmarks:
// kernelSpinLockSemaphorePriority and friends, Heterosync/main.cu:702-1493.
//
// The semaphore microbenchmark measured here (configuration 2): 148*k CTAs,
// one writer CTA per `writer_every` CTAs, every holder adds 1 to a shared
// counter `incs` times -- writers with a plain (non-atomic) read-modify-write
// of W, so any overlap between two writers loses updates; readers with an
// atomic add to R.  An occupancy gauge checks exclusion (a writer must be alone,
// at most `capacity` readers at a time).  W and R are checked exactly.
#include "internal.h"
#include <stddef.h>
#include "gsrb/locks.cuh"
#include "gsrb/cudaLocks.h"

#include <string.h>

using namespace gsrbrt;

namespace {

// Every lock buffer is preceded by one 128-byte line whose word 0 is the status
// word (gsrb::lock_status_word).
cudaError_t alloc_with_header(void** user, size_t bytes) {
  char* base = nullptr;
  cudaError_t e = cudaMalloc(&base, bytes + 128);
  if (e != cudaSuccess) return e;
  e = cudaMemset(base, 0, bytes + 128);
  if (e != cudaSuccess) {
    cudaFree(base);
    return e;
  }
  *user = base + 128;
  return cudaSuccess;
}
void free_with_header(void* user) {
  if (user) cudaFree((char*)user - 128);
}
uint32_t read_clear_word(uint32_t* w) {
  uint32_t v = 0;
  cudaMemcpy(&v, w, 4, cudaMemcpyDeviceToHost);
  if (v) cudaMemset(w, 0, 4);
  return v;
}

uint32_t read_clear_status(void* user) {
  if (!user) return 0;
  return read_clear_word((uint32_t*)((char*)user - 128));
}

// Status words of the stateless barrier wrappers (gsrb/cudaLocks.cuh): the
// native slot at the start of barrierBuffers, and the lock-free barrier's slot
// after its 2 * arrayStride flag words.
uint32_t read_clear_barrier_status(uint32_t* barrierBuffers, int arrayStride) {
  if (!barrierBuffers) return 0;
  const size_t status_word = offsetof(gsrb::BarrierSlot, status) / sizeof(uint32_t);
  uint32_t v = read_clear_word(barrierBuffers + status_word);
  const uint32_t v2 = read_clear_word(barrierBuffers + 2 * (size_t)arrayStride + status_word);
  return v ? v : v2;
}

__global__ void ring_init_kernel(int32_t* ring, size_t n, int stride) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    ring[i] = (i % (size_t)stride == 0) ? 1 : -1;
}

struct LockState {
  cudaLockData_t d;  // device pointers (user views)
};

cudaError_t locks_alloc(LockState* L, int maxBlocks, int numMutexes, int numSems, int numSM) {
  memset(L, 0, sizeof(*L));
  L->d.maxBufferSize = maxBlocks;
  L->d.arrayStride = (maxBlocks + numSM) / 16 * 16;
  if (L->d.arrayStride < 16) L->d.arrayStride = 16;
  L->d.mutexCount = numMutexes;
  L->d.semaphoreCount = numSems;
  // barrierBuffers: the reference's 2*arrayStride words (lock-free barrier
  // flags) followed by that barrier's status slot, and at least one native
  // barrier slot plus per-group counters for the stateless device API
  size_t bb = sizeof(uint32_t) * 2 * (size_t)L->d.arrayStride + sizeof(gsrb::BarrierSlot);
  const size_t native = sizeof(gsrb::BarrierSlot) + sizeof(gsrb::GroupSlot) * (size_t)(numSM > 0 ? numSM : 1);
  if (bb < native) bb = native;
  cudaError_t e = alloc_with_header((void**)&L->d.barrierBuffers, bb);
  if (!e) e = alloc_with_header((void**)&L->d.mutexBuffers, sizeof(int) * (size_t)L->d.arrayStride * numMutexes);
  if (!e) e = alloc_with_header((void**)&L->d.mutexBufferHeads, sizeof(uint32_t) * (size_t)numMutexes);
  if (!e) e = alloc_with_header((void**)&L->d.mutexBufferTails, sizeof(uint32_t) * (size_t)numMutexes);
  if (!e) e = alloc_with_header((void**)&L->d.semaphoreBuffers, sizeof(uint32_t) * 5 * (size_t)numSems);
  if (!e) {
    ring_init_kernel<<<64, 256>>>(L->d.mutexBuffers, (size_t)L->d.arrayStride * numMutexes, L->d.arrayStride);
    e = cudaGetLastError();
  }
  if (!e) e = cudaDeviceSynchronize();
  return e;
}

void locks_free(LockState* L) {
  free_with_header(L->d.barrierBuffers);
  free_with_header(L->d.mutexBuffers);
  free_with_header(L->d.mutexBufferHeads);
  free_with_header(L->d.mutexBufferTails);
  free_with_header(L->d.semaphoreBuffers);
  memset(L, 0, sizeof(*L));
}

// Semaphore record of the reference create (count + 1 in words 0 and 3, zeros
// elsewhere) for every SM id (Heterosync/cudaLocksSemaphoreSpin.cu:14-27).
cudaError_t sem_create(uint32_t* semBuffers, int semNum, unsigned count, int numSM, cudaStream_t s) {
  const size_t words = 5 * (size_t)numSM;
  uint32_t* host = (uint32_t*)calloc(words, sizeof(uint32_t));
  if (!host) return cudaErrorMemoryAllocation;
  for (int id = 0; id < numSM; ++id) {
    host[id * 5 + 0] = count + 1;
    host[id * 5 + 3] = count + 1;
  }
  cudaError_t e = cudaMemcpyAsync(semBuffers + (size_t)semNum * 5 * numSM, host, words * 4, cudaMemcpyHostToDevice, s);
  if (!e) e = cudaStreamSynchronize(s);
  free(host);
  return e;
}

// ---------------------------------------------------------------- benches ---
struct Counters {
  uint32_t W, R, inside, max_readers, violations, acquires, timeouts, pad;
};

template <int KIND>
__global__ void __launch_bounds__(256)
semaphore_bench_kernel(uint32_t* rec, const void* statbuf, int writer_every, int iters, int incs,
                       uint64_t timeout_ns, uint32_t spin_ns, Counters* c) {
  const bool writer = writer_every > 0 && (blockIdx.x % (uint32_t)writer_every) == 0;
  const uint32_t cap = rec[3] - 1;
  for (int it = 0; it < iters; ++it) {
    bool ok = true;
    if (KIND == GSRB_SEM_NONE)
      ok = true;  // the critical section alone (its timing is the semaphore's bound)
    else if (KIND == GSRB_SEM_PRIORITY)
      ok = gsrb::psem_wait(gsrb::PrioritySem{rec}, writer, statbuf, timeout_ns, spin_ns);
    else
      ok = gsrb::refsem_wait(gsrb::RefSem{rec}, writer, rec[3], KIND == GSRB_SEM_REF_PRIORITY ||
                             KIND == GSRB_SEM_REF_PRIORITY_EBO, KIND == GSRB_SEM_REF_EBO ||
                             KIND == GSRB_SEM_REF_PRIORITY_EBO, statbuf, timeout_ns);
    if (!ok) {
      if (threadIdx.x == 0) atomicAdd(&c->timeouts, 1u);
      break;  // lock loops have no cluster barriers: a per-CTA exit is safe
    }
    if (threadIdx.x == 0) {
      if (writer) {
        if (atomicAdd(&c->inside, 1000u) != 0u) atomicAdd(&c->violations, 1u);
        volatile uint32_t* W = &c->W;
        for (int k = 0; k < incs; ++k) *W = *W + 1u;
        atomicSub(&c->inside, 1000u);
      } else {
        const uint32_t in = atomicAdd(&c->inside, 1u) + 1u;
        if (in >= 1000u || in > cap) atomicAdd(&c->violations, 1u);
        atomicMax(&c->max_readers, in);
        for (int k = 0; k < incs; ++k) atomicAdd(&c->R, 1u);
        atomicSub(&c->inside, 1u);
      }
      atomicAdd(&c->acquires, 1u);
      __threadfence();
    }
    if (KIND == GSRB_SEM_NONE) {
      __syncthreads();
    } else if (KIND == GSRB_SEM_PRIORITY) {
      gsrb::psem_post(gsrb::PrioritySem{rec}, writer);
    } else {
      if (!gsrb::refsem_post(gsrb::RefSem{rec}, writer, rec[3], KIND == GSRB_SEM_REF_PRIORITY ||
                             KIND == GSRB_SEM_REF_PRIORITY_EBO, statbuf, timeout_ns)) {
        if (threadIdx.x == 0) atomicAdd(&c->timeouts, 1u);
        break;
      }
    }
  }
}

// Fault test: one CTA posts the native priority semaphore without having
// waited on it (an over-post, the usage error the count gauge catches), then
// waits on it as a reader and as a writer; both waits must report the
// invariant at once instead of running into their deadline.
__global__ void __launch_bounds__(256)
semaphore_overpost_kernel(uint32_t* rec, const void* statbuf, uint64_t timeout_ns, uint32_t* out) {
  gsrb::psem_post(gsrb::PrioritySem{rec}, false);
  const bool r = gsrb::psem_wait(gsrb::PrioritySem{rec}, false, statbuf, timeout_ns, 0);
  const bool w = gsrb::psem_wait(gsrb::PrioritySem{rec}, true, statbuf, timeout_ns, 0);
  if (threadIdx.x == 0) {
    out[0] = r ? 1u : 0u;
    out[1] = w ? 1u : 0u;
  }
}

// One CTA, in order: enters as a reader (count max - 1), waits as a writer
// while still holding the reader slot (the count never reaches max: that wait
// runs into its short deadline, after its ticket was served), leaves as a
// reader, then waits as a writer again with the next ticket.  The second
// writer is served only if the first handed its turn on.
__global__ void __launch_bounds__(32)
semaphore_writer_timeout_kernel(uint32_t* rec, const void* statbuf, uint64_t short_ns, uint64_t timeout_ns,
                                uint32_t* out) {
  const gsrb::PrioritySem s{rec};
  const bool r = gsrb::psem_wait(s, false, statbuf, timeout_ns, 0);
  const bool w1 = gsrb::psem_wait(s, true, statbuf, short_ns, 0);
  if (r) gsrb::psem_post(s, false);
  if (w1) gsrb::psem_post(s, true);
  const bool w2 = gsrb::psem_wait(s, true, statbuf, timeout_ns, 0);
  if (w2) gsrb::psem_post(s, true);
  if (threadIdx.x == 0) {
    out[0] = r ? 1u : 0u;
    out[1] = w1 ? 1u : 0u;
    out[2] = w2 ? 1u : 0u;
    out[3] = gsrb::ptx::ld_relaxed_gpu(rec);      // count after the run (max when balanced)
    out[4] = gsrb::ptx::ld_relaxed_gpu(rec + 4);  // serving
  }
}

template <int KIND>
__global__ void __launch_bounds__(256)
mutex_bench_kernel(uint32_t* heads, uint32_t* tails, int32_t* ring, uint32_t ring_max, const void* statbuf,
                   int iters, int incs, uint64_t timeout_ns, Counters* c) {
  for (int it = 0; it < iters; ++it) {
    bool ok;
    uint32_t slot = 0;
    if (KIND == GSRB_MUTEX_SPIN) ok = gsrb::mutex_spin_lock(heads, statbuf, timeout_ns, false);
    else if (KIND == GSRB_MUTEX_EBO) ok = gsrb::mutex_spin_lock(heads, statbuf, timeout_ns, true);
    else if (KIND == GSRB_MUTEX_FA) ok = gsrb::mutex_fa_lock(heads, tails, statbuf, timeout_ns);
    else ok = gsrb::mutex_sleep_lock(ring, tails, ring_max, statbuf, timeout_ns, &slot);
    if (!ok) {
      if (threadIdx.x == 0) atomicAdd(&c->timeouts, 1u);
      break;
    }
    if (threadIdx.x == 0) {
      if (atomicAdd(&c->inside, 1u) != 0u) atomicAdd(&c->violations, 1u);
      volatile uint32_t* W = &c->W;
      for (int k = 0; k < incs; ++k) *W = *W + 1u;
      atomicSub(&c->inside, 1u);
      atomicAdd(&c->acquires, 1u);
      __threadfence();
    }
    if (KIND == GSRB_MUTEX_SPIN || KIND == GSRB_MUTEX_EBO) gsrb::mutex_spin_unlock(heads);
    else if (KIND == GSRB_MUTEX_FA) gsrb::mutex_fa_unlock(tails);
    else gsrb::mutex_sleep_unlock(ring, slot, ring_max);
  }
}

const void* sem_fn(int kind) {
  switch (kind) {
    case GSRB_SEM_REF_SPIN: return (const void*)semaphore_bench_kernel<GSRB_SEM_REF_SPIN>;
    case GSRB_SEM_REF_EBO: return (const void*)semaphore_bench_kernel<GSRB_SEM_REF_EBO>;
    case GSRB_SEM_REF_PRIORITY: return (const void*)semaphore_bench_kernel<GSRB_SEM_REF_PRIORITY>;
    case GSRB_SEM_REF_PRIORITY_EBO: return (const void*)semaphore_bench_kernel<GSRB_SEM_REF_PRIORITY_EBO>;
    case GSRB_SEM_PRIORITY: return (const void*)semaphore_bench_kernel<GSRB_SEM_PRIORITY>;
    case GSRB_SEM_NONE: return (const void*)semaphore_bench_kernel<GSRB_SEM_NONE>;
    default: return nullptr;
  }
}
const void* mutex_fn(int kind) {
  switch (kind) {
    case GSRB_MUTEX_SPIN: return (const void*)mutex_bench_kernel<GSRB_MUTEX_SPIN>;
    case GSRB_MUTEX_EBO: return (const void*)mutex_bench_kernel<GSRB_MUTEX_EBO>;
    case GSRB_MUTEX_FA: return (const void*)mutex_bench_kernel<GSRB_MUTEX_FA>;
    case GSRB_MUTEX_SLEEP: return (const void*)mutex_bench_kernel<GSRB_MUTEX_SLEEP>;
    default: return nullptr;
  }
}

}  // namespace

struct gsrb_locks {
  gsrb_ctx* ctx;
  LockState st;
  int num_sm;
};

extern "C" {

cudaLockData_t* cpuLockData = nullptr;

gsrb_status_t gsrb_locks_create(gsrb_ctx_t ctx, int32_t maxBlocks, int32_t numMutexes, int32_t numSemaphores,
                                int32_t numSM, gsrb_locks_t* out) {
  if (!ctx || !out || maxBlocks <= 0 || numMutexes <= 0 || numSemaphores <= 0 || numSM <= 0) return GSRB_ERR_ARG;
  gsrb_locks* L = new gsrb_locks();
  L->ctx = ctx;
  L->num_sm = numSM;
  cudaError_t e = locks_alloc(&L->st, maxBlocks, numMutexes, numSemaphores, numSM);
  if (e) {
    locks_free(&L->st);
    delete L;
    return cuda_err(e, "locks_alloc");
  }
  *out = L;
  return GSRB_OK;
}

gsrb_status_t gsrb_locks_destroy(gsrb_locks_t L) {
  if (!L) return GSRB_ERR_ARG;
  cudaStreamSynchronize(L->ctx->stream);
  locks_free(&L->st);
  delete L;
  return GSRB_OK;
}

gsrb_status_t gsrb_locks_data(gsrb_locks_t L, gsrb_lock_data_t* out) {
  if (!L || !out) return GSRB_ERR_ARG;
  out->maxBufferSize = L->st.d.maxBufferSize;
  out->arrayStride = L->st.d.arrayStride;
  out->mutexCount = L->st.d.mutexCount;
  out->semaphoreCount = L->st.d.semaphoreCount;
  out->barrierBuffers = L->st.d.barrierBuffers;
  out->mutexBuffers = L->st.d.mutexBuffers;
  out->mutexBufferHeads = L->st.d.mutexBufferHeads;
  out->mutexBufferTails = L->st.d.mutexBufferTails;
  out->semaphoreBuffers = L->st.d.semaphoreBuffers;
  return GSRB_OK;
}

gsrb_status_t gsrb_semaphore_init(gsrb_locks_t L, int32_t semNum, uint32_t count, int32_t numSM) {
  if (!L || semNum < 0 || numSM <= 0 || (int64_t)(semNum + 1) * numSM > L->st.d.semaphoreCount) return GSRB_ERR_ARG;
  GSRB_CUDA(sem_create(L->st.d.semaphoreBuffers, semNum, count, numSM, L->ctx->stream));
  return GSRB_OK;
}

gsrb_status_t gsrb_locks_status(gsrb_locks_t L, uint32_t* code) {
  if (!L) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaStreamSynchronize(L->ctx->stream));
  uint32_t v = 0;
  void* bufs[] = {L->st.d.barrierBuffers, L->st.d.mutexBuffers, L->st.d.mutexBufferHeads,
                  L->st.d.mutexBufferTails, L->st.d.semaphoreBuffers};
  for (void* b : bufs) {
    uint32_t s = read_clear_status(b);
    if (!v) v = s;
  }
  if (code) *code = v;
  return map_dev(v);
}

gsrb_status_t gsrb_semaphore_bench(gsrb_ctx_t ctx, const gsrb_cfg_t* cfgin, int32_t kind, uint32_t capacity,
                                   int32_t writer_every, int32_t iters, int32_t incs, uint32_t* d_counters) {
  if (!ctx || !d_counters || capacity < 1 || capacity > 60000 || writer_every < 0 || iters < 0 || incs < 0)
    return GSRB_ERR_ARG;
  const void* fn = sem_fn(kind);
  if (!fn) return GSRB_ERR_ARG;
  gsrb_cfg_t c = resolve_cfg(ctx, cfgin);
  c.cluster = 1;
  if (c.threads > 256 || c.threads % 32) return GSRB_ERR_ARG;
  const int grid = grid_of(ctx, c);
  gsrb_locks_t L = nullptr;
  gsrb_status_t st = gsrb_locks_create(ctx, grid, 1, 1, 1, &L);
  if (st) return st;
  st = gsrb_semaphore_init(L, 0, capacity, 1);
  if (!st) {
    std::lock_guard<std::mutex> g(ctx->mu);
    uint32_t* rec = L->st.d.semaphoreBuffers;
    const void* statbuf = rec;
    uint64_t to = (uint64_t)c.timeout_ms * 1000000ull;
    uint32_t spin = (uint32_t)c.spin_ns;
    Counters* cc = (Counters*)d_counters;
    void* args[] = {&rec, &statbuf, &writer_every, &iters, &incs, &to, &spin, &cc};
    st = launch_persistent(ctx, fn, grid, c.threads, 0, 1, c.launch_mode == 1 ? 0 : 1, args);
  }
  gsrb_status_t st2 = gsrb_locks_status(L, nullptr);
  gsrb_locks_destroy(L);
  return st ? st : st2;
}

gsrb_status_t gsrb_semaphore_fault_overpost(gsrb_ctx_t ctx, uint32_t capacity, uint32_t* d_out) {
  if (!ctx || !d_out || capacity < 1 || capacity > 60000) return GSRB_ERR_ARG;
  gsrb_locks_t L = nullptr;
  gsrb_status_t st = gsrb_locks_create(ctx, 1, 1, 1, 1, &L);
  if (st) return st;
  st = gsrb_semaphore_init(L, 0, capacity, 1);
  if (!st) {
    std::lock_guard<std::mutex> g(ctx->mu);
    uint32_t* rec = L->st.d.semaphoreBuffers;
    const void* statbuf = rec;
    uint64_t to = 200ull * 1000000ull;  // a missed detection ends in 0.2 s, not a hang
    void* args[] = {&rec, &statbuf, &to, &d_out};
    st = launch_plain(ctx, (const void*)semaphore_overpost_kernel, dim3(1), dim3(32), 0, args);
  }
  gsrb_status_t st2 = gsrb_locks_status(L, nullptr);
  gsrb_locks_destroy(L);
  return st ? st : st2;
}

gsrb_status_t gsrb_semaphore_fault_writer_timeout(gsrb_ctx_t ctx, uint32_t capacity, uint32_t* d_out) {
  if (!ctx || !d_out || capacity < 1 || capacity > 60000) return GSRB_ERR_ARG;
  gsrb_locks_t L = nullptr;
  gsrb_status_t st = gsrb_locks_create(ctx, 1, 1, 1, 1, &L);
  if (st) return st;
  st = gsrb_semaphore_init(L, 0, capacity, 1);
  if (!st) {
    std::lock_guard<std::mutex> g(ctx->mu);
    uint32_t* rec = L->st.d.semaphoreBuffers;
    const void* statbuf = rec;
    uint64_t short_ns = 20ull * 1000000ull;  // the writer that must give up: 20 ms
    uint64_t to = 500ull * 1000000ull;       // every other wait: 0.5 s
    void* args[] = {&rec, &statbuf, &short_ns, &to, &d_out};
    st = launch_plain(ctx, (const void*)semaphore_writer_timeout_kernel, dim3(1), dim3(32), 0, args);
  }
  gsrb_status_t st2 = gsrb_locks_status(L, nullptr);
  gsrb_locks_destroy(L);
  return st ? st : st2;
}

gsrb_status_t gsrb_mutex_bench(gsrb_ctx_t ctx, const gsrb_cfg_t* cfgin, int32_t kind, int32_t iters, int32_t incs,
                               uint32_t* d_counters) {
  if (!ctx || !d_counters || iters < 0 || incs < 0) return GSRB_ERR_ARG;
  const void* fn = mutex_fn(kind);
  if (!fn) return GSRB_ERR_ARG;
  gsrb_cfg_t c = resolve_cfg(ctx, cfgin);
  c.cluster = 1;
  if (c.threads > 256 || c.threads % 32) return GSRB_ERR_ARG;
  const int grid = grid_of(ctx, c);
  gsrb_locks_t L = nullptr;
  gsrb_status_t st = gsrb_locks_create(ctx, grid, 1, 1, 1, &L);
  if (st) return st;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    uint32_t* heads = L->st.d.mutexBufferHeads;
    uint32_t* tails = L->st.d.mutexBufferTails;
    int32_t* ring = L->st.d.mutexBuffers;
    uint32_t ring_max = (uint32_t)L->st.d.maxBufferSize;  // atomicInc wrap, Heterosync/main.cu:1133
    const void* statbuf = heads;
    uint64_t to = (uint64_t)c.timeout_ms * 1000000ull;
    Counters* cc = (Counters*)d_counters;
    void* args[] = {&heads, &tails, &ring, &ring_max, &statbuf, &iters, &incs, &to, &cc};
    st = launch_persistent(ctx, fn, grid, c.threads, 0, 1, c.launch_mode == 1 ? 0 : 1, args);
  }
  gsrb_status_t st2 = gsrb_locks_status(L, nullptr);
  gsrb_locks_destroy(L);
  return st ? st : st2;
}

// ---- the reference-named host API (Heterosync/cudaLocks.h:24-27) -------------
static LockState g_compat;

cudaError_t cudaLocksInit(const int maxBlocksPerKernel, const int numMutexes, const int numSemaphores,
                          const bool pageAlign, const int NUM_SM) {
  (void)pageAlign;
  if (maxBlocksPerKernel <= 0 || numMutexes <= 0 || numSemaphores <= 0) return cudaErrorInitializationError;
  if (NUM_SM <= 0) return cudaErrorInitializationError;
  if (cpuLockData) cudaLocksDestroy();
  cudaError_t e = cudaMallocHost(&cpuLockData, sizeof(cudaLockData_t));
  if (e) return e;
  e = locks_alloc(&g_compat, maxBlocksPerKernel, numMutexes, numSemaphores, NUM_SM);
  if (e) {
    locks_free(&g_compat);
    cudaFreeHost(cpuLockData);
    cpuLockData = nullptr;
    return e;
  }
  *cpuLockData = g_compat.d;
  return cudaSuccess;
}

cudaError_t cudaLocksDestroy(void) {
  if (!cpuLockData) return cudaErrorInitializationError;
  cudaDeviceSynchronize();
  locks_free(&g_compat);
  cudaFreeHost(cpuLockData);
  cpuLockData = nullptr;
  return cudaSuccess;
}

cudaError_t cudaMutexCreateSpin(cudaMutex_t* const h, const int n) { *h = (cudaMutex_t)n; return cudaSuccess; }
cudaError_t cudaMutexCreateEBO(cudaMutex_t* const h, const int n) { *h = (cudaMutex_t)n; return cudaSuccess; }
cudaError_t cudaMutexCreateFA(cudaMutex_t* const h, const int n) { *h = (cudaMutex_t)n; return cudaSuccess; }
cudaError_t cudaMutexCreateSleep(cudaMutex_t* const h, const int n) { *h = (cudaMutex_t)n; return cudaSuccess; }

cudaError_t cudaSemaphoreCreateSpin(cudaSemaphore_t* const h, const int semNum, const unsigned int count,
                                    const int NUM_SM) {
  if (!cpuLockData) return cudaErrorInitializationError;
  if ((int64_t)(semNum + 1) * NUM_SM > cpuLockData->semaphoreCount) return cudaErrorInvalidValue;
  *h = (cudaSemaphore_t)semNum;
  return sem_create(cpuLockData->semaphoreBuffers, semNum, count, NUM_SM, 0);
}
cudaError_t cudaSemaphoreCreateEBO(cudaSemaphore_t* const h, const int semNum, const unsigned int count,
                                   const int NUM_SM) {
  return cudaSemaphoreCreateSpin(h, semNum, count, NUM_SM);
}

unsigned int gsrb_cudalocks_status(void) {
  if (!cpuLockData) return 0;
  cudaDeviceSynchronize();
  uint32_t v = 0;
  void* bufs[] = {cpuLockData->barrierBuffers, cpuLockData->mutexBuffers, cpuLockData->mutexBufferHeads,
                  cpuLockData->mutexBufferTails, cpuLockData->semaphoreBuffers};
  for (void* b : bufs) {
    uint32_t s = read_clear_status(b);
    if (!v) v = s;
  }
  const uint32_t sb = read_clear_barrier_status(cpuLockData->barrierBuffers, cpuLockData->arrayStride);
  if (!v) v = sb;
  return v;
}

}  // extern "C"
