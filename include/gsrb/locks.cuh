// gsrb/locks.cuh -- CTA-granularity mutexes and reader/writer semaphores for
// sm_100a with bounded waits.
//
// Behaviour restated from the Heterosync cudaLocks layer:
//   spin mutex        Heterosync/cudaLocksMutexSpin.cu:13-50
//   backoff mutex     Heterosync/cudaLocksMutexEBO.cu:13-65
//   ticket (FA) mutex Heterosync/cudaLocksMutexFA.cu:13-69
//   ring ("sleep")    Heterosync/cudaLocksMutexSleep.cu:20-108
//   spin semaphore    Heterosync/cudaLocksSemaphoreSpin.cu:31-218
//   backoff semaphore Heterosync/cudaLocksSemaphoreEBO.cu:30-244
//   priority spin sem Heterosync/cudaLocksSemaphoreSpin.cu:411-622
//   priority EBO sem  Heterosync/cudaLocksSemaphoreEBO.cu:456-694
// All are whole-CTA collectives (each begins with __syncthreads and one thread
// operates on the lock), like the reference.  Every wait is bounded by a
// %globaltimer deadline; when it runs out the call records
// GSRB_DEV_LOCK_TIMEOUT in the lock area's status word and returns false
// (the caller must then skip its critical section).
//
// Status word: every lock buffer allocated by this library is preceded by one
// 128-byte header line; word 0 of that line is the status word, so device code
// holding only the reference's raw buffer pointer can find it at ptr - 32 words.
//
// The B200-native priority semaphore (PrioritySem below) keeps the reference
// record (5 words per semaphore, word 3 = capacity + 1 as the reference harness
// reads it, Heterosync/main.cu:973) but changes the protocol: no lock word, the
// count is claimed with one compare-and-swap, releases are a single
// `red.release.gpu` (posts never wait: the reference's "priority to exiting
// blocks" idea, Heterosync/cudaLocksSemaphoreSpin.cu:569-575, taken to its
// limit), queued writers hold new readers back (writer precedence, the
// reference's writerWaiting flag, :489-492) and writers are served in ticket
// order.
#pragma once
#include <stdint.h>
#include "gsrb/ptx.cuh"
#include "gsrb/barrier.cuh"

namespace gsrb {

__device__ __forceinline__ uint32_t* lock_status_word(const void* buf) {
  return (uint32_t*)buf - 32;
}

struct LockWait {
  uint64_t t0;
  uint64_t timeout_ns;
  uint32_t it;
  __device__ __forceinline__ explicit LockWait(uint64_t to) : t0(0), timeout_ns(to), it(0) {}
  // Returns false once the deadline has passed.
  __device__ __forceinline__ bool tick() {
    if ((++it & 15u) != 0u) return true;
    const uint64_t now = ptx::globaltimer_ns();
    if (t0 == 0) { t0 = now; return true; }
    return now - t0 <= timeout_ns;
  }
};

__device__ __forceinline__ void lock_record_timeout(const void* buf) {
  ptx::atom_cas_acq_rel_gpu(lock_status_word(buf), 0u, GSRB_DEV_LOCK_TIMEOUT);
}
__device__ __forceinline__ void lock_record_invariant(const void* buf) {
  ptx::atom_cas_acq_rel_gpu(lock_status_word(buf), 0u, GSRB_DEV_INVARIANT);
}

__device__ __forceinline__ bool cta_bcast(bool v) {
  __shared__ int s_flag;
  __syncthreads();
  if (threadIdx.x == 0) s_flag = v ? 1 : 0;
  __syncthreads();
  return s_flag != 0;
}

constexpr uint32_t kMaxBackoffNs = 1024;  // cap of the exponential backoff (reference MAX_BACKOFF, Heterosync/main.cu:7)

// ---------------------------------------------------------------- mutexes ----
// Test-and-test-and-set spin lock on `head` (0 free / 1 held).
__device__ __forceinline__ bool mutex_spin_lock(uint32_t* head, const void* buf, uint64_t to,
                                                bool backoff) {
  bool ok = true;
  __syncthreads();
  if (threadIdx.x == 0) {
    LockWait w(to);
    uint32_t b = 32;
    for (;;) {
      if (ptx::ld_relaxed_gpu(head) == 0u && ptx::atom_cas_acquire_gpu(head, 0u, 1u) == 0u) break;
      if (!w.tick()) { lock_record_timeout(buf); ok = false; break; }
      if (backoff) { __nanosleep(b); b = (b << 1) < kMaxBackoffNs ? (b << 1) : kMaxBackoffNs; }
    }
  }
  return cta_bcast(ok);
}
__device__ __forceinline__ void mutex_spin_unlock(uint32_t* head) {
  __syncthreads();
  if (threadIdx.x == 0) ptx::st_release_gpu(head, 0u);
  __syncthreads();
}

// Ticket lock: take a ticket from `ticket`, wait until `turn` shows it.
__device__ __forceinline__ bool mutex_fa_lock(uint32_t* ticket, uint32_t* turn, const void* buf,
                                              uint64_t to) {
  bool ok = true;
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t my = ptx::atom_add_relaxed_gpu(ticket, 1u);
    LockWait w(to);
    while (ptx::ld_acquire_gpu(turn) != my) {
      if (!w.tick()) { lock_record_timeout(buf); ok = false; break; }
    }
  }
  return cta_bcast(ok);
}
__device__ __forceinline__ void mutex_fa_unlock(uint32_t* turn) {
  __syncthreads();
  if (threadIdx.x == 0) ptx::red_add_release_gpu(turn, 1u);
  __syncthreads();
}

// Ring-buffer lock: append to the ring (`tail` wraps after ring_max + 1 slots,
// like atomicInc(tail, maxRingBufferSize)); wait until the ring slot holds 1;
// unlock writes -1 to the own slot and 1 to the next.
__device__ __forceinline__ bool mutex_sleep_lock(int32_t* ring, uint32_t* tail, uint32_t ring_max,
                                                 const void* buf, uint64_t to, uint32_t* slot_out) {
  __shared__ uint32_t s_slot;
  bool ok = true;
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t pos = atomicInc(tail, ring_max);
    s_slot = pos;
    LockWait w(to);
    while (ptx::ld_acquire_gpu((const uint32_t*)(ring + pos)) != 1u) {
      if (!w.tick()) { lock_record_timeout(buf); ok = false; break; }
      __nanosleep(64);
    }
  }
  ok = cta_bcast(ok);
  *slot_out = s_slot;
  return ok;
}
__device__ __forceinline__ void mutex_sleep_unlock(int32_t* ring, uint32_t slot, uint32_t ring_max) {
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t next = slot >= ring_max ? 0u : slot + 1u;
    ptx::st_relaxed_gpu((uint32_t*)(ring + slot), 0xffffffffu);
    ptx::st_release_gpu((uint32_t*)(ring + next), 1u);
  }
  __syncthreads();
}

// ------------------------------------------------------------- semaphores ----
// Reference-protocol semaphore (lock word + count + writerWaiting [+ priority]):
// record words [count, lock, writerWaiting, max, priority].  `priority` selects
// the TPDS'22 priority variant (waiters stand back while posts are pending),
// `backoff` the EBO flavour.  The EBO backoff is asymmetric as in the reference
// (Heterosync/cudaLocksSemaphoreEBO.cu:160-181): a failing writer doubles its
// pause up to MAX_BACKOFF - 1 loop iterations, a failing reader adds 5; at about
// 16 ns per iteration that is a 16 us cap for writers and an 80 ns step for
// readers.  (Equal pauses for both let the readers' retries keep the count
// below max for seconds at 296 CTAs.)  A reader first checks writerWaiting and
// the count with plain loads and takes the lock word only when it could enter:
// the attempt it skips would have changed nothing.
constexpr uint32_t kSemWriterBackoffCapNs = 16383;
constexpr uint32_t kSemReaderBackoffStepNs = 80;
struct RefSem {
  uint32_t* rec;
  __device__ __forceinline__ uint32_t* count() const { return rec; }
  __device__ __forceinline__ uint32_t* lockw() const { return rec + 1; }
  __device__ __forceinline__ uint32_t* writer_waiting() const { return rec + 2; }
  __device__ __forceinline__ uint32_t* prio() const { return rec + 4; }
};

__device__ __forceinline__ bool refsem_wait(RefSem s, bool is_writer, uint32_t max_count,
                                            bool priority, bool backoff, const void* buf,
                                            uint64_t to) {
  bool ok = true;
  __syncthreads();
  if (threadIdx.x == 0) {
    LockWait w(to);
    uint32_t b = 32;
    for (;;) {
      if (priority) {
        while (ptx::ld_acquire_gpu(s.prio()) != 0u) {
          if (!w.tick()) { ok = false; break; }
          __nanosleep(b);
          b = (b << 1) < kMaxBackoffNs ? (b << 1) : kMaxBackoffNs;
        }
        if (!ok) break;
      }
      bool entered = false;
      const bool hopeless = !is_writer && (ptx::ld_relaxed_gpu(s.writer_waiting()) != 0u ||
                                           ptx::ld_relaxed_gpu(s.count()) <= 1u);
      if (!hopeless && ptx::atom_cas_acquire_gpu(s.lockw(), 0u, 1u) == 0u) {
        const uint32_t c = ptx::ld_relaxed_gpu(s.count());
        if (is_writer) {
          if (c == max_count) {
            ptx::st_relaxed_gpu(s.count(), c - max_count);
            ptx::st_relaxed_gpu(s.writer_waiting(), 0u);
            entered = true;
          } else {
            ptx::st_relaxed_gpu(s.writer_waiting(), 1u);
          }
        } else if (ptx::ld_relaxed_gpu(s.writer_waiting()) == 0u && c > 1u) {
          ptx::st_relaxed_gpu(s.count(), c - 1u);
          entered = true;
        }
        ptx::st_release_gpu(s.lockw(), 0u);
      }
      if (entered) break;
      if (!w.tick()) { ok = false; break; }
      if (backoff) {
        __nanosleep(b);
        if (is_writer) b = 2u * b + 1u < kSemWriterBackoffCapNs ? 2u * b + 1u : kSemWriterBackoffCapNs;
        else b += kSemReaderBackoffStepNs;
      }
    }
    if (!ok) lock_record_timeout(buf);
  }
  return cta_bcast(ok);
}

__device__ __forceinline__ bool refsem_post(RefSem s, bool is_writer, uint32_t max_count,
                                            bool priority, const void* buf, uint64_t to) {
  bool ok = true;
  __syncthreads();
  if (threadIdx.x == 0) {
    if (priority) ptx::atom_add_relaxed_gpu(s.prio(), 1u);
    LockWait w(to);
    while (ptx::atom_cas_acquire_gpu(s.lockw(), 0u, 1u) != 0u) {
      if (!w.tick()) { ok = false; break; }
    }
    if (ok) {
      const uint32_t c = ptx::ld_relaxed_gpu(s.count());
      ptx::st_relaxed_gpu(s.count(), c + (is_writer ? max_count : 1u));
      ptx::st_release_gpu(s.lockw(), 0u);
    } else {
      lock_record_timeout(buf);
    }
    if (priority) ptx::atom_add_relaxed_gpu(s.prio(), 0xffffffffu);
  }
  return cta_bcast(ok);
}

// B200-native priority semaphore on the reference's 5-word record
// [count, ticket, queued, max, serving]: count starts at max = capacity + 1
// (Heterosync/cudaLocksSemaphoreSpin.cu:14-27 writes count + 1 into words 0 and
// 3, and words 1, 2, 4 as 0, which are valid initial values here too).
//   reader enters : no writer queued and count > 1   -> CAS count, count - 1
//   writer enters : its ticket is being served and count == max -> CAS count, 0
//   reader leaves : red.release count += 1          (never waits)
//   writer leaves : red.release count += max, serving += 1 (never waits)
// Mutual exclusion and the capacity bound rest on the single CAS-ed count
// word; the queue and ticket words only order writers and hold readers back
// while a writer waits (writer precedence).  Every change of the count is an
// atomic read-modify-write, so in correct use it never exceeds max; a waiter
// that reads more than max has seen an over-post (a post without its wait)
// and reports GSRB_DEV_INVARIANT instead of waiting for its deadline.
struct PrioritySem {
  uint32_t* rec;
  __device__ __forceinline__ uint32_t* count() const { return rec; }
  __device__ __forceinline__ uint32_t* ticket() const { return rec + 1; }
  __device__ __forceinline__ uint32_t* queued() const { return rec + 2; }
  __device__ __forceinline__ uint32_t max_count() const { return ptx::ld_relaxed_gpu(rec + 3); }
  __device__ __forceinline__ uint32_t* serving() const { return rec + 4; }
};

__device__ __forceinline__ bool psem_wait(PrioritySem s, bool is_writer, const void* buf,
                                          uint64_t to, uint32_t spin_ns) {
  bool ok = true;
  __syncthreads();
  if (threadIdx.x == 0) {
    LockWait w(to);
    const uint32_t mx = s.max_count();
    uint32_t b = spin_ns ? spin_ns : 32;
    if (!is_writer) {
      for (;;) {
        if (ptx::ld_relaxed_gpu(s.queued()) == 0u) {
          const uint32_t c = ptx::ld_relaxed_gpu(s.count());
          if (c > mx) { lock_record_invariant(buf); ok = false; break; }  // over-post
          if (c > 1u && ptx::atom_cas_acquire_gpu(s.count(), c, c - 1u) == c) break;
        }
        if (!w.tick()) { ok = false; break; }
        __nanosleep(b);
        b = (b << 1) < kMaxBackoffNs ? (b << 1) : kMaxBackoffNs;
      }
    } else {
      const uint32_t my = ptx::atom_add_relaxed_gpu(s.ticket(), 1u);
      ptx::red_add_relaxed_gpu(s.queued(), 1u);  // hold new readers back
      while (ptx::ld_acquire_gpu(s.serving()) != my) {
        if (!w.tick()) { ok = false; break; }
        __nanosleep(spin_ns ? spin_ns : 64);
      }
      if (ok) {
        for (;;) {
          const uint32_t c = ptx::ld_relaxed_gpu(s.count());
          if (c > mx) { lock_record_invariant(buf); ok = false; break; }  // over-post
          if (c == mx && ptx::atom_cas_acquire_gpu(s.count(), mx, 0u) == mx) break;
          if (!w.tick()) { ok = false; break; }
          if (spin_ns) __nanosleep(spin_ns);
        }
        // a writer that was served but gave up on the count hands its turn
        // on, so the writers queued behind it are not held up by it
        if (!ok) ptx::red_add_release_gpu(s.serving(), 1u);
      }
      ptx::red_add_relaxed_gpu(s.queued(), 0xffffffffu);
    }
    if (!ok) lock_record_timeout(buf);  // no-op after an invariant report (first code wins)
  }
  return cta_bcast(ok);
}

__device__ __forceinline__ void psem_post(PrioritySem s, bool is_writer) {
  __syncthreads();
  if (threadIdx.x == 0) {
    if (is_writer) {
      ptx::red_add_release_gpu(s.count(), s.max_count());
      ptx::red_add_release_gpu(s.serving(), 1u);
    } else {
      ptx::red_add_release_gpu(s.count(), 1u);
    }
  }
  __syncthreads();
}

}  // namespace gsrb
