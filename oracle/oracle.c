/* oracle.c -- CPU restatement of the reference algorithms (test infrastructure
 * only; see oracle.h).  Plain C11, pthreads for the multi-threaded baselines. */
#define _GNU_SOURCE
#include "oracle.h"

#include <limits.h>
#include <math.h>
#include <pthread.h>
#include <sched.h>
#include <stdatomic.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

void orc_free(void* p) { free(p); }

static double now_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------------ reduce */
int64_t orc_sum_i32(const int32_t* in, size_t n) {
  int64_t s = 0;
  for (size_t i = 0; i < n; ++i) s += in[i];
  return s;
}

typedef struct {
  const int32_t* in;
  const uint32_t* uin;
  uint32_t* uout;
  size_t beg, end;
  int64_t sum;
  uint32_t usum;
  uint32_t carry;
} part_t;

static void* sum_worker(void* p) {
  part_t* t = (part_t*)p;
  t->sum = orc_sum_i32(t->in + t->beg, t->end - t->beg);
  return NULL;
}

int64_t orc_sum_i32_mt(const int32_t* in, size_t n, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t th[256];
  part_t pt[256];
  for (int t = 0; t < threads; ++t) {
    pt[t].in = in;
    pt[t].beg = n * (size_t)t / (size_t)threads;
    pt[t].end = n * (size_t)(t + 1) / (size_t)threads;
    pthread_create(&th[t], NULL, sum_worker, &pt[t]);
  }
  int64_t s = 0;
  for (int t = 0; t < threads; ++t) {
    pthread_join(th[t], NULL);
    s += pt[t].sum;
  }
  return s;
}

/* -------------------------------------------------------------------- scan */
void orc_scan_u32(const uint32_t* in, uint32_t* out, size_t n) {
  uint32_t run = 0; /* scan/main.cu:15-20: out[i] = running sum before in[i] */
  for (size_t i = 0; i < n; ++i) {
    out[i] = run;
    run = run + in[i];
  }
}

static void* scan_reduce_worker(void* p) {
  part_t* t = (part_t*)p;
  uint32_t s = 0;
  for (size_t i = t->beg; i < t->end; ++i) s += t->uin[i];
  t->usum = s;
  return NULL;
}
static void* scan_apply_worker(void* p) {
  part_t* t = (part_t*)p;
  uint32_t run = t->carry;
  for (size_t i = t->beg; i < t->end; ++i) {
    t->uout[i] = run;
    run += t->uin[i];
  }
  return NULL;
}

void orc_scan_u32_mt(const uint32_t* in, uint32_t* out, size_t n, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  pthread_t th[256];
  part_t pt[256];
  for (int t = 0; t < threads; ++t) {
    pt[t].uin = in;
    pt[t].uout = out;
    pt[t].beg = n * (size_t)t / (size_t)threads;
    pt[t].end = n * (size_t)(t + 1) / (size_t)threads;
    pthread_create(&th[t], NULL, scan_reduce_worker, &pt[t]);
  }
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  uint32_t carry = 0;
  for (int t = 0; t < threads; ++t) {
    pt[t].carry = carry;
    carry += pt[t].usum;
    pthread_create(&th[t], NULL, scan_apply_worker, &pt[t]);
  }
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
}

void orc_scan_f32_f64(const float* in, double* out, size_t n) {
  double run = 0.0;
  for (size_t i = 0; i < n; ++i) {
    out[i] = run;
    run += (double)in[i];
  }
}

double orc_max_rel_err_f32_f64(const float* gpu, const double* ref, size_t n, double floor_) {
  double worst = 0.0;
  for (size_t i = 0; i < n; ++i) {
    double d = fabs((double)gpu[i] - ref[i]);
    double den = fabs(ref[i]) > floor_ ? fabs(ref[i]) : floor_;
    double r = d / den;
    if (r > worst || r != r) worst = r;
  }
  return worst;
}

/* ------------------------------------------------------------------ graphs */
void orc_bfs(uint32_t n, const uint32_t* row, const uint32_t* dst, uint32_t src, int32_t* level) {
  for (uint32_t v = 0; v < n; ++v) level[v] = INT32_MAX;
  if (src >= n) return;
  uint32_t* q = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  size_t head = 0, tail = 0;
  level[src] = 0;
  q[tail++] = src;
  while (head < tail) {
    uint32_t u = q[head++];
    for (uint32_t j = row[u]; j < row[u + 1]; ++j) {
      uint32_t v = dst[j];
      if (level[v] == INT32_MAX) {
        level[v] = level[u] + 1;
        q[tail++] = v;
      }
    }
  }
  free(q);
}

typedef struct {
  int64_t d;
  uint32_t v;
} heap_item;

static void heap_push(heap_item* h, size_t* sz, heap_item it) {
  size_t i = (*sz)++;
  h[i] = it;
  while (i > 0) {
    size_t p = (i - 1) / 2;
    if (h[p].d <= h[i].d) break;
    heap_item t = h[p];
    h[p] = h[i];
    h[i] = t;
    i = p;
  }
}
static heap_item heap_pop(heap_item* h, size_t* sz) {
  heap_item top = h[0];
  h[0] = h[--(*sz)];
  size_t i = 0;
  for (;;) {
    size_t l = 2 * i + 1, r = l + 1, m = i;
    if (l < *sz && h[l].d < h[m].d) m = l;
    if (r < *sz && h[r].d < h[m].d) m = r;
    if (m == i) break;
    heap_item t = h[m];
    h[m] = h[i];
    h[i] = t;
    i = m;
  }
  return top;
}

void orc_dijkstra(uint32_t n, const uint32_t* row, const uint32_t* dst, const int32_t* w, uint32_t src,
                  int32_t* dist) {
  for (uint32_t v = 0; v < n; ++v) dist[v] = INT32_MAX;
  if (src >= n) return;
  size_t cap = (size_t)row[n] + 1, sz = 0;
  heap_item* h = (heap_item*)malloc(sizeof(heap_item) * cap);
  dist[src] = 0;
  heap_item s0 = {0, src};
  heap_push(h, &sz, s0);
  while (sz) {
    heap_item it = heap_pop(h, &sz);
    if (it.d != dist[it.v]) continue;
    uint32_t u = it.v;
    for (uint32_t j = row[u]; j < row[u + 1]; ++j) {
      int64_t nd = it.d + (int64_t)w[j];
      uint32_t v = dst[j];
      if (nd < dist[v]) {
        dist[v] = (int32_t)nd;
        heap_item ni = {nd, v};
        heap_push(h, &sz, ni);
      }
    }
  }
  free(h);
}

void orc_pagerank_pull(uint32_t n, const uint32_t* row, const uint32_t* dst, double alpha, int iters,
                       double* x) {
  double* c = (double*)malloc(sizeof(double) * (n ? n : 1));
  for (uint32_t v = 0; v < n; ++v) x[v] = 1.0 - alpha;
  for (int it = 0; it < iters; ++it) {
    for (uint32_t u = 0; u < n; ++u) {
      uint32_t d = row[u + 1] - row[u];
      c[u] = d ? x[u] / (double)d : 0.0;
    }
    for (uint32_t v = 0; v < n; ++v) {
      double s = 0.0;
      for (uint32_t j = row[v]; j < row[v + 1]; ++j) s += c[dst[j]];
      x[v] = (1.0 - alpha) + alpha * s;
    }
  }
  free(c);
}

/* The same fixed point for any graph, directed included, in scatter form:
 * x <- (1 - alpha) + alpha * sum_{u -> v} x_u / outdeg(u), where u -> v are the
 * CSR rows' out-edges.  This is the fixed point the reference's push-residual
 * PageRank converges to (LONESTAR/apps/pr/kernel_gsrb.cu:298-336 seeds
 * p = 1 - alpha and pushes alpha * residual / outdeg along out-edges); on a
 * symmetric graph it equals orc_pagerank_pull. */
void orc_pagerank_push(uint32_t n, const uint32_t* row, const uint32_t* dst, double alpha, int iters,
                       double* x) {
  double* y = (double*)malloc(sizeof(double) * (n ? n : 1));
  for (uint32_t v = 0; v < n; ++v) x[v] = 1.0 - alpha;
  for (int it = 0; it < iters; ++it) {
    for (uint32_t v = 0; v < n; ++v) y[v] = 1.0 - alpha;
    for (uint32_t u = 0; u < n; ++u) {
      uint32_t d = row[u + 1] - row[u];
      if (!d) continue;
      double c = alpha * x[u] / (double)d;
      for (uint32_t j = row[u]; j < row[u + 1]; ++j) y[dst[j]] += c;
    }
    memcpy(x, y, sizeof(double) * n);
  }
  free(y);
}

/* Multi-threaded forms for the CPU baseline (same results as orc_bfs and
 * orc_pagerank_pull).  BFS: level-synchronous top-down; every thread takes
 * chunks of the frontier from a shared counter, claims unvisited vertices
 * with a compare-and-swap on their level and appends them to the next
 * frontier through per-thread buffers.  Levels are unique, so the result does
 * not depend on the interleaving. */
typedef struct {
  uint32_t n;
  const uint32_t* row;
  const uint32_t* dst;
  int32_t* level;
  uint32_t* cur;
  uint32_t* next;
  size_t cur_n;
  size_t next_n; /* atomic */
  size_t take;   /* atomic chunk cursor over cur */
  int32_t depth;
  int done;
  pthread_barrier_t bar;
} bfsmt_t;

#define BFS_MT_CHUNK 256
#define BFS_MT_BUF 512

static void* bfs_mt_worker(void* p) {
  bfsmt_t* b = (bfsmt_t*)p;
  uint32_t buf[BFS_MT_BUF];
  for (;;) {
    size_t nb = 0;
    int32_t nl = b->depth + 1;
    for (;;) {
      size_t beg = __atomic_fetch_add(&b->take, BFS_MT_CHUNK, __ATOMIC_RELAXED);
      if (beg >= b->cur_n) break;
      size_t end = beg + BFS_MT_CHUNK < b->cur_n ? beg + BFS_MT_CHUNK : b->cur_n;
      for (size_t i = beg; i < end; ++i) {
        uint32_t u = b->cur[i];
        for (uint32_t j = b->row[u]; j < b->row[u + 1]; ++j) {
          uint32_t v = b->dst[j];
          int32_t inf = INT32_MAX;
          if (__atomic_load_n(&b->level[v], __ATOMIC_RELAXED) != INT32_MAX) continue;
          if (!__atomic_compare_exchange_n(&b->level[v], &inf, nl, 0, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) continue;
          buf[nb++] = v;
          if (nb == BFS_MT_BUF) {
            size_t at = __atomic_fetch_add(&b->next_n, nb, __ATOMIC_RELAXED);
            memcpy(b->next + at, buf, nb * sizeof(uint32_t));
            nb = 0;
          }
        }
      }
    }
    if (nb) {
      size_t at = __atomic_fetch_add(&b->next_n, nb, __ATOMIC_RELAXED);
      memcpy(b->next + at, buf, nb * sizeof(uint32_t));
    }
    if (pthread_barrier_wait(&b->bar) == PTHREAD_BARRIER_SERIAL_THREAD) {
      uint32_t* t = b->cur;
      b->cur = b->next;
      b->next = t;
      b->cur_n = b->next_n;
      b->next_n = 0;
      b->take = 0;
      b->depth += 1;
      b->done = b->cur_n == 0;
    }
    pthread_barrier_wait(&b->bar);
    if (b->done) return NULL;
  }
}

void orc_bfs_mt(uint32_t n, const uint32_t* row, const uint32_t* dst, uint32_t src, int32_t* level, int threads) {
  for (uint32_t v = 0; v < n; ++v) level[v] = INT32_MAX;
  if (src >= n) return;
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  bfsmt_t b;
  memset(&b, 0, sizeof(b));
  b.n = n;
  b.row = row;
  b.dst = dst;
  b.level = level;
  b.cur = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  b.next = (uint32_t*)malloc(sizeof(uint32_t) * (n ? n : 1));
  level[src] = 0;
  b.cur[0] = src;
  b.cur_n = 1;
  pthread_barrier_init(&b.bar, NULL, (unsigned)threads);
  pthread_t th[256];
  for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, bfs_mt_worker, &b);
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  pthread_barrier_destroy(&b.bar);
  free(b.cur);
  free(b.next);
}

typedef struct {
  uint32_t n;
  const uint32_t* row;
  const uint32_t* dst;
  double alpha;
  int iters;
  double* x;
  double* c;
  size_t take; /* atomic chunk cursor */
  pthread_barrier_t bar;
} prmt_t;

#define PR_MT_CHUNK 2048

static void* pr_mt_worker(void* p) {
  prmt_t* b = (prmt_t*)p;
  for (int it = 0; it < b->iters; ++it) {
    for (;;) {
      size_t beg = __atomic_fetch_add(&b->take, PR_MT_CHUNK, __ATOMIC_RELAXED);
      if (beg >= b->n) break;
      size_t end = beg + PR_MT_CHUNK < b->n ? beg + PR_MT_CHUNK : b->n;
      for (size_t u = beg; u < end; ++u) {
        uint32_t d = b->row[u + 1] - b->row[u];
        b->c[u] = d ? b->x[u] / (double)d : 0.0;
      }
    }
    if (pthread_barrier_wait(&b->bar) == PTHREAD_BARRIER_SERIAL_THREAD) b->take = 0;
    pthread_barrier_wait(&b->bar);
    for (;;) {
      size_t beg = __atomic_fetch_add(&b->take, PR_MT_CHUNK, __ATOMIC_RELAXED);
      if (beg >= b->n) break;
      size_t end = beg + PR_MT_CHUNK < b->n ? beg + PR_MT_CHUNK : b->n;
      for (size_t v = beg; v < end; ++v) {
        double s = 0.0;
        for (uint32_t j = b->row[v]; j < b->row[v + 1]; ++j) s += b->c[b->dst[j]];
        b->x[v] = (1.0 - b->alpha) + b->alpha * s;
      }
    }
    if (pthread_barrier_wait(&b->bar) == PTHREAD_BARRIER_SERIAL_THREAD) b->take = 0;
    pthread_barrier_wait(&b->bar);
  }
  return NULL;
}

void orc_pagerank_pull_mt(uint32_t n, const uint32_t* row, const uint32_t* dst, double alpha, int iters,
                          double* x, int threads) {
  if (threads < 1) threads = 1;
  if (threads > 256) threads = 256;
  prmt_t b;
  memset(&b, 0, sizeof(b));
  b.n = n;
  b.row = row;
  b.dst = dst;
  b.alpha = alpha;
  b.iters = iters;
  b.x = x;
  b.c = (double*)malloc(sizeof(double) * (n ? n : 1));
  for (uint32_t v = 0; v < n; ++v) x[v] = 1.0 - alpha;
  pthread_barrier_init(&b.bar, NULL, (unsigned)threads);
  pthread_t th[256];
  for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, pr_mt_worker, &b);
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  pthread_barrier_destroy(&b.bar);
  free(b.c);
}

double orc_normalized_l1(const float* a, const double* b, uint32_t n) {
  double sa = 0.0, sb = 0.0;
  for (uint32_t v = 0; v < n; ++v) {
    sa += (double)a[v];
    sb += b[v];
  }
  double l1 = 0.0;
  for (uint32_t v = 0; v < n; ++v) l1 += fabs((double)a[v] / sa - b[v] / sb);
  return l1;
}

uint64_t orc_traversed_edges(uint32_t n, const uint32_t* row, const int32_t* value) {
  uint64_t m = 0;
  for (uint32_t v = 0; v < n; ++v)
    if (value[v] != INT32_MAX) m += row[v + 1] - row[v];
  return m;
}

int orc_gr_read(const char* path, uint32_t* n_out, uint64_t* m_out, uint32_t** row_out, uint32_t** dst_out,
                int32_t** w_out) {
  FILE* f = fopen(path, "rb");
  if (!f) return -1;
  uint64_t hdr[4];
  if (fread(hdr, 8, 4, f) != 4 || hdr[0] != 1) {
    fclose(f);
    return -2;
  }
  uint64_t n = hdr[2], m = hdr[3];
  uint64_t* outIdx = (uint64_t*)malloc(8 * (n ? n : 1));
  uint32_t* dst = (uint32_t*)malloc(4 * (m ? m : 1));
  int32_t* w = (int32_t*)calloc(m ? m : 1, 4);
  uint32_t* row = (uint32_t*)malloc(4 * (n + 1));
  int rc = 0;
  if (fread(outIdx, 8, n, f) != n) rc = -3;
  if (!rc && fread(dst, 4, m, f) != m) rc = -4;
  if (!rc && (m & 1)) {
    uint32_t pad;
    if (fread(&pad, 4, 1, f) != 1) rc = -5;
  }
  if (!rc && hdr[1] == 4 && fread(w, 4, m, f) != m) rc = -6;
  fclose(f);
  row[0] = 0;
  for (uint64_t v = 0; !rc && v < n; ++v) row[v + 1] = (uint32_t)outIdx[v];
  free(outIdx);
  if (rc) {
    free(dst);
    free(w);
    free(row);
    return rc;
  }
  *n_out = (uint32_t)n;
  *m_out = m;
  *row_out = row;
  *dst_out = dst;
  *w_out = w;
  return 0;
}

/* -------------------------------------------------- Heterosync golden replay */
enum { WORDS_PER_LINE = 16, THREADS_PER_HALFWARP = 16 };

static void access_golden(float* s, int loc, int nlocs, int numLdSt) {
  /* Heterosync/main.cu:41-59: every location except the first cache line of a
   * half-warp's region copies the same word of the previous line. */
  if (loc % (THREADS_PER_HALFWARP * (numLdSt + 1)) >= WORDS_PER_LINE) {
    if (loc - WORDS_PER_LINE >= 0 && loc < nlocs) s[loc] = s[loc - WORDS_PER_LINE];
  }
}

int orc_heterosync_storage_locs(int p, int numLdSt, int numTBs, int numSM, int tpb) {
  int perSM = (numTBs + numSM - 1) / numSM; /* ceil((float)numTBs / NUM_SM), :2474 */
  int mult = 0;
  if ((p < 4 || p >= 37) || (p >= 24 && p <= 35)) mult = numTBs;
  else if (p >= 4 && p <= 7) mult = 1;
  else if (p >= 8 && p <= 19) mult = perSM;
  else if ((p >= 20 && p <= 23) || p == 36) mult = numTBs < numSM ? numTBs : numSM;
  return mult * tpb * (numLdSt + 1);
}

void orc_heterosync_golden(int p, int numLdSt, int numTBs, int numIters, int numRepeats, int numSM, int tpb,
                           float* s, int nlocs) {
  const int uniq = tpb * (numLdSt + 1); /* numUniqLocsAccPerTB, :2580 */
  const int perSM = (numTBs + numSM - 1) / numSM;
  for (int rep = 0; rep < numRepeats; ++rep) {
    for (int j = 0; j < numIters; ++j) {
      if (p < 4 || p >= 37) {
        const int acc = numTBs * uniq;
        for (int i = acc - 1; i >= 0; --i) access_golden(s, (i + j * uniq) % acc, nlocs, numLdSt);
        const int localExch = p == 1 || p == 3 || p == 38 || p == 40 || p == 42 || p == 44 || p == 46;
        if (localExch && perSM > 1) {
          for (int i = acc - 1; i >= 0; --i) {
            int loc = (i + perSM * uniq) % acc;
            loc = (loc + j * uniq) % acc;
            access_golden(s, loc, nlocs, numLdSt);
          }
        }
      } else if (p >= 4 && p <= 7) {
        for (int b = 0; b < numTBs; ++b)
          for (int i = uniq - 1; i >= 0; --i) access_golden(s, i, nlocs, numLdSt);
      } else if ((p >= 8 && p <= 19) || (p >= 32 && p <= 35)) {
        const int nsm = numTBs < numSM ? numTBs : numSM;
        for (int tb = 0; tb < numTBs; ++tb) {
          const int smID = tb % nsm, per = tb / nsm;
          if (per == smID % perSM)
            for (int k = 0; k < perSM; ++k)
              for (int i = uniq - 1; i >= 0; --i) access_golden(s, (i + k * uniq) % nlocs, nlocs, numLdSt);
        }
      } else if (p >= 20 && p <= 23) {
        const int acc = numTBs * uniq;
        for (int i = acc - 1; i >= 0; --i) access_golden(s, i % (numSM * uniq), nlocs, numLdSt);
      } else {
        const int acc = numTBs * uniq;
        for (int i = acc - 1; i >= 0; --i) access_golden(s, i, nlocs, numLdSt);
      }
    }
  }
}

/* ------------------------------------------- host-thread barrier model (CPU) */
typedef struct {
  _Alignas(64) atomic_uint count;
  char pad[60];
} grp_t;

typedef struct {
  _Alignas(64) atomic_uint count;
  char pad0[60];
  _Alignas(64) atomic_uint epoch;
  char pad1[60];
  grp_t* groups;
  int ngroups;
  int nthreads;
  int nparts;  /* participants (>= nthreads): thread t arrives for t, t + nthreads, ... */
  int episodes;
  atomic_uint* stamps; /* one per thread, each on its own line (stride 16) */
  atomic_ullong stale;
  int stall_permille;  /* injected stalls: chance per stall point, in 1/1000 */
  atomic_ullong stalls;
  int kill_id;         /* participant that leaves for good before kill_episode (-1: none) */
  int kill_episode;
  double deadline_s;   /* bound on each wait (0: none) */
  atomic_int abort;    /* set by the first wait that ran out; every waiter then gives up */
  atomic_ullong timeouts;
} srb_t;

typedef struct {
  srb_t* b;
  int id;
  uint64_t rng;
} srb_arg;

/* Injected stall: with probability permille/1000 the thread yields or sleeps
 * 5-100 us (xorshift64 per thread, seeded), so that arrivals, the completer's
 * reset-then-publish and the critical sections are reordered across threads. */
static int maybe_stall(uint64_t* rng, int permille) {
  if (permille <= 0) return 0;
  uint64_t x = *rng;
  x ^= x << 13;
  x ^= x >> 7;
  x ^= x << 17;
  *rng = x;
  if ((int)(x % 1000u) >= permille) return 0;
  if ((x >> 20) & 1u) {
    sched_yield();
  } else {
    struct timespec ts = {0, (long)(5000 + (x >> 32) % 95000)};
    nanosleep(&ts, NULL);
  }
  return 1;
}

static unsigned gsize(unsigned n, unsigned g, unsigned i) { return n / g + (i < n % g ? 1u : 0u); }

/* One arrival of participant `vid` (of b->nparts) in episode e; returns 1 if
 * it completed the episode and published it. */
static int srb_arrive(srb_t* b, unsigned vid, unsigned e, uint64_t* rng, unsigned long long* st) {
  unsigned n = (unsigned)b->nparts;
  if (b->ngroups > 1 && n > (unsigned)b->ngroups) {
    unsigned g = vid % (unsigned)b->ngroups;
    unsigned gs = gsize(n, (unsigned)b->ngroups, g);
    if (atomic_fetch_add_explicit(&b->groups[g].count, 1, memory_order_acq_rel) != gs - 1) return 0;
    atomic_store_explicit(&b->groups[g].count, 0, memory_order_relaxed);
    *st += maybe_stall(rng, b->stall_permille); /* group completer slow to go on */
    n = (unsigned)b->ngroups;
  }
  if (atomic_fetch_add_explicit(&b->count, 1, memory_order_acq_rel) != n - 1) return 0;
  atomic_store_explicit(&b->count, 0, memory_order_relaxed);
  *st += maybe_stall(rng, b->stall_permille); /* between the reset and the publish */
  atomic_store_explicit(&b->epoch, e + 1, memory_order_release);
  return 1;
}

/* A host thread arrives for each participant it stands for (vid = id,
 * id + nthreads, ...), then waits for the episode to be published. */
static int srb_sync(srb_t* b, int id, unsigned* epoch, uint64_t* rng) {
  const unsigned e = *epoch;
  int done = 0;
  unsigned long long st = 0;
  st += maybe_stall(rng, b->stall_permille); /* late arrival */
  for (unsigned v = (unsigned)id; v < (unsigned)b->nparts; v += (unsigned)b->nthreads)
    done |= srb_arrive(b, v, e, rng, &st);
  if (st) atomic_fetch_add(&b->stalls, st);
  if (!done) {
    unsigned spins = 0;
    const double t0 = b->deadline_s > 0 ? now_s() : 0.0;
    while (atomic_load_explicit(&b->epoch, memory_order_acquire) == e) {
      if (++spins > 4096) {
        sched_yield();
        spins = 0;
        if (atomic_load_explicit(&b->abort, memory_order_relaxed)) return 0;
        if (b->deadline_s > 0 && now_s() - t0 > b->deadline_s) {
          atomic_store(&b->abort, 1);
          atomic_fetch_add(&b->timeouts, 1);
          return 0;
        }
      }
    }
  }
  *epoch = e + 1;
  return 1;
}

static void* srb_worker(void* p) {
  srb_arg* a = (srb_arg*)p;
  srb_t* b = a->b;
  unsigned epoch = atomic_load_explicit(&b->epoch, memory_order_acquire);
  unsigned long long bad = 0;
  for (int e = 0; e < b->episodes; ++e) {
    if (a->id == b->kill_id && e == b->kill_episode) break; /* leaves, never arrives again */
    unsigned stamp = 0x9e3779b9u * (unsigned)(e + 1);
    atomic_store_explicit(&b->stamps[a->id * 16], stamp, memory_order_relaxed);
    if (!srb_sync(b, a->id, &epoch, &a->rng)) break;
    int peer = (a->id + 1 + e) % b->nthreads;
    if (atomic_load_explicit(&b->stamps[peer * 16], memory_order_relaxed) != stamp) ++bad;
    if (!srb_sync(b, a->id, &epoch, &a->rng)) break;
  }
  atomic_fetch_add(&b->stale, bad);
  return NULL;
}

static double srb_run(int nthreads, int nparts, int ngroups, int episodes, int stall_permille, uint64_t seed,
                      int kill_id, int kill_episode, int deadline_ms, uint64_t* stale, uint64_t* stalls,
                      uint64_t* timeouts);

double orc_cpu_srb_barrier(int nthreads, int ngroups, int episodes, uint64_t* stale) {
  return srb_run(nthreads, 0, ngroups, episodes, 0, 0, -1, 0, 0, stale, NULL, NULL);
}

double orc_cpu_srb_barrier_vcta(int nthreads, int nctas, int ngroups, int episodes, uint64_t* stale) {
  return srb_run(nthreads, nctas, ngroups, episodes, 0, 0, -1, 0, 0, stale, NULL, NULL);
}

double orc_cpu_srb_barrier_stalls(int nthreads, int ngroups, int episodes, int stall_permille, uint64_t seed,
                                  uint64_t* stale, uint64_t* stalls) {
  return srb_run(nthreads, 0, ngroups, episodes, stall_permille, seed, -1, 0, 0, stale, stalls, NULL);
}

double orc_cpu_srb_barrier_kill(int nthreads, int ngroups, int episodes, int kill_id, int kill_episode,
                                int deadline_ms, uint64_t* stale, uint64_t* timeouts) {
  return srb_run(nthreads, 0, ngroups, episodes, 0, 0, kill_id, kill_episode, deadline_ms > 0 ? deadline_ms : 1,
                 stale, NULL, timeouts);
}

static double srb_run(int nthreads, int nparts, int ngroups, int episodes, int stall_permille, uint64_t seed,
                      int kill_id, int kill_episode, int deadline_ms, uint64_t* stale, uint64_t* stalls,
                      uint64_t* timeouts) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 1024) nthreads = 1024;
  srb_t* b = (srb_t*)aligned_alloc(64, sizeof(srb_t));
  memset(b, 0, sizeof(*b));
  b->ngroups = ngroups;
  b->nthreads = nthreads;
  b->nparts = nparts > nthreads ? nparts : nthreads;
  b->episodes = episodes;
  b->stall_permille = stall_permille;
  b->kill_id = kill_id;
  b->kill_episode = kill_episode;
  b->deadline_s = deadline_ms * 1e-3;
  b->groups = (grp_t*)aligned_alloc(64, sizeof(grp_t) * (size_t)(ngroups > 0 ? ngroups : 1));
  memset(b->groups, 0, sizeof(grp_t) * (size_t)(ngroups > 0 ? ngroups : 1));
  b->stamps = (atomic_uint*)aligned_alloc(64, sizeof(atomic_uint) * 16 * (size_t)nthreads);
  memset(b->stamps, 0, sizeof(atomic_uint) * 16 * (size_t)nthreads);
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
  srb_arg* args = (srb_arg*)malloc(sizeof(srb_arg) * (size_t)nthreads);
  double t0 = now_s();
  for (int t = 0; t < nthreads; ++t) {
    args[t].b = b;
    args[t].id = t;
    args[t].rng = (seed + 1u) * 0x9e3779b97f4a7c15ull ^ (uint64_t)(t + 1) * 0xbf58476d1ce4e5b9ull;
    if (!args[t].rng) args[t].rng = 1;
    pthread_create(&th[t], NULL, srb_worker, &args[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  double t1 = now_s();
  if (stale) *stale = atomic_load(&b->stale);
  if (stalls) *stalls = atomic_load(&b->stalls);
  if (timeouts) *timeouts = atomic_load(&b->timeouts);
  free(th);
  free(args);
  free(b->stamps);
  free(b->groups);
  free(b);
  /* two barrier episodes per loop iteration */
  return episodes > 0 ? (t1 - t0) * 1e9 / (2.0 * episodes) : 0.0;
}

/* --------------------------------------- host-thread semaphore model (CPU) */
typedef struct {
  _Alignas(64) atomic_uint state; /* bits 0-15 readers, bit 16 writer in, 17+ writers queued */
  char p0[60];
  _Alignas(64) atomic_uint ticket;
  char p1[60];
  _Alignas(64) atomic_uint serving;
  char p2[60];
  _Alignas(64) volatile uint64_t W;
  char p3[56];
  _Alignas(64) atomic_ullong R;
  char p4[56];
  _Alignas(64) atomic_uint inside;
  atomic_uint max_readers;
  atomic_uint violations;
  int capacity, writer_every, iters, incs;
  int stall_permille;
  atomic_ullong stalls;
} sem_t_;

typedef struct {
  sem_t_* s;
  int id;
  uint64_t rng;
} sem_arg;

static void* sem_worker(void* p) {
  sem_arg* a = (sem_arg*)p;
  sem_t_* s = a->s;
  const int writer = (a->id % s->writer_every) == 0;
  unsigned long long st = 0;
  for (int it = 0; it < s->iters; ++it) {
    st += maybe_stall(&a->rng, s->stall_permille); /* before the acquire */
    if (writer) {
      unsigned my = atomic_fetch_add(&s->ticket, 1);
      atomic_fetch_add(&s->state, 1u << 17);
      while (atomic_load_explicit(&s->serving, memory_order_acquire) != my) sched_yield();
      for (;;) {
        unsigned v = atomic_load_explicit(&s->state, memory_order_relaxed);
        if ((v & 0x1ffffu) == 0 &&
            atomic_compare_exchange_weak_explicit(&s->state, &v, v - (1u << 17) + (1u << 16),
                                                  memory_order_acquire, memory_order_relaxed))
          break;
        sched_yield();
      }
      if (atomic_fetch_add(&s->inside, 1000) != 0) atomic_fetch_add(&s->violations, 1);
      for (int k = 0; k < s->incs; ++k) {
        s->W = s->W + 1;
        if (k == 0) st += maybe_stall(&a->rng, s->stall_permille); /* holding it */
      }
      atomic_fetch_sub(&s->inside, 1000);
      atomic_fetch_sub_explicit(&s->state, 1u << 16, memory_order_release);
      atomic_fetch_add_explicit(&s->serving, 1, memory_order_release);
    } else {
      for (;;) {
        unsigned v = atomic_load_explicit(&s->state, memory_order_relaxed);
        if ((v >> 16) == 0 && (v & 0xffffu) < (unsigned)s->capacity &&
            atomic_compare_exchange_weak_explicit(&s->state, &v, v + 1, memory_order_acquire,
                                                  memory_order_relaxed))
          break;
        sched_yield();
      }
      unsigned in = atomic_fetch_add(&s->inside, 1) + 1;
      if (in >= 1000 || in > (unsigned)s->capacity) atomic_fetch_add(&s->violations, 1);
      unsigned mr = atomic_load(&s->max_readers);
      while (in > mr && !atomic_compare_exchange_weak(&s->max_readers, &mr, in)) {
      }
      for (int k = 0; k < s->incs; ++k) {
        atomic_fetch_add_explicit(&s->R, 1, memory_order_relaxed);
        if (k == 0) st += maybe_stall(&a->rng, s->stall_permille); /* holding it */
      }
      atomic_fetch_sub(&s->inside, 1);
      atomic_fetch_sub_explicit(&s->state, 1, memory_order_release);
    }
  }
  if (st) atomic_fetch_add(&s->stalls, st);
  return NULL;
}

double orc_cpu_semaphore(int nthreads, int capacity, int writer_every, int iters, int incs, uint64_t* W,
                         uint64_t* R, uint32_t* max_readers, uint32_t* violations) {
  return orc_cpu_semaphore_stalls(nthreads, capacity, writer_every, iters, incs, 0, 0, W, R, max_readers,
                                  violations, NULL);
}

double orc_cpu_semaphore_stalls(int nthreads, int capacity, int writer_every, int iters, int incs,
                                int stall_permille, uint64_t seed, uint64_t* W, uint64_t* R,
                                uint32_t* max_readers, uint32_t* violations, uint64_t* stalls) {
  if (nthreads < 1) nthreads = 1;
  if (writer_every < 1) writer_every = 1;
  sem_t_* s = (sem_t_*)aligned_alloc(64, sizeof(sem_t_));
  memset((void*)s, 0, sizeof(*s));
  s->capacity = capacity;
  s->writer_every = writer_every;
  s->iters = iters;
  s->incs = incs;
  s->stall_permille = stall_permille;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)nthreads);
  sem_arg* args = (sem_arg*)malloc(sizeof(sem_arg) * (size_t)nthreads);
  double t0 = now_s();
  for (int t = 0; t < nthreads; ++t) {
    args[t].s = s;
    args[t].id = t;
    args[t].rng = (seed + 7u) * 0x9e3779b97f4a7c15ull ^ (uint64_t)(t + 1) * 0x94d049bb133111ebull;
    if (!args[t].rng) args[t].rng = 1;
    pthread_create(&th[t], NULL, sem_worker, &args[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  double t1 = now_s();
  if (W) *W = s->W;
  if (R) *R = atomic_load(&s->R);
  if (max_readers) *max_readers = atomic_load(&s->max_readers);
  if (violations) *violations = atomic_load(&s->violations);
  if (stalls) *stalls = atomic_load(&s->stalls);
  free(th);
  free(args);
  free(s);
  return (double)nthreads * iters / (t1 - t0);
}

/* ---------------------------------------------- policy MLP (FP64 checker) */
enum { MF = 12, MH = 32, MO = 4 };
typedef struct {
  const float *w1, *b1, *w2, *b2, *w3, *b3;
} mlp_view;

static mlp_view mlp_split(const float* p) {
  mlp_view v;
  v.w1 = p;
  v.b1 = v.w1 + MH * MF;
  v.w2 = v.b1 + MH;
  v.b2 = v.w2 + MH * MH;
  v.w3 = v.b2 + MH;
  v.b3 = v.w3 + MO * MH;
  return v;
}

static void mlp_fwd1(mlp_view v, const float* x, double* a1, double* a2, double* z3) {
  for (int j = 0; j < MH; ++j) {
    double s = v.b1[j];
    for (int i = 0; i < MF; ++i) s += (double)v.w1[j * MF + i] * x[i];
    a1[j] = s > 0 ? s : 0;
  }
  for (int j = 0; j < MH; ++j) {
    double s = v.b2[j];
    for (int k = 0; k < MH; ++k) s += (double)v.w2[j * MH + k] * a1[k];
    a2[j] = s > 0 ? s : 0;
  }
  for (int o = 0; o < MO; ++o) {
    double s = v.b3[o];
    for (int k = 0; k < MH; ++k) s += (double)v.w3[o * MH + k] * a2[k];
    z3[o] = s;
  }
}

void orc_mlp_forward(const float* params, const float* X, int B, double* out) {
  mlp_view v = mlp_split(params);
  double a1[MH], a2[MH];
  for (int b = 0; b < B; ++b) mlp_fwd1(v, X + b * MF, a1, a2, out + b * MO);
}

void orc_mlp_loss_grad(const float* params, const float* X, const float* Y, const float* M, int B, double* grad,
                       double* loss) {
  mlp_view v = mlp_split(params);
  const int P = MH * MF + MH + MH * MH + MH + MO * MH + MO;
  for (int p = 0; p < P; ++p) grad[p] = 0.0;
  double* gw1 = grad;
  double* gb1 = gw1 + MH * MF;
  double* gw2 = gb1 + MH;
  double* gb2 = gw2 + MH * MH;
  double* gw3 = gb2 + MH;
  double* gb3 = gw3 + MO * MH;
  double L = 0.0;
  for (int b = 0; b < B; ++b) {
    const float* x = X + b * MF;
    const float* y = Y + b * MO;
    const float* m = M + b * MO;
    double a1[MH], a2[MH], z[MO], g3[MO], g2[MH], g1[MH];
    mlp_fwd1(v, x, a1, a2, z);
    for (int o = 0; o < MO; ++o) {
      if (o < 2) {
        double sp = (z[o] > 0 ? z[o] : 0) + log1p(exp(-fabs(z[o])));
        L += m[o] * (sp - y[o] * z[o]);
        g3[o] = m[o] * (1.0 / (1.0 + exp(-z[o])) - y[o]) / B;
      } else {
        double e = z[o] - y[o];
        L += m[o] * 0.5 * e * e;
        g3[o] = m[o] * e / B;
      }
    }
    for (int k = 0; k < MH; ++k) {
      double s = 0;
      for (int o = 0; o < MO; ++o) s += (double)v.w3[o * MH + k] * g3[o];
      g2[k] = a2[k] > 0 ? s : 0;
    }
    for (int k = 0; k < MH; ++k) {
      double s = 0;
      for (int j = 0; j < MH; ++j) s += (double)v.w2[j * MH + k] * g2[j];
      g1[k] = a1[k] > 0 ? s : 0;
    }
    for (int j = 0; j < MH; ++j) {
      for (int i = 0; i < MF; ++i) gw1[j * MF + i] += g1[j] * x[i];
      gb1[j] += g1[j];
      for (int k = 0; k < MH; ++k) gw2[j * MH + k] += g2[j] * a1[k];
      gb2[j] += g2[j];
    }
    for (int o = 0; o < MO; ++o) {
      for (int k = 0; k < MH; ++k) gw3[o * MH + k] += g3[o] * a2[k];
      gb3[o] += g3[o];
    }
  }
  if (loss) *loss = L / B;
}
