// libgsrb runtime: context lifetime, device facts, the persistent-launch helper
// with co-residency refusal, sticky device status, memory and timing plumbing.
//
// The reference allocates its barrier state with cudaMallocManaged per call and
// launches persistent grids with <<<>>> without checking co-residency
// (Reduce/reduce_gsrb.cu:352-384, scan/scan_gsrb.cu:735-761,
// LONESTAR/apps/bfs/kernel_gsrb.cu:673-696); a grid that is not co-resident
// hangs there.  Here the state lives in one context-owned device block, every
// persistent launch is checked against the occupancy API first (and made
// cooperative whenever the driver accepts it), and every device wait is bounded.
#include "internal.h"
#include <string.h>
#include <stdlib.h>

namespace gsrbrt {

std::atomic<uint64_t> g_launches{0};

gsrb_status_t cuda_err(cudaError_t e, const char* what) {
  if (getenv("GSRB_VERBOSE")) fprintf(stderr, "[gsrb] %s failed: %s\n", what, cudaGetErrorString(e));
  // a failed call that did not break the context leaves its code as the
  // thread's last error: clear it, so that the next entry point's own checks
  // do not report this failure again (a sticky error stays and is reported)
  (void)cudaGetLastError();
  if (e == cudaErrorMemoryAllocation) return GSRB_ERR_NOMEM;
  if (e == cudaErrorCooperativeLaunchTooLarge) return GSRB_ERR_NOT_CORESIDENT;
  return GSRB_ERR_CUDA;
}

bool is_cluster_variant(int v) {
  return v == gsrb::V_CLUSTER || v == gsrb::V_CLUSTER_ALLPOLL || v == gsrb::V_DSMEM ||
         v == gsrb::V_CLUSTER_RED || v == gsrb::V_CLUSTER_FANOUT;
}

gsrb_cfg_t resolve_cfg(const gsrb_ctx* ctx, const gsrb_cfg_t* in) {
  gsrb_cfg_t c;
  gsrb_cfg_default(&c);
  if (in) {
    c = *in;
    gsrb_cfg_t d;
    gsrb_cfg_default(&d);
    if (c.cluster <= 0) c.cluster = d.cluster;
    if (c.ctas_per_sm <= 0) c.ctas_per_sm = d.ctas_per_sm;
    if (c.threads <= 0) c.threads = d.threads;
    if (c.timeout_ms == 0) c.timeout_ms = d.timeout_ms;
    if (c.fanin_groups < 0) c.fanin_groups = 0;
    if (c.spin_ns < 0) c.spin_ns = 0;
  }
  if (!is_cluster_variant(c.variant)) c.cluster = 1;
  (void)ctx;
  return c;
}

int grid_of(const gsrb_ctx* ctx, const gsrb_cfg_t& c) {
  if (c.grid_override > 0) return c.grid_override;
  return c.ctas_per_sm * ctx->num_sms;
}

gsrb::GridBarrier make_barrier(gsrb_ctx* ctx, const gsrb_cfg_t& c, int slot, uint32_t np,
                               uint32_t first, uint32_t group_base) {
  gsrb::GridBarrier gb;
  gb.slot = ctx->slots + slot;
  gb.groups = ctx->groups + group_base;
  gb.nparticipants = np;
  gb.first_cta = first;
  uint32_t ng = 0, nflip = 0;
  switch (c.variant) {
    case gsrb::V_SOFT2:
    case gsrb::V_TREE:
      // the reference groups CTAs by blockIdx % min(grid, NUM_SM)
      // (Reduce/reduce_gsrb.cu:253-255, Heterosync/main.cu:159)
      ng = c.fanin_groups > 0 ? (uint32_t)c.fanin_groups
                              : (np < (uint32_t)ctx->num_sms ? np : (uint32_t)ctx->num_sms);
      break;
    case gsrb::V_CLUSTER:
    case gsrb::V_CLUSTER_ALLPOLL:
    case gsrb::V_DSMEM:
    case gsrb::V_FLIP:
      // split sum-to-flip words: fanin_groups of them (at most 8)
      nflip = c.fanin_groups > 0 ? (uint32_t)c.fanin_groups : 1u;
      if (nflip > 8u) nflip = 8u;
      break;
    case gsrb::V_HIER:
      // group counters: fanin_groups (the arrivals are spread over them)
      ng = c.fanin_groups > 0 ? (uint32_t)c.fanin_groups : 0u;
      // fall through: wake-up lines
    case gsrb::V_FANOUT:
    case gsrb::V_CLUSTER_FANOUT:
      nflip = c.wake_lines > 0 ? (uint32_t)c.wake_lines : 8u;
      if (nflip > 8u) nflip = 8u;
      break;
    case gsrb::V_LOCKFREE:
      // the reference goes two-level (per-SM local barrier + global) when
      // there is more than one CTA per SM (cudaLocksBarrierFast.cu:310-329)
      ng = c.fanin_groups > 0 ? (uint32_t)c.fanin_groups
                              : (np > (uint32_t)ctx->num_sms ? (uint32_t)ctx->num_sms : 0u);
      if (ng > gsrb::detail::kLfGroups) ng = gsrb::detail::kLfGroups;
      break;
    default:
      ng = 0;
  }
  if (c.variant != gsrb::V_LOCKFREE && ng + group_base > (uint32_t)kGroups) ng = kGroups - group_base;
  gb.ngroups = ng;
  gb.spin_ns = (uint32_t)c.spin_ns;
  gb.timeout_ns = (uint64_t)c.timeout_ms * 1000000ull;
  gb.flip = c.variant == gsrb::V_LOCKFREE ? ctx->lf : ctx->flip + (size_t)slot * kMaxFlip * 32;
  gb.nflip = nflip;
  gb._pad = 0;
  return gb;
}

static gsrb_status_t coresident_query(gsrb_ctx* ctx, const void* fn, int block, size_t smem, int cluster,
                                      int* ctas);

gsrb_status_t coresident_ctas(gsrb_ctx* ctx, const void* fn, int block, size_t smem, int cluster,
                              int* ctas) {
  {
    std::lock_guard<std::mutex> g(ctx->occ_mu);
    for (int i = 0; i < ctx->occ_n; ++i) {
      const gsrb_ctx::Coresident& e = ctx->occ[i];
      if (e.fn == fn && e.block == block && e.smem == smem && e.cluster == cluster) {
        *ctas = e.ctas;
        return GSRB_OK;
      }
    }
  }
  gsrb_status_t st = coresident_query(ctx, fn, block, smem, cluster, ctas);
  if (st) return st;
  std::lock_guard<std::mutex> g(ctx->occ_mu);
  // a full table starts over (the shapes in use are few)
  if (ctx->occ_n == (int)(sizeof(ctx->occ) / sizeof(ctx->occ[0]))) ctx->occ_n = 0;
  ctx->occ[ctx->occ_n++] = {fn, block, smem, cluster, *ctas};
  return GSRB_OK;
}

static gsrb_status_t coresident_query(gsrb_ctx* ctx, const void* fn, int block, size_t smem, int cluster,
                                      int* ctas) {
  // raise the kernel's dynamic shared-memory limit to what the device allows
  // next to the kernel's static shared memory (a limit set to this launch's
  // size could be below a later, cached shape's)
  if (smem > 48 * 1024) {
    cudaFuncAttributes fa;
    GSRB_CUDA(cudaFuncGetAttributes(&fa, fn));
    int lim = ctx->max_smem_optin - (int)fa.sharedSizeBytes;
    if (lim < (int)smem) lim = (int)smem;  // too large: the call below reports it
    GSRB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  }
  if (cluster <= 1) {
    int nb = 0;
    GSRB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, smem));
    *ctas = nb * ctx->num_sms;
    return GSRB_OK;
  }
  if (cluster > 8) GSRB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)cluster, 1, 1);
  cfg.blockDim = dim3((unsigned)block, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cluster;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int ncl = 0;
  GSRB_CUDA(cudaOccupancyMaxActiveClusters(&ncl, fn, &cfg));
  *ctas = ncl * cluster;
  return GSRB_OK;
}

gsrb_status_t launch_persistent(gsrb_ctx* ctx, const void* fn, int grid, int block, size_t smem,
                                int cluster, int coop, void** args, bool pdl) {
  if (grid <= 0 || block <= 0 || block > 1024) return GSRB_ERR_ARG;
  if (pdl && coop > 0) return GSRB_ERR_UNSUPPORTED;
  if (cluster < 1) cluster = 1;
  if (grid % cluster) return GSRB_ERR_ARG;
  int cap = 0;
  gsrb_status_t st = coresident_ctas(ctx, fn, block, smem, cluster, &cap);
  if (st) return st;
  if (grid > cap) {
    if (getenv("GSRB_VERBOSE"))
      fprintf(stderr, "[gsrb] refusing persistent grid %d > co-resident capacity %d (cluster %d)\n",
              grid, cap, cluster);
    return GSRB_ERR_NOT_CORESIDENT;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid, 1, 1);
  cfg.blockDim = dim3((unsigned)block, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[3];
  unsigned na = 0;
  if (pdl) {
    attr[na].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[na].val.programmaticStreamSerializationAllowed = 1;
    ++na;
  }
  if (cluster > 1) {
    attr[na].id = cudaLaunchAttributeClusterDimension;
    attr[na].val.clusterDim.x = (unsigned)cluster;
    attr[na].val.clusterDim.y = 1;
    attr[na].val.clusterDim.z = 1;
    ++na;
  }
  if (coop > 0) {
    attr[na].id = cudaLaunchAttributeCooperative;
    attr[na].val.cooperative = 1;
    ++na;
  }
  cfg.attrs = attr;
  cfg.numAttrs = na;
  cudaError_t e = cudaLaunchKernelExC(&cfg, fn, args);
  if (e != cudaSuccess && coop == 1 && cluster > 1 && e != cudaErrorCooperativeLaunchTooLarge) {
    // Some drivers refuse cooperative + cluster; the occupancy check above
    // already guarantees the grid fits, and every device wait is bounded.
    (void)cudaGetLastError();
    cfg.numAttrs = na - 1;
    e = cudaLaunchKernelExC(&cfg, fn, args);
  }
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return cuda_err(e, "cudaLaunchKernelExC(persistent)");
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return GSRB_OK;
}

gsrb_status_t launch_plain(gsrb_ctx* ctx, const void* fn, dim3 grid, dim3 block, size_t smem,
                           void** args) {
  if (smem > 48 * 1024) GSRB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  cudaError_t e = cudaLaunchKernel(fn, grid, block, args, smem, ctx->stream);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    return cuda_err(e, "cudaLaunchKernel");
  }
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return GSRB_OK;
}

gsrb_status_t scratch(gsrb_ctx* ctx, size_t bytes, void** p) {
  if (bytes > ctx->scratch_bytes) {
    if (ctx->scratch) {
      GSRB_CUDA(cudaStreamSynchronize(ctx->stream));
      GSRB_CUDA(cudaFree(ctx->scratch));
      ctx->scratch = nullptr;
      ctx->scratch_bytes = 0;
    }
    size_t sz = bytes < (1u << 20) ? (1u << 20) : bytes;
    GSRB_CUDA(cudaMalloc(&ctx->scratch, sz));
    ctx->scratch_bytes = sz;
  }
  *p = ctx->scratch;
  return GSRB_OK;
}

gsrb_status_t map_dev(uint32_t code) {
  switch (code) {
    case gsrb::GSRB_DEV_OK: return GSRB_OK;
    case gsrb::GSRB_DEV_TIMEOUT: return GSRB_ERR_TIMEOUT;
    case gsrb::GSRB_DEV_BAD_CONFIG: return GSRB_ERR_ARG;
    case gsrb::GSRB_DEV_OVERFLOW: return GSRB_ERR_OVERFLOW;
    case gsrb::GSRB_DEV_LOCK_TIMEOUT: return GSRB_ERR_LOCK_TIMEOUT;
    case gsrb::GSRB_DEV_INVARIANT: return GSRB_ERR_INVARIANT;
    default: return GSRB_ERR_STATE;
  }
}

}  // namespace gsrbrt

using namespace gsrbrt;

namespace {
// Reads (does not write) a buffer of twice the L2 size, so the next timed
// kernel starts with clean, unrelated lines in L2 and pays no write-backs.
__global__ void l2_flush_kernel(const uint4* buf, size_t n, uint32_t salt, uint32_t* sink) {
  uint32_t acc = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const uint4 v = __ldcg(buf + i);
    acc ^= v.x ^ v.y ^ v.z ^ v.w;
  }
  if (acc == salt) sink[0] = acc;  // practically never; keeps the loads alive
}
}  // namespace

extern "C" {

void gsrb_cfg_default(gsrb_cfg_t* c) {
  if (!c) return;
  memset(c, 0, sizeof(*c));
  c->variant = GSRB_BAR_CLUSTER;
  c->cluster = 2;
  c->ctas_per_sm = 2;
  c->threads = 256;
  c->fanin_groups = 0;
  c->spin_ns = 0;
  c->timeout_ms = 2000;
  c->tile = 0;
  c->grid_override = 0;
  // plain launches: a cooperative launch costs ~2 us more on B200 and buys
  // nothing here (co-residency is checked first and every wait is bounded)
  c->launch_mode = 1;
}

const char* gsrb_status_string(gsrb_status_t s) {
  switch (s) {
    case GSRB_OK: return "ok";
    case GSRB_ERR_ARG: return "invalid argument";
    case GSRB_ERR_CUDA: return "CUDA runtime error";
    case GSRB_ERR_NOT_CORESIDENT: return "persistent grid is not co-resident (refused)";
    case GSRB_ERR_TIMEOUT: return "device wait timed out";
    case GSRB_ERR_NOMEM: return "out of memory";
    case GSRB_ERR_STATE: return "bad context state";
    case GSRB_ERR_UNSUPPORTED: return "unsupported";
    case GSRB_ERR_OVERFLOW: return "device worklist overflow";
    case GSRB_ERR_LOCK_TIMEOUT: return "lock wait timed out";
    case GSRB_ERR_INVARIANT: return "device invariant violated";
    default: return "unknown status";
  }
}

gsrb_status_t gsrb_ctx_create(int device, gsrb_ctx_t* out) {
  if (!out) return GSRB_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  GSRB_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaSetDevice(device));
  gsrb_ctx* c = new gsrb_ctx();
  c->device = device;
  cudaDeviceProp p;
  cudaError_t e = cudaGetDeviceProperties(&p, device);
  if (e != cudaSuccess) { delete c; return cuda_err(e, "cudaGetDeviceProperties"); }
  c->num_sms = p.multiProcessorCount;
  c->l2_bytes = p.l2CacheSize;
  c->max_smem_optin = (int)p.sharedMemPerBlockOptin;
  e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) { delete c; return cuda_err(e, "cudaStreamCreate"); }
  c->stream = c->own_stream;
  size_t sbytes = sizeof(gsrb::BarrierSlot) * kSlots;
  size_t gbytes = sizeof(gsrb::GroupSlot) * kGroups;
  e = cudaMalloc(&c->slots, sbytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->groups, gbytes);
  const size_t fbytes = sizeof(uint32_t) * 32 * (size_t)kSlots * kMaxFlip;
  if (e == cudaSuccess) e = cudaMalloc(&c->flip, fbytes);
  if (e == cudaSuccess) e = cudaMemset(c->flip, 0, fbytes);
  if (e == cudaSuccess) e = cudaMalloc(&c->lf, sizeof(uint32_t) * gsrb::detail::kLfWords);
  if (e == cudaSuccess) e = cudaMemset(c->lf, 0, sizeof(uint32_t) * gsrb::detail::kLfWords);
  if (e == cudaSuccess) e = cudaMemset(c->slots, 0, sbytes);
  if (e == cudaSuccess) e = cudaMemset(c->groups, 0, gbytes);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    gsrb_ctx_destroy(c);
    return cuda_err(e, "context allocation");
  }
  *out = c;
  return GSRB_OK;
}

gsrb_status_t gsrb_ctx_destroy(gsrb_ctx_t c) {
  if (!c) return GSRB_ERR_ARG;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (auto& ev : c->events)
    if (ev) cudaEventDestroy(ev);
  if (c->slots) cudaFree(c->slots);
  if (c->groups) cudaFree(c->groups);
  if (c->flip) cudaFree(c->flip);
  if (c->lf) cudaFree(c->lf);
  if (c->scratch) cudaFree(c->scratch);
  if (c->flush) cudaFree(c->flush);
  if (c->own_stream) cudaStreamDestroy(c->own_stream);
  delete c;
  return GSRB_OK;
}

gsrb_status_t gsrb_ctx_set_stream(gsrb_ctx_t c, void* stream) {
  if (!c) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  return GSRB_OK;
}

gsrb_status_t gsrb_ctx_info(gsrb_ctx_t c, int32_t* num_sms, int64_t* l2, int32_t* dev) {
  if (!c) return GSRB_ERR_ARG;
  if (num_sms) *num_sms = c->num_sms;
  if (l2) *l2 = c->l2_bytes;
  if (dev) *dev = c->device;
  return GSRB_OK;
}

gsrb_status_t gsrb_ctx_synchronize(gsrb_ctx_t c) {
  if (!c) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaStreamSynchronize(c->stream));
  return GSRB_OK;
}

gsrb_status_t gsrb_ctx_status(gsrb_ctx_t c, uint32_t* code, uint32_t* where, uint32_t* who) {
  if (!c) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(c->mu);
  GSRB_CUDA(cudaStreamSynchronize(c->stream));
  uint32_t worst = 0, w_where = 0, w_who = 0;
  // every slot may carry an error (sub-grid barriers use slots 1..)
  static thread_local gsrb::BarrierSlot host[kSlots];
  GSRB_CUDA(cudaMemcpy(host, c->slots, sizeof(host), cudaMemcpyDeviceToHost));
  for (int i = 0; i < kSlots; ++i) {
    if (host[i].status && !worst) {
      worst = host[i].status;
      w_where = host[i].where;
      w_who = host[i].who;
    }
  }
  if (code) *code = worst;
  if (where) *where = w_where;
  if (who) *who = w_who;
  if (worst) {
    // a failed episode leaves counters half-way: reset all barrier state
    GSRB_CUDA(cudaMemset(c->slots, 0, sizeof(gsrb::BarrierSlot) * kSlots));
    GSRB_CUDA(cudaMemset(c->groups, 0, sizeof(gsrb::GroupSlot) * kGroups));
    GSRB_CUDA(cudaMemset(c->flip, 0, sizeof(uint32_t) * 32 * (size_t)kSlots * kMaxFlip));
    GSRB_CUDA(cudaMemset(c->lf, 0, sizeof(uint32_t) * gsrb::detail::kLfWords));
    GSRB_CUDA(cudaDeviceSynchronize());
  }
  return map_dev(worst);
}

gsrb_status_t gsrb_malloc(void** p, size_t bytes) {
  if (!p) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaMalloc(p, bytes ? bytes : 1));
  return GSRB_OK;
}
gsrb_status_t gsrb_free(void* p) {
  if (p) GSRB_CUDA(cudaFree(p));
  return GSRB_OK;
}
gsrb_status_t gsrb_host_alloc(void** p, size_t bytes) {
  if (!p) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaMallocHost(p, bytes ? bytes : 1));
  return GSRB_OK;
}
gsrb_status_t gsrb_host_free(void* p) {
  if (p) GSRB_CUDA(cudaFreeHost(p));
  return GSRB_OK;
}
gsrb_status_t gsrb_memcpy_h2d(gsrb_ctx_t c, void* d, const void* h, size_t n) {
  if (!c) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaMemcpyAsync(d, h, n, cudaMemcpyHostToDevice, c->stream));
  return GSRB_OK;
}
gsrb_status_t gsrb_memcpy_d2h(gsrb_ctx_t c, void* h, const void* d, size_t n) {
  if (!c) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaMemcpyAsync(h, d, n, cudaMemcpyDeviceToHost, c->stream));
  return GSRB_OK;
}
gsrb_status_t gsrb_memset(gsrb_ctx_t c, void* d, int v, size_t n) {
  if (!c) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaMemsetAsync(d, v, n, c->stream));
  return GSRB_OK;
}

gsrb_status_t gsrb_event_record(gsrb_ctx_t c, int32_t slot) {
  if (!c || slot < 0 || slot >= 64) return GSRB_ERR_ARG;
  if (!c->events[slot]) GSRB_CUDA(cudaEventCreate(&c->events[slot]));
  GSRB_CUDA(cudaEventRecord(c->events[slot], c->stream));
  return GSRB_OK;
}

gsrb_status_t gsrb_event_elapsed_ms(gsrb_ctx_t c, int32_t a, int32_t b, float* ms) {
  if (!c || a < 0 || b < 0 || a >= 64 || b >= 64 || !ms || !c->events[a] || !c->events[b]) return GSRB_ERR_ARG;
  GSRB_CUDA(cudaEventSynchronize(c->events[b]));
  GSRB_CUDA(cudaEventElapsedTime(ms, c->events[a], c->events[b]));
  return GSRB_OK;
}

gsrb_status_t gsrb_l2_flush(gsrb_ctx_t c) {
  if (!c) return GSRB_ERR_ARG;
  size_t want = (size_t)(c->l2_bytes > 0 ? c->l2_bytes : (128 << 20)) * 2;
  if (c->flush_bytes < want) {
    if (c->flush) GSRB_CUDA(cudaFree(c->flush));
    c->flush = nullptr;
    GSRB_CUDA(cudaMalloc(&c->flush, want + 256));
    GSRB_CUDA(cudaMemsetAsync(c->flush, 0x5a, want + 256, c->stream));
    c->flush_bytes = want;
  }
  static uint32_t salt = 1;
  const uint4* buf = (const uint4*)c->flush;
  size_t n = c->flush_bytes / sizeof(uint4);
  uint32_t s = salt++;
  uint32_t* sink = (uint32_t*)((char*)c->flush + c->flush_bytes);
  void* args[] = {&buf, &n, &s, &sink};
  return launch_plain(c, (const void*)l2_flush_kernel, dim3(c->num_sms * 4), dim3(512), 0, args);
}

uint64_t gsrb_launch_count(void) { return g_launches.load(); }

}  // extern "C"
