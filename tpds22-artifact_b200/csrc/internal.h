// Internal host-side runtime of libgsrb: the context object, the persistent
// launch helper (co-residency check + cooperative / cluster launch) and the
// translation of a gsrb_cfg_t into the device GridBarrier descriptor.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <mutex>
#include <stdint.h>
#include <stdio.h>
#include "gsrb.h"
#include "gsrb/barrier.cuh"

struct gsrb_ctx {
  int device = 0;
  int num_sms = 0;
  int64_t l2_bytes = 0;
  int max_smem_optin = 0;
  cudaStream_t stream = nullptr;
  cudaStream_t own_stream = nullptr;
  std::mutex mu;
  // barrier state: kSlots slots + kGroups fan-in groups (device)
  gsrb::BarrierSlot* slots = nullptr;
  gsrb::GroupSlot* groups = nullptr;
  uint32_t* flip = nullptr;  // kSlots * kMaxFlip lines of 32 words
  uint32_t* lf = nullptr;    // lock-free flag barrier area (gsrb::detail::kLfWords words)
  // general scratch (device), grown on demand
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // L2 flush buffer
  void* flush = nullptr;
  size_t flush_bytes = 0;
  cudaEvent_t events[64] = {};
  // co-resident capacity per (kernel, block, dynamic smem, cluster): the
  // occupancy query and the shared-memory attribute cost microseconds of host
  // time before every persistent launch, so each shape is asked once
  struct Coresident {
    const void* fn;
    int block;
    size_t smem;
    int cluster;
    int ctas;
  };
  std::mutex occ_mu;
  Coresident occ[64] = {};
  int occ_n = 0;
};

namespace gsrbrt {

constexpr int kSlots = 128;     // slot 0: whole-grid barrier; others: sub-grid barriers
constexpr int kGroups = 8192;   // fan-in / per-group counters shared by all slots
constexpr int kMaxFlip = 16;    // flip words per slot (native variants)

extern std::atomic<uint64_t> g_launches;

gsrb_status_t cuda_err(cudaError_t e, const char* what);
#define GSRB_CUDA(call)                                         \
  do {                                                          \
    cudaError_t _e = (call);                                    \
    if (_e != cudaSuccess) return gsrbrt::cuda_err(_e, #call);  \
  } while (0)

// Fill defaults into a possibly partially-set configuration.
gsrb_cfg_t resolve_cfg(const gsrb_ctx* ctx, const gsrb_cfg_t* in);
int grid_of(const gsrb_ctx* ctx, const gsrb_cfg_t& c);
bool is_cluster_variant(int v);

// Device barrier descriptor for slot `slot`, `nparticipants` CTAs starting at
// block `first`, group counters starting at `group_base`.
gsrb::GridBarrier make_barrier(gsrb_ctx* ctx, const gsrb_cfg_t& c, int slot, uint32_t nparticipants,
                               uint32_t first, uint32_t group_base);

// Launch a persistent kernel.  Refuses (GSRB_ERR_NOT_CORESIDENT) a grid larger
// than the co-resident capacity; attaches the cluster dimension.  coop:
// 2 = cooperative launch required (GSRB_BAR_CCG), 1 = cooperative when the
// driver accepts it, 0 = plain launch (safe: co-residency was checked and every
// device wait is bounded).  pdl (plain launches only): launch with programmatic
// stream serialisation, so that the kernel may start while the one before it on
// the stream is still running (it must call ptx::griddep_wait before touching
// anything that kernel uses).
gsrb_status_t launch_persistent(gsrb_ctx* ctx, const void* fn, int grid, int block, size_t smem,
                                int cluster, int coop, void** args, bool pdl = false);
inline int coop_of(const gsrb_cfg_t& c) {
  if (c.variant == gsrb::V_CCG) return 2;
  return c.launch_mode == 1 ? 0 : 1;
}
// Plain (non-persistent) launch on the context stream.
gsrb_status_t launch_plain(gsrb_ctx* ctx, const void* fn, dim3 grid, dim3 block, size_t smem, void** args);
// Co-resident capacity (CTAs) of fn for the given shape.
gsrb_status_t coresident_ctas(gsrb_ctx* ctx, const void* fn, int block, size_t smem, int cluster, int* ctas);

// Scratch device memory of at least `bytes` (context-owned, reused).
gsrb_status_t scratch(gsrb_ctx* ctx, size_t bytes, void** p);

// Map a device status code to the host status.
gsrb_status_t map_dev(uint32_t code);

}  // namespace gsrbrt

