// Co-residency queries for the persistent kernel families (used by the
// autotuner and by callers that want to size a grid before launching).
#include "internal.h"

const void* gsrb_bench_kernel_for(int variant);
const void* gsrb_reduce_kernel_for(int variant);
size_t gsrb_reduce_smem_for(const gsrb_cfg_t& c);

extern "C" gsrb_status_t gsrb_max_coresident(gsrb_ctx_t ctx, const gsrb_cfg_t* cfgin, int32_t family,
                                             int32_t* ctas) {
  if (!ctx || !ctas) return GSRB_ERR_ARG;
  gsrb_cfg_t c = gsrbrt::resolve_cfg(ctx, cfgin);
  const void* fn = nullptr;
  size_t smem = 0;
  switch (family) {
    case 0: fn = gsrb_bench_kernel_for(c.variant); break;
    case 1:
      fn = gsrb_reduce_kernel_for(c.variant);
      smem = gsrb_reduce_smem_for(c);
      break;
    default: return GSRB_ERR_ARG;
  }
  if (!fn) return GSRB_ERR_UNSUPPORTED;
  int cap = 0;
  gsrb_status_t st = gsrbrt::coresident_ctas(ctx, fn, c.threads, smem, c.cluster, &cap);
  *ctas = cap;
  return st;
}
