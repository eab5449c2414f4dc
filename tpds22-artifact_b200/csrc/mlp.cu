// The learned part: a 12 -> 32 -> 32 -> 4 FP32 MLP (ReLU) with hand-written
// inference and training kernels.  It is trained on per-level traces that the
// plain traversals emit (gsrb_graph_trace) and drives the per-level direction
// choice of the learned BFS (graph.cu); the policy falls back to the fixed
// heuristic once a prediction of the next frontier misses by more than 2x, so
// it changes the schedule and never the results.
//
// Heads: [0] logit(pull is faster), [1] logit(topology push is faster than the
// worklist push), [2] log2(1 + next frontier size), [3] spare.
// Loss: masked binary cross-entropy with logits on heads 0-1, masked
// 0.5 * squared error on heads 2-3, averaged over the batch.
//
// Training is one persistent kernel on the grid barrier: per step, phase A
// (sample-parallel forward + backward deltas) -> barrier -> phase B
// (parameter-parallel gradient sums in a fixed sample order, Adam update) ->
// barrier.  Deterministic: no floating-point atomics.
#include "internal.h"
#include "graph_common.cuh"

#include <math.h>
#include <string.h>

using namespace gsrbrt;
using gsrbg::kFeat;
using gsrbg::kHid;
using gsrbg::kOut;
using gsrbg::MLPWeights;

namespace {

constexpr int kParams = sizeof(MLPWeights) / sizeof(float);
static_assert(kParams == kHid * kFeat + kHid + kHid * kHid + kHid + kOut * kHid + kOut, "param layout");

struct TrainBufs {
  float* h1;   // [B][32] post-ReLU layer 1
  float* h2;   // [B][32] post-ReLU layer 2
  float* d1;   // [B][32] dL/d(pre-activation 1)
  float* d2;   // [B][32]
  float* d3;   // [B][4]  dL/d(output)
  float* lsum; // [B] per-sample loss
  float* m;    // Adam first moment [P]
  float* v;    // Adam second moment [P]
};

__device__ __forceinline__ float softplus(float z) { return fmaxf(z, 0.f) + log1pf(expf(-fabsf(z))); }
__device__ __forceinline__ float sigmoidf_(float z) { return 1.f / (1.f + expf(-z)); }

// Forward + backward of one sample; writes activations and deltas.
__device__ void sample_fwd_bwd(const MLPWeights* __restrict__ W, const float* __restrict__ x, const float* __restrict__ y,
                               const float* __restrict__ msk, float* h1, float* h2, float* d1, float* d2, float* d3,
                               float* loss, float invB) {
  float a1[kHid], a2[kHid];
  for (int j = 0; j < kHid; ++j) {
    float s = W->b1[j];
    for (int i = 0; i < kFeat; ++i) s = fmaf(W->w1[j][i], x[i], s);
    a1[j] = fmaxf(s, 0.f);
  }
  for (int j = 0; j < kHid; ++j) {
    float s = W->b2[j];
    for (int k = 0; k < kHid; ++k) s = fmaf(W->w2[j][k], a1[k], s);
    a2[j] = fmaxf(s, 0.f);
  }
  float l = 0.f;
  float g3[kOut];
  for (int o = 0; o < kOut; ++o) {
    float s = W->b3[o];
    for (int k = 0; k < kHid; ++k) s = fmaf(W->w3[o][k], a2[k], s);
    if (o < 2) {
      l += msk[o] * (softplus(s) - y[o] * s);
      g3[o] = msk[o] * (sigmoidf_(s) - y[o]) * invB;
    } else {
      const float e = s - y[o];
      l += msk[o] * 0.5f * e * e;
      g3[o] = msk[o] * e * invB;
    }
  }
  float g2[kHid], g1[kHid];
  for (int k = 0; k < kHid; ++k) {
    float s = 0.f;
    for (int o = 0; o < kOut; ++o) s = fmaf(W->w3[o][k], g3[o], s);
    g2[k] = a2[k] > 0.f ? s : 0.f;
  }
  for (int k = 0; k < kHid; ++k) {
    float s = 0.f;
    for (int j = 0; j < kHid; ++j) s = fmaf(W->w2[j][k], g2[j], s);
    g1[k] = a1[k] > 0.f ? s : 0.f;
  }
  for (int j = 0; j < kHid; ++j) {
    h1[j] = a1[j];
    h2[j] = a2[j];
    d1[j] = g1[j];
    d2[j] = g2[j];
  }
  for (int o = 0; o < kOut; ++o) d3[o] = g3[o];
  *loss = l * invB;
}

// Gradient of parameter p (flat index into MLPWeights) from the stored deltas,
// summed over samples in index order.
__device__ float param_grad(int p, const float* __restrict__ X, int B, const TrainBufs& t) {
  float g = 0.f;
  int q = p;
  if (q < kHid * kFeat) {
    const int j = q / kFeat, i = q % kFeat;
    for (int b = 0; b < B; ++b) g = fmaf(t.d1[b * kHid + j], X[b * kFeat + i], g);
    return g;
  }
  q -= kHid * kFeat;
  if (q < kHid) {
    for (int b = 0; b < B; ++b) g += t.d1[b * kHid + q];
    return g;
  }
  q -= kHid;
  if (q < kHid * kHid) {
    const int j = q / kHid, k = q % kHid;
    for (int b = 0; b < B; ++b) g = fmaf(t.d2[b * kHid + j], t.h1[b * kHid + k], g);
    return g;
  }
  q -= kHid * kHid;
  if (q < kHid) {
    for (int b = 0; b < B; ++b) g += t.d2[b * kHid + q];
    return g;
  }
  q -= kHid;
  if (q < kOut * kHid) {
    const int o = q / kHid, k = q % kHid;
    for (int b = 0; b < B; ++b) g = fmaf(t.d3[b * kOut + o], t.h2[b * kHid + k], g);
    return g;
  }
  q -= kOut * kHid;
  for (int b = 0; b < B; ++b) g += t.d3[b * kOut + q];
  return g;
}

__global__ void mlp_forward_kernel(const MLPWeights* __restrict__ W, const float* __restrict__ X, int B,
                                   float* __restrict__ out) {
  // one warp per sample, the same routine the traversal uses
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  for (int b = warp; b < B; b += nw) {
    float feat[kFeat], o[kOut];
    for (int i = 0; i < kFeat; ++i) feat[i] = X[b * kFeat + i];
    gsrbg::mlp_forward_warp(W, feat, o);
    if ((threadIdx.x & 31) == 0)
      for (int k = 0; k < kOut; ++k) out[b * kOut + k] = o[k];
  }
}

// One evaluation of loss and gradient (for checking against the CPU oracle).
__global__ void mlp_grad_phaseA(const MLPWeights* W, const float* X, const float* Y, const float* M, int B,
                                TrainBufs t) {
  const float invB = 1.f / (float)B;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x)
    sample_fwd_bwd(W, X + b * kFeat, Y + b * kOut, M + b * kOut, t.h1 + b * kHid, t.h2 + b * kHid,
                   t.d1 + b * kHid, t.d2 + b * kHid, t.d3 + b * kOut, t.lsum + b, invB);
}
__global__ void mlp_grad_phaseB(const float* X, int B, TrainBufs t, float* grad, float* loss) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < kParams; p += gridDim.x * blockDim.x)
    grad[p] = param_grad(p, X, B, t);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    float l = 0.f;
    for (int b = 0; b < B; ++b) l += t.lsum[b];
    *loss = l;
  }
}

// Persistent training loop: Adam (beta1 0.9, beta2 0.999, eps 1e-8).
template <int V>
__global__ void __launch_bounds__(256)
mlp_train_kernel(gsrb::GridBarrier gb, float* params, const float* X, const float* Y, const float* M, int B,
                 int steps, float lr, TrainBufs t, float* loss_hist) {
  __shared__ gsrb::BarrierShared bsh;
  gsrb::GridSync<V> bar;
  bool ok = bar.init(gb, &bsh);
  const MLPWeights* W = reinterpret_cast<const MLPWeights*>(params);
  const float invB = 1.f / (float)B;
  const int tid = blockIdx.x * blockDim.x + threadIdx.x, nt = gridDim.x * blockDim.x;
  for (int p = tid; p < kParams; p += nt) {
    t.m[p] = 0.f;
    t.v[p] = 0.f;
  }
  float b1p = 1.f, b2p = 1.f;
  for (int s = 0; ok && s < steps; ++s) {
    for (int b = tid; b < B; b += nt)
      sample_fwd_bwd(W, X + b * kFeat, Y + b * kOut, M + b * kOut, t.h1 + b * kHid, t.h2 + b * kHid,
                     t.d1 + b * kHid, t.d2 + b * kHid, t.d3 + b * kOut, t.lsum + b, invB);
    ok = bar.sync();
    if (!ok) break;
    b1p *= 0.9f;
    b2p *= 0.999f;
    for (int p = tid; p < kParams; p += nt) {
      const float g = param_grad(p, X, B, t);
      const float m = 0.9f * t.m[p] + 0.1f * g;
      const float v = 0.999f * t.v[p] + 0.001f * g * g;
      t.m[p] = m;
      t.v[p] = v;
      const float mh = m / (1.f - b1p), vh = v / (1.f - b2p);
      params[p] -= lr * mh / (sqrtf(vh) + 1e-8f);
    }
    if (tid == 0 && loss_hist) {
      float l = 0.f;
      for (int b = 0; b < B; ++b) l += t.lsum[b];
      loss_hist[s] = l;
    }
    ok = bar.sync();
  }
  bar.finish();
}

gsrb_status_t train_bufs(gsrb_ctx* ctx, int B, TrainBufs* t) {
  const size_t per = (size_t)B * (4 * kHid + kOut + 1) + 2 * (size_t)kParams;
  void* p = nullptr;
  gsrb_status_t st = scratch(ctx, per * sizeof(float), &p);
  if (st) return st;
  float* f = (float*)p;
  t->h1 = f; f += (size_t)B * kHid;
  t->h2 = f; f += (size_t)B * kHid;
  t->d1 = f; f += (size_t)B * kHid;
  t->d2 = f; f += (size_t)B * kHid;
  t->d3 = f; f += (size_t)B * kOut;
  t->lsum = f; f += B;
  t->m = f; f += kParams;
  t->v = f;
  return GSRB_OK;
}

uint64_t smix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

}  // namespace

extern "C" {

size_t gsrb_mlp_param_count(void) { return (size_t)kParams; }

gsrb_status_t gsrb_mlp_init(uint64_t seed, float* h) {
  if (!h) return GSRB_ERR_ARG;
  MLPWeights w;
  memset(&w, 0, sizeof(w));
  uint64_t s = seed;
  auto uni = [&](float lim) { return (float)(((smix(s) >> 40) * (1.0 / 16777216.0)) * 2.0 - 1.0) * lim; };
  // He-uniform initialisation: U(-sqrt(6/fan_in), +sqrt(6/fan_in))
  for (int j = 0; j < kHid; ++j)
    for (int i = 0; i < kFeat; ++i) w.w1[j][i] = uni(sqrtf(6.f / kFeat));
  for (int j = 0; j < kHid; ++j)
    for (int k = 0; k < kHid; ++k) w.w2[j][k] = uni(sqrtf(6.f / kHid));
  for (int o = 0; o < kOut; ++o)
    for (int k = 0; k < kHid; ++k) w.w3[o][k] = uni(sqrtf(6.f / kHid));
  memcpy(h, &w, sizeof(w));
  return GSRB_OK;
}

void gsrb_level_features(uint32_t n, uint32_t m, uint32_t level, uint32_t nf, uint64_t mf, uint32_t nu, uint64_t mu,
                         uint32_t prev_nf, uint32_t prev_dir, float* out12) {
  if (out12) gsrbg::level_features(out12, n, m, level, nf, mf, nu, mu, prev_nf, prev_dir);
}

gsrb_status_t gsrb_mlp_forward(gsrb_ctx_t ctx, const float* d_params, const float* d_x, int32_t B, float* d_out) {
  if (!ctx || !d_params || !d_x || !d_out || B < 0) return GSRB_ERR_ARG;
  if (B == 0) return GSRB_OK;
  std::lock_guard<std::mutex> g(ctx->mu);
  const MLPWeights* W = (const MLPWeights*)d_params;
  void* args[] = {&W, (void*)&d_x, &B, &d_out};
  return launch_plain(ctx, (const void*)mlp_forward_kernel, dim3(ctx->num_sms), dim3(256), 0, args);
}

gsrb_status_t gsrb_mlp_loss_grad(gsrb_ctx_t ctx, const float* d_params, const float* d_x, const float* d_y,
                                 const float* d_mask, int32_t B, float* d_grad, float* d_loss) {
  if (!ctx || !d_params || !d_x || !d_y || !d_mask || !d_grad || !d_loss || B <= 0) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  TrainBufs t;
  gsrb_status_t st = train_bufs(ctx, B, &t);
  if (st) return st;
  const MLPWeights* W = (const MLPWeights*)d_params;
  void* a1[] = {&W, (void*)&d_x, (void*)&d_y, (void*)&d_mask, &B, &t};
  st = launch_plain(ctx, (const void*)mlp_grad_phaseA, dim3(ctx->num_sms), dim3(128), 0, a1);
  if (st) return st;
  void* a2[] = {(void*)&d_x, &B, &t, &d_grad, &d_loss};
  return launch_plain(ctx, (const void*)mlp_grad_phaseB, dim3((kParams + 255) / 256), dim3(256), 0, a2);
}

gsrb_status_t gsrb_mlp_train(gsrb_ctx_t ctx, float* d_params, const float* d_x, const float* d_y,
                             const float* d_mask, int32_t B, int32_t steps, float lr, float* d_loss_hist) {
  if (!ctx || !d_params || !d_x || !d_y || !d_mask || B <= 0 || steps < 0 || !(lr > 0.f)) return GSRB_ERR_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  TrainBufs t;
  gsrb_status_t st = train_bufs(ctx, B, &t);
  if (st) return st;
  gsrb_cfg_t c = resolve_cfg(ctx, nullptr);
  c.variant = gsrb::V_FLIP;
  c.cluster = 1;
  c.threads = 256;
  const int grid = ctx->num_sms;
  gsrb::GridBarrier gb = make_barrier(ctx, c, 1, (uint32_t)grid, 0, 0);
  void* args[] = {&gb, &d_params, (void*)&d_x, (void*)&d_y, (void*)&d_mask, &B, &steps, &lr, &t, &d_loss_hist};
  return launch_persistent(ctx, (const void*)mlp_train_kernel<gsrb::V_FLIP>, grid, 256, 0, 1, coop_of(c), args);
}

}  // extern "C"
