// Reference-named drop-in host entry points (see gsrb/compat.h).
#include "internal.h"
#include "gsrb/compat.h"

namespace {

std::mutex g_default_mu;
gsrb_ctx_t g_default = nullptr;

gsrb_ctx_t default_ctx() {
  std::lock_guard<std::mutex> g(g_default_mu);
  if (!g_default) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) dev = 0;
    if (gsrb_ctx_create(dev, &g_default) != GSRB_OK) g_default = nullptr;
  }
  return g_default;
}

void report(const char* what, gsrb_status_t st) {
  if (st) fprintf(stderr, "[gsrb] %s failed: %s (%d)\n", what, gsrb_status_string(st), st);
}

}  // namespace

int reduce(const int* arr, unsigned int N, unsigned int threads_per_block) {
  gsrb_ctx_t ctx = default_ctx();
  if (!ctx || (N && !arr)) {
    fprintf(stderr, "[gsrb] reduce: no device context\n");
    return 0;
  }
  gsrb_cfg_t c;
  gsrb_cfg_default(&c);
  // the reference's block size is honoured when it is a legal CTA size
  if (threads_per_block >= 32 && threads_per_block <= 1024 && threads_per_block % 32 == 0)
    c.threads = (int)threads_per_block;
  int32_t* d_in = nullptr;
  int64_t* d_out = nullptr;
  long long sum = 0;
  gsrb_status_t st = gsrb_malloc((void**)&d_in, sizeof(int32_t) * (size_t)N);
  if (!st) st = gsrb_malloc((void**)&d_out, sizeof(int64_t));
  if (!st && N) st = gsrb_memcpy_h2d(ctx, d_in, arr, sizeof(int32_t) * (size_t)N);
  if (!st) st = gsrb_event_record(ctx, 60);
  if (!st) st = gsrb_reduce_i32(ctx, d_in, N, d_out, &c);
  if (!st) st = gsrb_event_record(ctx, 61);
  float ms = 0.f;
  if (!st) st = gsrb_event_elapsed_ms(ctx, 60, 61, &ms);
  if (!st) st = gsrb_memcpy_d2h(ctx, &sum, d_out, sizeof(sum));
  if (!st) st = gsrb_ctx_status(ctx, nullptr, nullptr, nullptr);
  report("reduce", st);
  printf("time (ms) is %f\n", ms);
  gsrb_free(d_in);
  gsrb_free(d_out);
  // the reference accumulates in int: the low 32 bits of the exact sum
  return (int)(unsigned int)(unsigned long long)sum;
}

void sum_scan_blelloch(unsigned int* d_out, unsigned int* d_in, const size_t numElems) {
  gsrb_ctx_t ctx = default_ctx();
  if (!ctx) {
    fprintf(stderr, "[gsrb] sum_scan_blelloch: no device context\n");
    return;
  }
  // the reference works on the legacy default stream; order with it
  cudaDeviceSynchronize();
  gsrb_status_t st = gsrb_event_record(ctx, 60);
  if (!st) st = gsrb_scan_u32(ctx, d_in, d_out, numElems, nullptr);
  if (!st) st = gsrb_event_record(ctx, 61);
  float ms = 0.f;
  if (!st) st = gsrb_event_elapsed_ms(ctx, 60, 61, &ms);
  if (!st) st = gsrb_ctx_status(ctx, nullptr, nullptr, nullptr);
  report("sum_scan_blelloch", st);
  printf("Kernel time (ms) %f\n", ms);
}

void sum_scan_naive(unsigned int* const d_out, const unsigned int* const d_in, const size_t numElems) {
  sum_scan_blelloch(d_out, const_cast<unsigned int*>(d_in), numElems);
}
