// Kernel-level tracing: when enabled, every pass launch is bracketed by CUDA
// events recorded on the launching stream, tagged with the pass kind and its
// algorithmic byte count.  wap_profile_read sums the elapsed times per kind.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <vector>

#include "wap_internal.h"

namespace wap {

namespace {
struct Rec {
  int kind;
  double bytes;
  cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;

cudaEvent_t take() {
  if (!g_pool.empty()) {
    cudaEvent_t e = g_pool.back();
    g_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}
}  // namespace

bool prof_on() { return g_on; }

// FP32 peak probe: every thread runs 8 independent FMA chains (a dependent
// FMA's latency is covered by the other chains and the other warps), the
// outer loop unrolled so that loop control is a few percent of the issue.
__global__ void __launch_bounds__(256) fma_probe_kernel(int iters, float x, float y, float* out) {
  float a[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) a[j] = 1e-3f * (float)threadIdx.x + (float)j;
#pragma unroll 16
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = fmaf(a[j], x, y);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += a[j];
  out[(long long)blockIdx.x * blockDim.x + threadIdx.x] = s;
}

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

ProfToken prof_begin(int kind, cudaStream_t st) {
  ProfToken t{};
  if (!g_on) return t;
  std::lock_guard<std::mutex> lk(g_mu);
  t.active = true;
  t.kind = kind;
  t.a = take();
  t.b = take();
  cudaEventRecord(t.a, st);
  return t;
}

void prof_end(const ProfToken& t, cudaStream_t st, double bytes) {
  if (!t.active) return;
  cudaEventRecord(t.b, st);
  std::lock_guard<std::mutex> lk(g_mu);
  g_recs.push_back(Rec{t.kind, bytes, t.a, t.b});
}

}  // namespace wap

using namespace wap;

extern "C" {

long long wap_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int wap_profile_enable(int on) {
  clear_error();
  std::lock_guard<std::mutex> lk(g_mu);
  g_on = on != 0;
  return WAP_OK;
}

int wap_profile_reset(void) {
  clear_error();
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto& r : g_recs) {
    g_pool.push_back(r.a);
    g_pool.push_back(r.b);
  }
  g_recs.clear();
  return WAP_OK;
}

int wap_fp32_probe(int blocks, int iters, float* out, void* stream) {
  clear_error();
  if (blocks < 1 || iters < 1 || !out) return fail(WAP_ERR_ARG, "need blocks >= 1, iters >= 1 and an output buffer");
  count_launch();
  fma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(iters, 0.999999f, 1e-6f, out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, "fma_probe_kernel");
}

int wap_profile_read(int kind, long long* launches, double* total_ms, double* total_bytes) {
  clear_error();
  if (!launches || !total_ms || !total_bytes) return fail(WAP_ERR_ARG, "NULL output pointer");
  std::lock_guard<std::mutex> lk(g_mu);
  long long n = 0;
  double ms = 0, by = 0;
  for (auto& r : g_recs) {
    if (r.kind != kind) continue;
    cudaError_t e = cudaEventSynchronize(r.b);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventSynchronize");
    float t = 0;
    e = cudaEventElapsedTime(&t, r.a, r.b);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventElapsedTime");
    ++n;
    ms += t;
    by += r.bytes;
  }
  *launches = n;
  *total_ms = ms;
  *total_bytes = by;
  return WAP_OK;
}

}  // extern "C"
