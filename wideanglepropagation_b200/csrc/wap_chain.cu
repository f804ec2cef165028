// One-launch multislice of a single probe (or two): every slice's row and
// column pass in one cooperative kernel, separated by grid-wide barriers.
//
// A probe's pass is a few hundred CTAs and a few microseconds of work, so the
// per-pass chain (2 N + 1 launches, programmatic dependent launch) is bound by
// launch and L2 latencies, and by the host's launch rate.  Here the grid is
// made of CTAs that are all resident (cooperative launch), the twiddle table
// is loaded into shared memory once, and each pass is a loop over tiles with
// the same bodies as the pass kernels (row_pass_body / col_pass_body), the
// passes separated by a barrier over the grid: each CTA publishes its writes
// (__threadfence), bumps a counter and waits until it reaches
// (barrier index) x (grid size).  The waits are bounded: past the spin limit
// the CTA records WAP_ERR_TIMEOUT in the plan's status word and returns, and
// the other CTAs leave at their next barrier (wap_plan_status_async reads it).
// Waves written inside the kernel are read back only through L2 (__ldcg).
#include <cuda_runtime.h>

#include <algorithm>

#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

constexpr int kChainThreads = 256;
constexpr long long kChainSpinLimit = 1LL << 24;   // polls of a barrier before it gives up (~seconds)

struct ChainArgs {
  RowArgs r;
  ColArgs c;
  int n_slices, n_probes;
  float2* stack;            // (B, n_slices, ny, nx) or null
  const float4* tw;         // (n, E) table
  unsigned* count;          // barrier counter (zeroed before the launch)
  int* status;              // 0 or WAP_ERR_TIMEOUT
  long long spin_limit;
};

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// grid-wide barrier number k (1, 2, ...): false if this CTA must stop
__device__ __forceinline__ bool chain_barrier(const ChainArgs& a, unsigned k) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    atomicAdd(a.count, 1u);
    const unsigned target = k * gridDim.x;
    long long spins = 0;
    unsigned ns = 32;
    while (ld_acquire_u32(a.count) < target) {
      if (++spins > a.spin_limit || *(volatile int*)a.status != 0) {
        atomicCAS(a.status, 0, WAP_ERR_TIMEOUT);
        ok = 0;
        break;
      }
      __nanosleep(ns);
      if (ns < 256) ns <<= 1;
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

template <int N, int E>
__global__ void __launch_bounds__(kChainThreads, 2) chain_kernel(const ChainArgs a) {
  using P = FFTPlan<N, E>;
  constexpr int T = P::T;
  extern __shared__ float4 chain_smem[];
  float4* tw = chain_smem;
  float2* buf = reinterpret_cast<float2*>(tw + P::TW_SIZE);
  for (int i = threadIdx.x; i < P::TW_SIZE; i += blockDim.x) tw[i] = __ldg(a.tw + i);
  __syncthreads();
  RowArgs r = a.r;
  ColArgs c = a.c;
  const long long plane = (long long)N * N;
  const int rblocks = N / (kChainThreads / T);   // row tiles per probe
  const int cblocks = N / (kChainThreads / T);   // column tiles per probe
  const int runits = rblocks * a.n_probes, cunits = cblocks * a.n_probes;
  const int tflag = r.ttab ? ROW_TRANS_TAB : ROW_TRANS;
  unsigned k = 0;
  for (int s = 0; s <= a.n_slices; ++s) {
    r.slice = s;
    r.flags = (s == 0 ? ROW_LOAD_SRC : ROW_IFFT) | (s < a.n_slices ? (tflag | ROW_FFT) : 0);
    r.snap = (a.stack && s >= 1) ? a.stack + (long long)(s - 1) * plane : nullptr;
    r.snap_bstride = (long long)a.n_slices * plane;
    for (int u = blockIdx.x; u < runits; u += gridDim.x) {
      row_pass_body<N, E>(r, tw, buf, u % rblocks, u / rblocks);
      __syncthreads();
    }
    if (s == a.n_slices) break;
    if (!chain_barrier(a, ++k)) return;
    c.flags = (s == a.n_slices - 1 && c.dp) ? COL_DP : 0;
    for (int u = blockIdx.x; u < cunits; u += gridDim.x) {
      col_pass_body<N, E, false>(c, tw, buf, u % cblocks, u / cblocks);
      __syncthreads();
    }
    if (!chain_barrier(a, ++k)) return;
  }
}

// elements per thread of the chain for an n x n grid: T = n / E <= 128, so
// that a 256-thread CTA holds at least two column tiles' lanes
static int chain_elems(int n) { return n <= 256 ? 4 : n <= 1024 ? 8 : 16; }

template <int N, int E>
static size_t chain_smem_bytes() {
  constexpr int T = N / E;
  const size_t rows = kChainThreads / T, w = kChainThreads / T;
  const size_t row_buf = rows * RowCfg<N, E>::PADN * sizeof(float2);
  const size_t col_buf = (size_t)N * w * sizeof(float2);
  return FFTPlan<N, E>::TW_SIZE * sizeof(float4) + std::max(row_buf, col_buf);
}

template <int N, int E>
static cudaError_t chain_launch_t(const ChainArgs& a, cudaStream_t st, int* grid_out) {
  auto kern = chain_kernel<N, E>;
  const size_t smem = chain_smem_bytes<N, E>();
  cudaError_t e;
  if (smem > 48 * 1024 && (e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) !=
                              cudaSuccess)
    return e;
  int dev = 0, sms = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kChainThreads, smem)) != cudaSuccess) return e;
  constexpr int T = N / E;
  const int units = (N / (kChainThreads / T)) * a.n_probes;
  const int grid = std::min(units, per_sm * sms);
  if (grid < 1) return cudaErrorInvalidConfiguration;
  *grid_out = grid;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(kChainThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  count_launch();
  return cudaLaunchKernelEx(&cfg, kern, a);
}

static cudaError_t chain_launch(int n, int e, const ChainArgs& a, cudaStream_t st, int* grid) {
  switch (e * 100000 + n) {
    case 4 * 100000 + 128: return chain_launch_t<128, 4>(a, st, grid);
    case 8 * 100000 + 128: return chain_launch_t<128, 8>(a, st, grid);
    case 4 * 100000 + 256: return chain_launch_t<256, 4>(a, st, grid);
    case 8 * 100000 + 256: return chain_launch_t<256, 8>(a, st, grid);
    case 16 * 100000 + 256: return chain_launch_t<256, 16>(a, st, grid);
    case 4 * 100000 + 512: return chain_launch_t<512, 4>(a, st, grid);
    case 8 * 100000 + 512: return chain_launch_t<512, 8>(a, st, grid);
    case 16 * 100000 + 512: return chain_launch_t<512, 16>(a, st, grid);
    case 8 * 100000 + 1024: return chain_launch_t<1024, 8>(a, st, grid);
    case 16 * 100000 + 1024: return chain_launch_t<1024, 16>(a, st, grid);
    case 16 * 100000 + 2048: return chain_launch_t<2048, 16>(a, st, grid);
    default: return cudaErrorInvalidValue;
  }
}

constexpr int kChainMaxProbes = 2;

// The chain pays one grid-wide barrier per pass (about two microseconds) in
// place of a launch; measured on B200 it wins where the per-pass chain is
// bound by the host's launch rate (up to 256^2: C1 0.18 vs 0.23 ms per call)
// and loses on larger grids (1024^2 x 100 slices: 3.58 vs 2.69 ms), so by
// default it serves grids up to kChainMaxSize.  WAP_KNOB_CHAIN: 0 off, 1 the
// default, 4 / 8 / 16 that many elements per thread on any chain size.
constexpr int kChainMaxSize = 256;

int chain_forward(wap_plan* p, const RowArgs& r, const ColArgs& c, int n_probes, int n_slices, float2* stack,
                  cudaStream_t st) {
  const int n = p->nx;
  const int kv = knob_value(WAP_KNOB_CHAIN);
  if (kv == 0) return -1;
  if (p->generic || p->ny != n || n < 128 || n > 2048 || n_probes > kChainMaxProbes) return -1;
  if (kv < 2 && n > kChainMaxSize) return -1;
  cudaError_t e;
  int E = chain_elems(n);
  if (kv == 4 || kv == 8 || kv == 16) E = kv;
  if (n / E > 128 || n / E < 8) return -1;   // whole rows and >= 2 column lanes per 256-thread CTA
  if (p->chain_e != E) {
    cudaFree(p->chain_tw);
    p->chain_tw = nullptr;
    p->chain_e = 0;
    const std::vector<float4> h = twiddle_table(n, E);
    if ((e = cudaMalloc(&p->chain_tw, h.size() * sizeof(float4))) != cudaSuccess ||
        (e = cudaMemcpy(p->chain_tw, h.data(), h.size() * sizeof(float4), cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_fail(e, "chain twiddle table");
    p->chain_e = E;
  }
  if (!p->chain_count) {
    if ((e = cudaMalloc(&p->chain_count, sizeof(unsigned))) != cudaSuccess ||
        (e = cudaMalloc(&p->chain_status, sizeof(int))) != cudaSuccess ||
        (e = cudaMemset(p->chain_status, 0, sizeof(int))) != cudaSuccess)
      return cuda_fail(e, "chain counters");
  }
  if ((e = cudaMemsetAsync(p->chain_count, 0, sizeof(unsigned), st)) != cudaSuccess ||
      (e = cudaMemsetAsync(p->chain_status, 0, sizeof(int), st)) != cudaSuccess)
    return cuda_fail(e, "chain counter reset");
  ChainArgs a{};
  a.r = r;
  a.c = c;
  a.r.tw = p->chain_tw;
  a.c.tw = p->chain_tw;
  a.r.probe0 = a.c.probe0 = 0;
  a.n_slices = n_slices;
  a.n_probes = n_probes;
  a.stack = stack;
  a.tw = p->chain_tw;
  a.count = p->chain_count;
  a.status = p->chain_status;
  a.spin_limit = kChainSpinLimit;
  int grid = 0;
  const ProfToken tok = prof_begin(WAP_KIND_ROW, st);
  if ((e = chain_launch(n, E, a, st, &grid)) != cudaSuccess) return cuda_fail(e, "chain_kernel");
  p->chain_ran = 1;
  // one slice step: wave in / out twice, potential or table once
  prof_end(tok, st, (double)n_probes * n_slices * n * n * 20.0);
  return WAP_OK;
}

}  // namespace wap

using namespace wap;

extern "C" int wap_plan_status_pending(wap_plan* p, int* pending) {
  clear_error();
  if (!p || !pending) return fail(WAP_ERR_ARG, "NULL argument");
  *pending = p->chain_ran;
  return WAP_OK;
}

extern "C" int wap_plan_status_async(wap_plan* p, int* host_status, void* stream) {
  clear_error();
  if (!p || !host_status) return fail(WAP_ERR_ARG, "NULL argument");
  if (!p->chain_status) {
    *host_status = 0;
    return WAP_OK;
  }
  cudaError_t e = cudaMemcpyAsync(host_status, p->chain_status, sizeof(int), cudaMemcpyDeviceToHost,
                                  (cudaStream_t)stream);
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, "plan status copy");
}
