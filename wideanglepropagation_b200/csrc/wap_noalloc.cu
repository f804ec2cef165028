// Allocation-free Fresnel / angular-spectrum forward.
//
// Some callers cannot allocate device memory at the time they want to run a
// multislice: code that is recording a CUDA graph through a framework that
// forbids allocation calls while it captures, hosts that carve the whole GPU
// into fixed pools up front and reject any later cudaMalloc, and plugin
// interfaces that give a plugin nothing but the input and output buffers.
// For them, wap_multislice_fwd_noalloc runs the same row/column pass kernels
// as wap_multislice_fwd without a plan: the only memory those kernels need
// beyond the caller's inputs and outputs - the FFT twiddle tables of both grid
// axes - lives in a fixed array compiled into the library (kNoAllocScratchBytes
// per GPU that loads it, held until the process exits).  The tables are
// rewritten on the device by every call, so nothing needs clearing, but calls
// that overlap on the GPU (different streams, or different sizes in flight)
// share the array and race.  The transmission is evaluated per probe (no
// shared transmission table, which would need scratch proportional to the
// potential).
#include <cuda_runtime.h>

#include <mutex>

#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

// twiddle tables of the row axis (nx) and the column axis (ny): at most
// 2 x 2304 float4 entries for 2048-point transforms with 16 elements/thread
constexpr size_t kNoAllocScratchBytes = 128 * 1024;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once
// per device (the host-side name is only a stand-in for the device symbol).
int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) return fail(WAP_ERR_ARG, "device %d beyond the supported %d", dev, kMaxDevices);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
    g_noalloc_ptr[dev] = p;
  }
  *out = g_noalloc_ptr[dev];
  return WAP_OK;
}
}  // namespace

// One thread per table entry: W_{LR}^{jk} (j >= 1) of stage s >= 1 at
// tw_offset(s) + (j - 1) L + k, float64 value split into float hi + lo.
__global__ void twiddle_fill_kernel(float4* __restrict__ tw, int n, int e) {
  const PlanShape p = make_plan_shape(n, e);
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int size = p.tw_size();
  if (idx >= size) return;
  if (p.stages < 2) {
    tw[idx] = make_float4(1.f, 0.f, 0.f, 0.f);
    return;
  }
  int s = 1;
  while (s + 1 < p.stages && idx >= p.tw_offset(s + 1)) ++s;
  const int R = p.radix(s), L = p.span(s);
  const int local = idx - p.tw_offset(s);
  const int j = local / L + 1, k = local - (j - 1) * L;
  const long long LR = (long long)L * R;
  const long long m = ((long long)j * k) % LR;
  double sn, c;
  sincospi(-2.0 * (double)m / (double)LR, &sn, &c);
  const float ch = (float)c, sh = (float)sn;
  tw[idx] = make_float4(ch, sh, (float)(c - (double)ch), (float)(sn - (double)sh));
}

}  // namespace wap

using namespace wap;

extern "C" int wap_multislice_fwd_noalloc(const float* V, int n_slices, int ny, int nx, const float* psi0, int n_probes,
                                          int psi0_per_probe, const int32_t* positions, const float* H,
                                          const float* H_lo, double dz, double energy, float* exit, float* dp,
                                          float* stack, void* stream) {
  clear_error();
  if (!V || !psi0 || !H || !exit) return fail(WAP_ERR_ARG, "V, psi0, H and exit must be non-NULL device pointers");
  if (n_slices < 1) return fail(WAP_ERR_ARG, "need at least one slice (got %d)", n_slices);
  if (n_probes < 1 || n_probes > 65535 * 64) return fail(WAP_ERR_ARG, "n_probes=%d out of range", n_probes);
  if (!size_supported(ny) || !size_supported(nx))
    return fail(WAP_ERR_UNSUPPORTED, "unsupported grid %d x %d: each axis must be a power of two in [32, 2048]", ny, nx);
  const int row_e = nx >= 64 ? 16 : 8, col_e = ny >= 64 ? 16 : 8;
  const size_t row_bytes = ((make_plan_shape(nx, row_e).tw_size() * sizeof(float4)) + 255) / 256 * 256;
  const size_t col_bytes = make_plan_shape(ny, col_e).tw_size() * sizeof(float4);
  if (row_bytes + col_bytes > kNoAllocScratchBytes)
    return fail(WAP_ERR_UNSUPPORTED, "twiddle tables for %d x %d need %zu bytes, beyond the %zu-byte no-alloc scratch",
                ny, nx, row_bytes + col_bytes, kNoAllocScratchBytes);
  void* scratch = nullptr;
  int rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  float4* tw_row = reinterpret_cast<float4*>(scratch);
  float4* tw_col = reinterpret_cast<float4*>(static_cast<unsigned char*>(scratch) + row_bytes);
  cudaError_t e;
  const int nr = make_plan_shape(nx, row_e).tw_size(), nc = make_plan_shape(ny, col_e).tw_size();
  count_launch();
  twiddle_fill_kernel<<<(nr + 255) / 256, 256, 0, st>>>(tw_row, nx, row_e);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "twiddle_fill_kernel");
  count_launch();
  twiddle_fill_kernel<<<(nc + 255) / 256, 256, 0, st>>>(tw_col, ny, col_e);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "twiddle_fill_kernel");

  const Physics ph = physics(energy, dz);
  const long long plane = (long long)ny * nx;
  RowArgs r{};
  r.psi = reinterpret_cast<float2*>(exit);
  r.psi_bstride = plane;
  r.src = reinterpret_cast<const float2*>(psi0);
  r.src_bstride = psi0_per_probe ? plane : 0;
  r.shifts = positions;
  r.V = V;
  r.v_draw_stride = (long long)n_slices * plane;
  r.tw = tw_row;
  r.ny = ny;
  r.nx = nx;
  r.scale = (float)(1.0 / (double)plane);
  r.src_scale = 1.0f;
  r.ri_a = (float)ph.ri_a;
  r.ri_inv_den = (float)ph.ri_inv_den;
  r.kphase = (float)ph.kphase;
  r.e_plus_e0 = (float)ph.e_plus_e0;
  ColArgs c{};
  c.psi = r.psi;
  c.psi_bstride = plane;
  c.H = reinterpret_cast<const float2*>(H);
  c.H_lo = reinterpret_cast<const float2*>(H_lo);
  c.tw = tw_col;
  c.ny = ny;
  c.nx = nx;
  c.dp = dp;
  c.det = Detector{0, 0, ny, nx};   // the whole pattern
  int col_w = 16;
  while (col_w > 1 && (col_w * (ny / col_e) > kColThreads || (size_t)ny * col_w * 8 > 96 * 1024)) col_w >>= 1;
  if (col_w > nx) col_w = nx;
  const int rows = rows_per_cta(nx, row_e, ny);
  for (int s = 0; s <= n_slices; ++s) {
    r.slice = s;
    r.flags = (s == 0 ? ROW_LOAD_SRC : ROW_IFFT) | (s < n_slices ? (ROW_TRANS | ROW_FFT) : 0);
    r.snap = (stack && s >= 1) ? reinterpret_cast<float2*>(stack) + (long long)(s - 1) * plane : nullptr;
    r.snap_bstride = (long long)n_slices * plane;
    for (int b0 = 0; b0 < n_probes; b0 += 65535) {
      r.probe0 = b0;
      if ((e = launch_row(nx, row_e, r, std::min(65535, n_probes - b0), rows, st)) != cudaSuccess)
        return cuda_fail(e, "row pass");
    }
    if (s == n_slices) break;
    c.flags = (s == n_slices - 1 && dp) ? COL_DP : 0;
    for (int b0 = 0; b0 < n_probes; b0 += 65535) {
      c.probe0 = b0;
      if ((e = launch_col(ny, col_e, c, std::min(65535, n_probes - b0), col_w, st)) != cudaSuccess)
        return cuda_fail(e, "column pass");
    }
  }
  return WAP_OK;
}
