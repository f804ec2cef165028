// Convergent probe built on the device, and per-position accumulation of
// diffraction patterns.
//
// Probe (the benchmark configurations' probe model; the reference's notebooks
// build theirs on the host with abTEM's Probe(...).build(), e.g.
// wpm/cbed.ipynb): a hard aperture |f| lambda < alpha with the defocus phase
// exp(-i pi lambda df |f|^2) inside it, inverse-transformed, normalised to
// sum |psi|^2 = ny nx and, if centred, rolled to the grid centre.  In float64
// up to the spectrum; the inverse transform runs in the pass kernels.
//   1. spectrum_kernel: X = aperture * phase * (-1)^(ky + kx) when centred
//      (the fftshift of ifft2 for even sizes), counting the aperture pixels;
//   2. the inverse column and row transforms (pass kernels, unnormalised);
//   3. normalise_kernel: X / sqrt(count).  By Parseval the unnormalised
//      inverse transform of a 0/1-magnitude spectrum has norm^2 = ny nx count,
//      so this is the sqrt(ny nx) / ||ifft2(X)|| normalisation.
#include <cuda_runtime.h>

#include <cmath>

#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

struct ProbeArgs {
  int ny, nx;
  double ps_y, ps_x, lambda, alpha, defocus;
  int centred;
  float2* out;
  unsigned long long* count;
};

__global__ void __launch_bounds__(256) probe_spectrum_kernel(const ProbeArgs a) {
  const long long total = (long long)a.ny * a.nx;
  unsigned inside = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i / a.nx), x = (int)(i - (long long)y * a.nx);
    const double fy = fftfreq_d(y, a.ny, a.ps_y), fx = fftfreq_d(x, a.nx, a.ps_x);
    // f2 = fy^2 + fx^2 and the comparison in the order NumPy evaluates them
    const double f2 = __dadd_rn(__dmul_rn(fy, fy), __dmul_rn(fx, fx));
    const bool in = __dmul_rn(sqrt(f2), a.lambda) < a.alpha;
    float2 v = make_float2(0.f, 0.f);
    if (in) {
      const double ph = __dmul_rn(__dmul_rn(__dmul_rn(-M_PI, a.lambda), a.defocus), f2);
      double s, c;
      sincos(ph, &s, &c);
      const double sign = (a.centred && ((x + y) & 1)) ? -1.0 : 1.0;
      v = make_float2((float)(sign * c), (float)(sign * s));
      ++inside;
    }
    a.out[i] = v;
  }
  // one atomic per warp
  for (int o = 16; o > 0; o >>= 1) inside += __shfl_down_sync(0xffffffffu, inside, o);
  if ((threadIdx.x & 31) == 0 && inside) atomicAdd(a.count, (unsigned long long)inside);
}

__global__ void __launch_bounds__(256) probe_normalise_kernel(float2* out, long long total,
                                                               const unsigned long long* count) {
  const unsigned long long c = *count;
  const float s = c ? (float)(1.0 / sqrt((double)c)) : 0.0f;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x)
    out[i] = cscale(out[i], s);
}

// out[p] = sum over j in [start[p], start[p+1]) of dp[probes[j]], in j order
// (deterministic: no atomics), float4 at a time when the plane allows.
__global__ void __launch_bounds__(256) pattern_accumulate_kernel(const float* __restrict__ dp, int n_probes,
                                                                  long long plane, const int32_t* __restrict__ start,
                                                                  const int32_t* __restrict__ probes, int n_patterns,
                                                                  float* __restrict__ out, int* bad) {
  const bool vec = (plane & 3) == 0;
  const long long per = vec ? plane / 4 : plane;
  const long long total = (long long)n_patterns * per;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(i / per);
    const long long r = i - (long long)p * per;
    const int j0 = __ldg(start + p), j1 = __ldg(start + p + 1);
    if (vec) {
      float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
      for (int j = j0; j < j1; ++j) {
        const int b = __ldg(probes + j);
        if ((unsigned)b >= (unsigned)n_probes) {
          if (bad) *bad = 1;
          continue;
        }
        const float4 v = __ldcs(reinterpret_cast<const float4*>(dp + (long long)b * plane) + r);
        acc.x += v.x;
        acc.y += v.y;
        acc.z += v.z;
        acc.w += v.w;
      }
      reinterpret_cast<float4*>(out + (long long)p * plane)[r] = acc;
    } else {
      float acc = 0.f;
      for (int j = j0; j < j1; ++j) {
        const int b = __ldg(probes + j);
        if ((unsigned)b >= (unsigned)n_probes) {
          if (bad) *bad = 1;
          continue;
        }
        acc += __ldcs(dp + (long long)b * plane + r);
      }
      out[(long long)p * plane + r] = acc;
    }
  }
}

}  // namespace wap

using namespace wap;

extern "C" {

int wap_aperture_probe(wap_plan* p, double ps_y, double ps_x, double energy, double alpha_mrad, double defocus,
                       int centred, float* out, void* stream) {
  clear_error();
  if (!p || !out) return fail(WAP_ERR_ARG, "plan and out must be non-NULL");
  if (!(ps_y > 0) || !(ps_x > 0) || !(energy > 0)) return fail(WAP_ERR_ARG, "sampling and energy must be positive");
  if (!(alpha_mrad >= 0) || !std::isfinite(defocus)) return fail(WAP_ERR_ARG, "bad aperture or defocus");
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != p->device) return fail(WAP_ERR_ARG, "plan was created on device %d, current device is %d", p->device, dev);
  if (p->generic) return fail(WAP_ERR_UNSUPPORTED, "the probe builder needs a power-of-two grid");
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e;
  if (!p->counter && (e = cudaMalloc(&p->counter, sizeof(unsigned long long))) != cudaSuccess)
    return cuda_fail(e, "cudaMalloc(probe counter)");
  if ((e = cudaMemsetAsync(p->counter, 0, sizeof(unsigned long long), st)) != cudaSuccess)
    return cuda_fail(e, "probe counter reset");
  ProbeArgs a{p->ny, p->nx, ps_y, ps_x, physics(energy, 1.0).lambda, alpha_mrad * 1e-3, defocus, centred ? 1 : 0,
              reinterpret_cast<float2*>(out), p->counter};
  const long long total = (long long)p->ny * p->nx;
  const unsigned blocks = (unsigned)std::min<long long>((total + 255) / 256, 148LL * 8);
  count_launch();
  probe_spectrum_kernel<<<blocks, 256, 0, st>>>(a);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "probe_spectrum_kernel");
  // inverse column transform (no propagator), then inverse row transform
  ColArgs c = base_col_args(p, nullptr, nullptr);
  c.psi = reinterpret_cast<float2*>(out);
  c.psi_bstride = total;
  c.flags = COL_NO_FFT | COL_NO_H;
  c.det = Detector{0, 0, p->ny, p->nx};
  if ((e = col_chunks(p, c, 1, st)) != cudaSuccess) return cuda_fail(e, "probe column pass");
  RowArgs r{};
  r.psi = reinterpret_cast<float2*>(out);
  r.psi_bstride = total;
  r.tw = p->tw_row;
  r.ny = p->ny;
  r.nx = p->nx;
  r.flags = ROW_IFFT;
  r.scale = 1.0f;
  r.tw_ready = 1;
  if ((e = row_chunks(p, r, 1, st)) != cudaSuccess) return cuda_fail(e, "probe row pass");
  count_launch();
  probe_normalise_kernel<<<blocks, 256, 0, st>>>(reinterpret_cast<float2*>(out), total, p->counter);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "probe_normalise_kernel");
  return WAP_OK;
}

int wap_pattern_accumulate(const float* dp, int n_probes, long long plane, const int32_t* start,
                           const int32_t* probes, int n_patterns, float* out, int* bad, void* stream) {
  clear_error();
  if (!dp || !start || !probes || !out) return fail(WAP_ERR_ARG, "NULL argument");
  if (n_probes < 1 || plane < 1 || n_patterns < 1) return fail(WAP_ERR_ARG, "sizes must be positive");
  const long long total = (long long)n_patterns * ((plane & 3) == 0 ? plane / 4 : plane);
  count_launch();
  pattern_accumulate_kernel<<<(unsigned)std::min<long long>((total + 255) / 256, 148LL * 16), 256, 0,
                              (cudaStream_t)stream>>>(dp, n_probes, plane, start, probes, n_patterns, out, bad);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, "pattern_accumulate_kernel");
}

}  // extern "C"
