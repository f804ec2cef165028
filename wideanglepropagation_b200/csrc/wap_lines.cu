// 1D line helpers and the naive per-pixel WPM step.
//
//   wap_line_transfer     fresnel_kernel_1d / angular_spectrum_kernel_1d
//                         (propagation.py:617-626), float64
//   wap_line_propagate    propagate_1d: ifft(fft(psi) H) per line
//                         (propagation.py:629-633) on the radix-16 core
//   wap_line_wpm          wpm_kernel_1d(_vmap): ifft(psi_k exp(i dy kz(n_k)))
//                         for K refractive indices (propagation.py:636-652),
//                         the transfer function evaluated in float64
//   wap_wpm_naive_step    wpm_step (propagation.py:184-212): pixel p takes
//                         pixel p of ifft2(fft2(wave) H(n_p)); evaluated as
//                         direct float64 sums (a small-grid exactness check
//                         for the binned WPM)
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <utility>

#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

constexpr int kLineThreads = 256;
constexpr int kLineE = 16;

struct LineArgs {
  const float2* in;          // propagate: (n_lines, n); wpm: one spectral line (n)
  float2* out;               // (n_lines, n)
  int n_lines;
  int mode;                  // 0: propagate, 1: wpm
  const float2* H;           // propagate: transfer function hi part
  const float2* H_lo;        //   and lo part (or null)
  long long h_stride;        //   0: one H for every line, n: one per line
  const double* n_vals;      // wpm: refractive index of each line
  const double* kx_sq;       // wpm: (n) kx^2
  double k0, dy;
  const float4* tw;
};

// float64 value split into float hi + lo
__device__ __forceinline__ void split_c(double re, double im, float2& hi, float2& lo) {
  hi = make_float2((float)re, (float)im);
  lo = make_float2((float)(re - (double)hi.x), (float)(im - (double)hi.y));
}

// exp(i dy sqrt(q)) with the principal complex square root of the real q
// (q < 0: sqrt(q) = i sqrt(-q), an evanescent decay exp(-dy sqrt(-q)))
__device__ __forceinline__ void exp_i_dy_sqrt(double q, double dy, double& re, double& im) {
  if (q >= 0.0) {
    sincos(dy * sqrt(q), &im, &re);
  } else {
    re = exp(-dy * sqrt(-q));
    im = 0.0;
  }
}

template <int N>
__global__ void __launch_bounds__(kLineThreads) line_kernel(const LineArgs a) {
  using P = FFTPlan<N, kLineE>;
  constexpr int E = kLineE;
  constexpr int T = P::T;
  constexpr int PADN = RowExchange<true>::padded(N);
  const int rows = blockDim.x / T;
  extern __shared__ float4 line_smem[];
  float4* tw = line_smem;
  float2* xbuf = reinterpret_cast<float2*>(tw + P::TW_SIZE);
  for (int i = threadIdx.x; i < P::TW_SIZE; i += blockDim.x) tw[i] = a.tw[i];
  __syncthreads();
  const int rl = threadIdx.x / T, t = threadIdx.x - rl * T;
  const int line = blockIdx.x * rows + rl;
  const bool live = line < a.n_lines;
  const int src = a.mode == 0 ? (live ? line : a.n_lines - 1) : 0;   // idle rows still join the barriers
  const RowExchange<(T <= 32)> xs{xbuf + rl * PADN};

  float2 v[E];
  const float2* in = a.in + (long long)src * N;
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = __ldg(in + t + T * e);
  if (a.mode == 0) {
    fft<N, E, false>(v, t, xs, tw);
    const float2* h = a.H + (long long)src * a.h_stride;
    const float2* hl = a.H_lo ? a.H_lo + (long long)src * a.h_stride : nullptr;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int x = t + T * e;
      v[e] = hl ? cmul_hl(v[e], __ldg(h + x), __ldg(hl + x)) : cmul(v[e], __ldg(h + x));
    }
  } else {
    const double nk = a.n_vals[live ? line : a.n_lines - 1] * a.k0;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int x = t + T * e;
      double re, im;
      exp_i_dy_sqrt(nk * nk - a.kx_sq[x], a.dy, re, im);
      float2 hi, lo;
      split_c(re, im, hi, lo);
      v[e] = cmul_hl(v[e], hi, lo);
    }
  }
  fft<N, E, true>(v, t, xs, tw);
  if (!live) return;
  float2* out = a.out + (long long)line * N;
  const float s = 1.0f / (float)N;   // numpy ifft normalisation (a power of two: exact)
#pragma unroll
  for (int e = 0; e < E; ++e) out[t + T * e] = cscale(v[e], s);
}

template <int N>
static cudaError_t launch_line_t(const LineArgs& a, cudaStream_t st) {
  constexpr int T = N / kLineE;
  const int rows = kLineThreads / T;
  const size_t smem = (size_t)rows * RowExchange<true>::padded(N) * sizeof(float2) +
                      FFTPlan<N, kLineE>::TW_SIZE * sizeof(float4);
  cudaError_t e = cudaFuncSetAttribute(line_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  count_launch();
  line_kernel<N><<<(a.n_lines + rows - 1) / rows, rows * T, smem, st>>>(a);
  return cudaGetLastError();
}

static cudaError_t launch_line(int n, const LineArgs& a, cudaStream_t st) {
  switch (n) {
    case 32: return launch_line_t<32>(a, st);
    case 64: return launch_line_t<64>(a, st);
    case 128: return launch_line_t<128>(a, st);
    case 256: return launch_line_t<256>(a, st);
    case 512: return launch_line_t<512>(a, st);
    case 1024: return launch_line_t<1024>(a, st);
    case 2048: return launch_line_t<2048>(a, st);
    default: return cudaErrorInvalidValue;
  }
}

// Twiddles of the n-point line transforms, uploaded once per (device, n) and
// kept for the life of the process.
static int line_twiddles(int n, const float4** out) {
  static std::mutex mu;
  static std::map<std::pair<int, int>, float4*> cache;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find({dev, n});
  if (it != cache.end()) {
    *out = it->second;
    return WAP_OK;
  }
  std::vector<float4> h = twiddle_table(n, kLineE);
  float4* d = nullptr;
  if ((e = cudaMalloc(&d, h.size() * sizeof(float4))) != cudaSuccess) return cuda_fail(e, "cudaMalloc(line twiddles)");
  if ((e = cudaMemcpy(d, h.data(), h.size() * sizeof(float4), cudaMemcpyHostToDevice)) != cudaSuccess) {
    cudaFree(d);
    return cuda_fail(e, "cudaMemcpy(line twiddles)");
  }
  cache[{dev, n}] = d;
  *out = d;
  return WAP_OK;
}

// ---------------------------------------------------------------------------
// 1D transfer functions, float64 (propagation.py:617-626)
// ---------------------------------------------------------------------------
__global__ void line_transfer_kernel(int kind, int n, const double* __restrict__ kx_sq, double k0, double dy,
                                     double2* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double re, im;
  if (kind == WAP_TF_FRESNEL) {
    sincos(-kx_sq[i] * dy / (2.0 * k0), &im, &re);
  } else {
    exp_i_dy_sqrt(k0 * k0 - kx_sq[i], dy, re, im);
  }
  out[i] = make_double2(re, im);
}

// ---------------------------------------------------------------------------
// naive WPM step (propagation.py:184-212) as direct float64 sums
// ---------------------------------------------------------------------------
// exp(i 2 pi m / n) for an integer phase m in [0, n)
__device__ __forceinline__ double2 unit_root(long long m, int n) {
  double s, c;
  sincospi(2.0 * (double)m / (double)n, &s, &c);
  return make_double2(c, s);
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// A[i][kx] = sum_x w[i][x] exp(-2 pi i kx x / nx)   (one output per thread)
__global__ void naive_dft_rows(const double2* __restrict__ w, double2* __restrict__ A, int ny, int nx) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
  if (kx >= nx) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int x = 0; x < nx; ++x) {
    const double2 r = unit_root((nx - ((long long)kx * x) % nx) % nx, nx);
    const double2 z = zmul(w[(long long)i * nx + x], r);
    acc.x += z.x;
    acc.y += z.y;
  }
  A[(long long)i * nx + kx] = acc;
}

// Ek[ky][kx] = sum_y A[y][kx] exp(-2 pi i ky y / ny)
__global__ void naive_dft_cols(const double2* __restrict__ A, double2* __restrict__ Ek, int ny, int nx) {
  const int kx = blockIdx.x * blockDim.x + threadIdx.x, ky = blockIdx.y;
  if (kx >= nx) return;
  double2 acc = make_double2(0.0, 0.0);
  for (int y = 0; y < ny; ++y) {
    const double2 r = unit_root((ny - ((long long)ky * y) % ny) % ny, ny);
    const double2 z = zmul(A[(long long)y * nx + kx], r);
    acc.x += z.x;
    acc.y += z.y;
  }
  Ek[(long long)ky * nx + kx] = acc;
}

// out[p] = (1/P) sum_k Ek[k] exp(i dz sqrt((n_p k0)^2 - k_perp^2[k])) exp(2 pi i (ky y/ny + kx x/nx)),
// one CTA per output pixel, k_perp^2 = (2 pi fftfreq(ny, ps0)[ky])^2 + (2 pi fftfreq(nx, ps1)[kx])^2
constexpr int kNaiveThreads = 256;
__global__ void __launch_bounds__(kNaiveThreads) naive_wpm_out(const double2* __restrict__ Ek,
                                                               const double* __restrict__ n_map, int ny, int nx,
                                                               double dz, double k0, double ps0, double ps1,
                                                               double2* __restrict__ out) {
  const int p = blockIdx.x;
  const int y = p / nx, x = p - y * nx;
  const double nk = n_map[p] * k0;
  const long long P = (long long)ny * nx;
  double2 acc = make_double2(0.0, 0.0);
  for (long long k = threadIdx.x; k < P; k += blockDim.x) {
    const int ky = (int)(k / nx), kx = (int)(k - (long long)ky * nx);
    const double fy = fftfreq_d(ky, ny, ps0), fx = fftfreq_d(kx, nx, ps1);
    const double kp2 = (2.0 * M_PI * fy) * (2.0 * M_PI * fy) + (2.0 * M_PI * fx) * (2.0 * M_PI * fx);
    double hre, him;
    exp_i_dy_sqrt(nk * nk - kp2, dz, hre, him);
    // exp(2 pi i (ky y / ny + kx x / nx)) from the two exact integer phases
    const double2 ry = unit_root(((long long)ky * y) % ny, ny);
    const double2 rx = unit_root(((long long)kx * x) % nx, nx);
    const double2 z = zmul(zmul(Ek[k], make_double2(hre, him)), zmul(ry, rx));
    acc.x += z.x;
    acc.y += z.y;
  }
  __shared__ double2 red[kNaiveThreads];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = kNaiveThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[threadIdx.x].x += red[threadIdx.x + s].x;
      red[threadIdx.x].y += red[threadIdx.x + s].y;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) out[p] = make_double2(red[0].x / (double)P, red[0].y / (double)P);
}

}  // namespace wap

using namespace wap;

extern "C" {

int wap_line_transfer(int kind, int n, const double* kx_sq, double k0, double dy, double* out, void* stream) {
  clear_error();
  if (!kx_sq || !out) return fail(WAP_ERR_ARG, "kx_sq and out must be non-NULL device pointers");
  if (kind != WAP_TF_FRESNEL && kind != WAP_TF_ANGULAR) return fail(WAP_ERR_ARG, "unknown transfer function %d", kind);
  if (n < 1) return fail(WAP_ERR_ARG, "n must be positive (got %d)", n);
  if (!(k0 > 0)) return fail(WAP_ERR_ARG, "k0 must be positive");
  count_launch();
  line_transfer_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(kind, n, kx_sq, k0, dy,
                                                                         reinterpret_cast<double2*>(out));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, "line_transfer_kernel");
}

int wap_line_propagate(int n, int n_lines, const float* psi, const float* H, const float* H_lo, int h_per_line,
                       float* out, void* stream) {
  clear_error();
  if (!psi || !H || !out) return fail(WAP_ERR_ARG, "psi, H and out must be non-NULL device pointers");
  if (!size_supported(n)) return fail(WAP_ERR_UNSUPPORTED, "line length %d: must be a power of two in [32, 2048]", n);
  if (n_lines < 1 || n_lines > (1 << 24)) return fail(WAP_ERR_ARG, "n_lines=%d out of range", n_lines);
  LineArgs a{};
  if (int rc = line_twiddles(n, &a.tw)) return rc;
  a.in = reinterpret_cast<const float2*>(psi);
  a.out = reinterpret_cast<float2*>(out);
  a.n_lines = n_lines;
  a.mode = 0;
  a.H = reinterpret_cast<const float2*>(H);
  a.H_lo = reinterpret_cast<const float2*>(H_lo);
  a.h_stride = h_per_line ? n : 0;
  cudaError_t e = launch_line(n, a, (cudaStream_t)stream);
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, "line_kernel (propagate)");
}

int wap_line_wpm(int n, int n_refs, const float* psi_k, const double* n_vals, double k0, const double* kx_sq,
                 double dy, float* out, void* stream) {
  clear_error();
  if (!psi_k || !n_vals || !kx_sq || !out) return fail(WAP_ERR_ARG, "NULL device pointer");
  if (!size_supported(n)) return fail(WAP_ERR_UNSUPPORTED, "line length %d: must be a power of two in [32, 2048]", n);
  if (n_refs < 1 || n_refs > (1 << 24)) return fail(WAP_ERR_ARG, "n_refs=%d out of range", n_refs);
  LineArgs a{};
  if (int rc = line_twiddles(n, &a.tw)) return rc;
  a.in = reinterpret_cast<const float2*>(psi_k);
  a.out = reinterpret_cast<float2*>(out);
  a.n_lines = n_refs;
  a.mode = 1;
  a.n_vals = n_vals;
  a.kx_sq = kx_sq;
  a.k0 = k0;
  a.dy = dy;
  cudaError_t e = launch_line(n, a, (cudaStream_t)stream);
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, "line_kernel (wpm)");
}

int wap_wpm_naive_step(int ny, int nx, const double* wave, const double* n_map, double dz, double energy, double ps0,
                       double ps1, double* out, double* work, void* stream) {
  clear_error();
  if (!wave || !n_map || !out || !work) return fail(WAP_ERR_ARG, "NULL device pointer");
  if (ny < 1 || nx < 1 || (long long)ny * nx > 65536)
    return fail(WAP_ERR_UNSUPPORTED, "naive WPM step on %d x %d: at most 65536 pixels (direct O(P^2) sums)", ny, nx);
  if (!(energy > 0) || !(ps0 > 0) || !(ps1 > 0)) return fail(WAP_ERR_ARG, "energy and sampling must be positive");
  const Physics ph = physics(energy, dz);
  cudaStream_t st = (cudaStream_t)stream;
  const long long P = (long long)ny * nx;
  double2* A = reinterpret_cast<double2*>(work);
  double2* Ek = A + P;
  const dim3 g((nx + 127) / 128, ny);
  count_launch();
  naive_dft_rows<<<g, 128, 0, st>>>(reinterpret_cast<const double2*>(wave), A, ny, nx);
  count_launch();
  naive_dft_cols<<<g, 128, 0, st>>>(A, Ek, ny, nx);
  count_launch();
  naive_wpm_out<<<(unsigned)P, kNaiveThreads, 0, st>>>(Ek, n_map, ny, nx, dz, ph.k0, ps0, ps1,
                                                       reinterpret_cast<double2*>(out));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? WAP_OK : cuda_fail(e, "naive WPM step");
}

}  // extern "C"
