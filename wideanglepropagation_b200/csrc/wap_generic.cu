// Grids whose sides are not powers of two (any n in [17, 1024] per axis).
//
// The reference takes any n x m grid (get_frequencies, propagation.py:102-107,
// and jnp.fft.fft2 everywhere); its notebooks use e.g. gpts = 100
// (wpm/wpm_adaptive_comparison.ipynb).  Here a length-n DFT along such an axis
// is Bluestein's chirp convolution through the power-of-two FFT core:
//
//   X_k = w_k sum_j (x_j w_j) conj(w_{k-j}),   w_q = exp(-i pi q^2 / n),
//
// i.e. premultiply by the chirp, circular convolution of length m >= 2n - 1
// (m-point FFT, times fft_m(b) / m, inverse m-point FFT) with b_q =
// conj(w_q) for |q| < n, postmultiply by the chirp; the inverse transform uses
// the conjugate chirp.  The chirp angles pi (q^2 mod 2n) / n and fft_m(b) are
// evaluated in float64 on the host and stored as float hi + lo parts: they
// are applied identically in every slice, so a float-only table's rounding
// would add up coherently (as for the propagator H).  A power-of-two axis of
// such a grid keeps its plain FFT.
//
// Kernels mirror the power-of-two passes (wap_passes.cuh): a row kernel
// ([inverse row DFT, 1/(ny nx)] -> [snapshot] -> [* t(V)] -> [row DFT]) and a
// column kernel ([column DFT] -> [* H] -> [pattern] -> [inverse column DFT]);
// the WPM forward uses generic versions of its column (K fields) and row
// (blend) kernels.  One thread group holds the m-point vector of one row or
// column in registers (positions >= n are zero on input and ignored on
// output), so the pointwise steps chain in registers as on the fast path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

__host__ __device__ constexpr bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// length-n DFT (INV: unnormalised inverse) of the vector held as x[t + T e]
// (T = M / E threads, positions < ax.n), result in the same layout
template <int M, int E, bool INV, class X>
__device__ __forceinline__ void axis_dft(float2 (&v)[E], int t, const X& xs, const GenAxis& ax) {
  if (!ax.blue) {
    fft<M, E, INV>(v, t, xs, ax.tw);
    return;
  }
  constexpr int T = M / E;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int p = t + T * e;
    if (p < ax.n) {
      const float4 w = __ldg(ax.chirp + p);
      v[e] = INV ? cmulc_hl(v[e], make_float2(w.x, w.y), make_float2(w.z, w.w))
                 : cmul_hl(v[e], make_float2(w.x, w.y), make_float2(w.z, w.w));
    } else {
      v[e] = make_float2(0.f, 0.f);
    }
  }
  fft<M, E, false>(v, t, xs, ax.tw);
  const float4* bh = INV ? ax.bhat_i : ax.bhat_f;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const float4 b = __ldg(bh + t + T * e);
    v[e] = cmul_hl(v[e], make_float2(b.x, b.y), make_float2(b.z, b.w));
  }
  fft<M, E, true>(v, t, xs, ax.tw);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int p = t + T * e;
    if (p < ax.n) {
      const float4 w = __ldg(ax.chirp + p);
      v[e] = INV ? cmulc_hl(v[e], make_float2(w.x, w.y), make_float2(w.z, w.w))
                 : cmul_hl(v[e], make_float2(w.x, w.y), make_float2(w.z, w.w));
    }
  }
}

__device__ __forceinline__ int pmod(int a, int n) {
  const int r = a % n;
  return r < 0 ? r + n : r;
}

// fftshift position of index k on an n-point axis (numpy roll by n // 2)
__device__ __forceinline__ int shifted(int k, int n) {
  const int s = k + (n >> 1);
  return s >= n ? s - n : s;
}

struct GenRowArgs {
  float2* psi;
  long long psi_bstride;
  const float2* src;          // ROW_LOAD_SRC: initial wave(s)
  long long src_bstride;
  const int* shifts;          // (B, 2) probe centres or null
  const float* V;             // ROW_TRANS: (draws, n_slices, ny, nx) volts
  const int* draw;
  long long v_draw_stride;
  float2* snap;               // spatial wave entering `slice`, or null
  long long snap_bstride;
  GenAxis ax;                 // along x
  int ny, nx, slice, flags, probe0;
  float scale;                // after the inverse row DFT
  float ri_a, ri_inv_den, kphase;
};

template <int M, int E>
__global__ void __launch_bounds__(kRowThreads) gen_row_kernel(const GenRowArgs a) {
  constexpr int T = M / E;
  constexpr int PADN = RowExchange<true>::padded(M);
  extern __shared__ float2 gen_row_smem[];
  const int rl = threadIdx.x / T, t = threadIdx.x - rl * T;
  const int rows = blockDim.x / T;
  const int row = blockIdx.x * rows + rl;
  const bool live = row < a.ny;
  const int b = a.probe0 + blockIdx.y;
  const int nx = a.nx;
  const long long plane = (long long)a.ny * nx;
  float2* prow = a.psi + (long long)b * a.psi_bstride + (long long)row * nx;
  const RowExchange<(T <= 32)> xs{gen_row_smem + rl * PADN};
  const int f = a.flags;
  float2 v[E];
  if (f & ROW_LOAD_SRC) {
    int sy = 0, sx = 0;
    if (a.shifts) {
      sy = pmod(a.shifts[2 * b] - (a.ny >> 1), a.ny);
      sx = pmod(a.shifts[2 * b + 1] - (nx >> 1), nx);
    }
    const int srow = live ? pmod(row - sy, a.ny) : 0;
    const float2* s = a.src + (long long)b * a.src_bstride + (long long)srow * nx;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int p = t + T * e;
      v[e] = (live && p < nx) ? __ldg(s + pmod(p - sx, nx)) : make_float2(0.f, 0.f);
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int p = t + T * e;
      v[e] = (live && p < nx) ? __ldcg(prow + p) : make_float2(0.f, 0.f);
    }
  }
  if (f & ROW_IFFT) {
    axis_dft<M, E, true>(v, t, xs, a.ax);
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cscale(v[e], a.scale);
  }
  if (a.snap && live) {
    float2* sp = a.snap + (long long)b * a.snap_bstride + (long long)row * nx;
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (t + T * e < nx) __stcs(sp + t + T * e, v[e]);
  }
  if ((f & ROW_TRANS) && live) {
    const int d = a.draw ? a.draw[b] : 0;
    const float* vrow = a.V + (long long)d * a.v_draw_stride + (long long)a.slice * plane + (long long)row * nx;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int p = t + T * e;
      if (p < nx) v[e] = cmul(v[e], transmission(__ldg(vrow + p), a.ri_a, a.ri_inv_den, a.kphase));
    }
  }
  if (f & ROW_FFT) axis_dft<M, E, false>(v, t, xs, a.ax);
  if (live) {
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (t + T * e < nx) __stcg(prow + t + T * e, v[e]);
  }
}

struct GenColArgs {
  float2* psi;
  long long psi_bstride;
  const float2* H;            // (ny, nx) or null (COL_NO_H)
  const float2* H_lo;
  float* dp;                  // COL_DP: (B, det window)
  Detector det;
  GenAxis ax;                 // along y
  int ny, nx, flags, probe0;
};

// column tile [M][W] <-> global (rows < ny, columns < nx of this tile); the
// generic Fresnel / AS column kernel stages its columns this way (measured
// 3 % faster at 100^2 than per-thread loads of the live rows only)
template <int M>
__device__ __forceinline__ void gen_tile_load(float2* tile, const float2* __restrict__ g, int W, int ny, int nx,
                                              int col0) {
  for (int i = threadIdx.x; i < M * W; i += blockDim.x) {
    const int r = i / W, c = i - r * W;
    tile[i] = (r < ny && col0 + c < nx) ? __ldcg(g + (long long)r * nx + col0 + c) : make_float2(0.f, 0.f);
  }
}
template <int M>
__device__ __forceinline__ void gen_tile_store(float2* __restrict__ g, const float2* tile, int W, int ny, int nx,
                                               int col0) {
  for (int i = threadIdx.x; i < M * W; i += blockDim.x) {
    const int r = i / W, c = i - r * W;
    if (r < ny && col0 + c < nx) __stcg(g + (long long)r * nx + col0 + c, tile[i]);
  }
}

template <int M, int E>
__global__ void __launch_bounds__(kColThreads) gen_col_kernel(const GenColArgs a) {
  constexpr int T = M / E;
  const int W = blockDim.x / T;
  extern __shared__ float2 gen_col_tile[];
  const int c = threadIdx.x % W, t = threadIdx.x / W;
  const int col0 = blockIdx.x * W;
  const int col = col0 + c;
  const bool live = col < a.nx;
  const int b = a.probe0 + blockIdx.y;
  const int nx = a.nx, ny = a.ny;
  float2* base = a.psi + (long long)b * a.psi_bstride;
  const ColExchange<> xs{gen_col_tile, W, c};
  const int f = a.flags;
  gen_tile_load<M>(gen_col_tile, base, W, ny, nx, col0);
  __syncthreads();
  float2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = xs.ld(t + T * e);
  if (!(f & COL_NO_FFT)) axis_dft<M, E, false>(v, t, xs, a.ax);
  if (!(f & COL_NO_H) && live) {
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int ky = t + T * e;
      if (ky < ny) {
        const long long o = (long long)ky * nx + col;
        v[e] = a.H_lo ? cmul_hl(v[e], __ldg(a.H + o), __ldg(a.H_lo + o)) : cmul(v[e], __ldg(a.H + o));
      }
    }
  }
  if ((f & COL_DP) && live) {
    const int drx = shifted(col, nx) - a.det.x0;
    if ((unsigned)drx < (unsigned)a.det.nx) {
      float* dp = a.dp + (long long)b * a.det.plane() + drx;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int ky = t + T * e;
        const int ry = shifted(ky, ny) - a.det.y0;
        if (ky < ny && (unsigned)ry < (unsigned)a.det.ny) __stcs(dp + ry * a.det.nx, fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
      }
    }
  }
  if (!(f & COL_FWD_ONLY)) axis_dft<M, E, true>(v, t, xs, a.ax);
  __syncthreads();
#pragma unroll
  for (int e = 0; e < E; ++e) xs.st(t + T * e, v[e]);
  __syncthreads();
  gen_tile_store<M>(base, gen_col_tile, W, ny, nx, col0);
}

// ----------------------------------------------------------------------------
// WPM on generic grids: the column kernel forms the K reference fields
// (column DFT, * H_k, inverse column DFT) and the row kernel blends them (per
// bin: inverse row DFT; smoothstep weights of the bracketing bins), as
// wpm_col_kernel / wpm_row_kernel do on power-of-two grids.  H_k =
// Hvac exp(i dz a_k / (kz_k + kz_vac)) with Hvac tabulated in float64.
// ----------------------------------------------------------------------------
struct GenWpmColArgs {
  const float2* psi;          // (B, ny, nx) row-transformed wave
  float2* fields;             // (B, K, ny, nx)
  const float2* hvac;
  const float2* hvac_lo;
  const float* ky2;
  const float* kx2;
  const float* refs;          // (draws, n_slices, K)
  const int* draw;
  float* dp;                  // dp mode: |fft2|^2 (fftshifted, detector window), no fields
  Detector det;
  GenAxis ax;
  int ny, nx, K, slice, n_slices, probe0, dp_mode;
  float k02, dz;
};

template <int M, int E>
__global__ void __launch_bounds__(kColThreads) gen_wpm_col_kernel(const GenWpmColArgs a) {
  constexpr int T = M / E;
  const int W = blockDim.x / T;
  extern __shared__ float2 gen_wcol_tile[];
  float* srefs = reinterpret_cast<float*>(gen_wcol_tile + M * W);
  const int c = threadIdx.x % W, t = threadIdx.x / W;
  const int col0 = blockIdx.x * W;
  const int col = col0 + c;
  const bool live = col < a.nx;
  const int b = a.probe0 + blockIdx.y;
  const int nx = a.nx, ny = a.ny;
  const long long plane = (long long)ny * nx;
  if (!a.dp_mode) {
    const int d = a.draw ? a.draw[b] : 0;
    const float* r = a.refs + ((long long)d * a.n_slices + a.slice) * a.K;
    for (int i = threadIdx.x; i < a.K; i += blockDim.x) srefs[i] = r[i];
  }
  const ColExchange<> xs{gen_wcol_tile, W, c};
  __syncthreads();   // srefs
  // the column straight between global memory and registers (rows past ny:
  // the transform's zero padding); the tile serves the transforms only
  const float2* pin = a.psi + (long long)b * plane + col;
  float2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int r = t + T * e;
    v[e] = (live && r < ny) ? __ldcg(pin + (long long)r * nx) : make_float2(0.f, 0.f);
  }
  axis_dft<M, E, false>(v, t, xs, a.ax);
  if (a.dp_mode) {
    if (!live) return;   // no barrier follows
    const int drx = shifted(col, nx) - a.det.x0;
    if ((unsigned)drx >= (unsigned)a.det.nx) return;
    float* dp = a.dp + (long long)b * a.det.plane() + drx;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int ky = t + T * e;
      const int ry = shifted(ky, ny) - a.det.y0;
      if (ky < ny && (unsigned)ry < (unsigned)a.det.ny) __stcs(dp + ry * a.det.nx, fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
    }
    return;
  }
  float q0[E];
  const float kx2 = live ? __ldg(a.kx2 + col) : 0.f;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int ky = t + T * e;
    const bool in = live && ky < ny;
    q0[e] = in ? a.k02 - (__ldg(a.ky2 + ky) + kx2) : 1.0f;
    if (in) v[e] = cmul_hl(v[e], __ldg(a.hvac + (long long)ky * nx + col), __ldg(a.hvac_lo + (long long)ky * nx + col));
    else v[e] = make_float2(0.f, 0.f);
  }
  float2* ftile = a.fields + (long long)b * a.K * plane;
  for (int k = 0; k < a.K; ++k) {
    const float dk = srefs[k];
    const float ak = a.k02 * dk * (2.0f + dk);   // n_k^2 k0^2 - k0^2
    float2 u[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int ky = t + T * e;
      // dz (sqrt(q0 + ak) - sqrt(q0)) = dz ak / (sqrt(q0 + ak) + sqrt(q0)) on propagating pixels
      const float pr = 1.0f / q0[e];
      if (q0[e] > 0.0f && fabsf(ak * pr) <= 0.0078125f) {
        const float x = ak * pr;
        const float ph = ak * (0.5f * a.dz * sqrtf(pr)) * fmaf(x, fmaf(x, fmaf(x, -0.078125f, 0.125f), -0.25f), 1.0f);
        u[e] = cmul(v[e], cis_small(ph));
      } else if (live && ky < ny) {
        u[e] = wpm_bin_direct(v[e], pr, ak, a.dz, a.hvac + (long long)ky * nx + col);
      } else {
        u[e] = make_float2(0.f, 0.f);
      }
    }
    axis_dft<M, E, true>(u, t, xs, a.ax);
    float2* fk = ftile + (long long)k * plane + col;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int r = t + T * e;
      if (live && r < ny) __stcg(fk + (long long)r * nx, u[e]);
    }
  }
}

struct GenWpmRowArgs {
  float2* psi;                // out: row-transformed next wave
  const float2* fields;       // (B, K, ny, nx)
  float2* dpbuf;              // last slice: the row DFT of the exit wave goes here
  const float* V;
  const int* draw;
  long long v_draw_stride;
  const float* refs;
  float2* snap;
  long long snap_bstride;
  GenAxis ax;
  int ny, nx, K, slice, n_slices, probe0, last;
  float scale, ri_a, ri_inv_den;
};

template <int M, int E>
__global__ void __launch_bounds__(kRowThreads) gen_wpm_row_kernel(const GenWpmRowArgs a) {
  constexpr int T = M / E;
  constexpr int PADN = RowExchange<true>::padded(M);
  extern __shared__ float2 gen_wrow_smem[];
  const int rows = blockDim.x / T;
  float* srefs = reinterpret_cast<float*>(gen_wrow_smem + rows * PADN);
  const int b = a.probe0 + blockIdx.y;
  const int d = a.draw ? a.draw[b] : 0;
  {
    const float* r = a.refs + ((long long)d * a.n_slices + a.slice) * a.K;
    for (int i = threadIdx.x; i < a.K; i += blockDim.x) srefs[i] = r[i];
  }
  __syncthreads();
  const int rl = threadIdx.x / T, t = threadIdx.x - rl * T;
  const int row = blockIdx.x * rows + rl;
  const bool live = row < a.ny;
  const int nx = a.nx;
  const long long plane = (long long)a.ny * nx;
  const RowExchange<(T <= 32)> xs{gen_wrow_smem + rl * PADN};
  const int K = a.K;
  int il[E];
  float wr[E];
  const float* vrow = a.V + (long long)d * a.v_draw_stride + (long long)a.slice * plane + (long long)row * nx;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int p = t + T * e;
    il[e] = -2;
    wr[e] = 0.f;
    if (!live || p >= nx) continue;
    const float dn = refr_minus_one(__ldg(vrow + p), a.ri_a, a.ri_inv_den);
    // searchsorted(side='left'), clip(1, K - 1), smoothstep (propagation.py:239-249)
    int lo = 0, hi = K;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if (srefs[mid] < dn) lo = mid + 1; else hi = mid;
    }
    const int ir = min(max(lo, 1), K - 1);
    const float nl = srefs[ir - 1], nr = srefs[ir];
    const float den = nr - nl;
    float w = (dn - nl) / (den == 0.0f ? 1.0f : den);
    w = fminf(fmaxf(w, 0.0f), 1.0f);
    wr[e] = w * w * (3.0f - 2.0f * w);
    il[e] = ir - 1;
  }
  float2 acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = make_float2(0.f, 0.f);
  const float2* frow = a.fields + (long long)b * K * plane + (long long)row * nx;
  for (int k = 0; k < K; ++k) {
    float2 u[E];
    const float2* fk = frow + (long long)k * plane;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int p = t + T * e;
      u[e] = (live && p < nx) ? __ldcg(fk + p) : make_float2(0.f, 0.f);
    }
    axis_dft<M, E, true>(u, t, xs, a.ax);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const float cw = (il[e] == k) ? (1.0f - wr[e]) : ((il[e] + 1 == k) ? wr[e] : 0.0f);
      acc[e] = make_float2(fmaf(cw, u[e].x, acc[e].x), fmaf(cw, u[e].y, acc[e].y));
    }
  }
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = cscale(acc[e], a.scale);
  if (a.snap && live) {
    float2* sp = a.snap + (long long)b * a.snap_bstride + (long long)row * nx;
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (t + T * e < nx) __stcs(sp + t + T * e, acc[e]);
  }
  float2* prow = a.psi + (long long)b * plane + (long long)row * nx;
  if (a.last && live) {
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (t + T * e < nx) __stcg(prow + t + T * e, acc[e]);
  }
  axis_dft<M, E, false>(acc, t, xs, a.ax);
  float2* orow = a.last ? a.dpbuf + (long long)b * plane + (long long)row * nx : prow;
  if (live) {
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (t + T * e < nx) __stcg(orow + t + T * e, acc[e]);
  }
}

// wpm_bins_kernel for any pixel count (no float4 loads)
static __global__ void __launch_bounds__(1024) gen_wpm_bins_kernel(const WpmBinsArgs a) {
  const int s = blockIdx.x, d = blockIdx.y;
  const float* vs = a.V + ((long long)d * a.n_slices + s) * a.n_px;
  float lo = 3.0e38f, hi = -3.0e38f;
  for (int i = threadIdx.x; i < a.n_px; i += blockDim.x) {
    const float dn = refr_minus_one(__ldg(vs + i), a.ri_a, a.ri_inv_den);
    lo = fminf(lo, dn);
    hi = fmaxf(hi, dn);
  }
  __shared__ float slo[32], shi[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    slo[w] = lo;
    shi[w] = hi;
  }
  __syncthreads();
  if (w == 0) {
    const int nw = blockDim.x >> 5;
    lo = l < nw ? slo[l] : 3.0e38f;
    hi = l < nw ? shi[l] : -3.0e38f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    float* out = a.refs + ((long long)d * a.n_slices + s) * a.K;
    const double dlo = lo, dhi = hi;
    for (int k = l; k < a.K; k += 32) {
      const double tk = (k == a.K - 1) ? 1.0 : (double)k * (1.0 / (double)(a.K - 1));
      const double tp = (a.power == 1.0) ? tk : pow(tk, a.power);
      out[k] = (float)(dlo + (dhi - dlo) * tp);
    }
  }
}

// ----------------------------------------------------------------------------
// launches: one instance per transform size m (E = 8 up to 128 points, else 16)
// ----------------------------------------------------------------------------
__host__ __device__ constexpr int gen_e(int m) { return m <= 128 ? 8 : 16; }

template <class K>
static cudaError_t set_smem(K kern, size_t smem) {
  return smem > 48 * 1024 ? cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                          : cudaSuccess;
}

static int gen_rows(int m) { return std::max(1, kRowThreads / (m / gen_e(m))); }
static int gen_cols(int m) { return std::max(1, std::min(16, kColThreads / (m / gen_e(m)))); }

template <int M>
static cudaError_t launch_gen_row_t(const GenRowArgs& a, int nb, cudaStream_t st) {
  constexpr int E = gen_e(M), T = M / E;
  const int rows = gen_rows(M);
  const size_t smem = (size_t)rows * RowExchange<true>::padded(M) * sizeof(float2);
  cudaError_t e = set_smem(gen_row_kernel<M, E>, smem);
  if (e != cudaSuccess) return e;
  count_launch();
  gen_row_kernel<M, E><<<dim3((a.ny + rows - 1) / rows, nb), rows * T, smem, st>>>(a);
  return cudaGetLastError();
}

template <int M>
static cudaError_t launch_gen_col_t(const GenColArgs& a, int nb, cudaStream_t st) {
  constexpr int E = gen_e(M), T = M / E;
  const int w = gen_cols(M);
  const size_t smem = (size_t)M * w * sizeof(float2);
  cudaError_t e = set_smem(gen_col_kernel<M, E>, smem);
  if (e != cudaSuccess) return e;
  count_launch();
  gen_col_kernel<M, E><<<dim3((a.nx + w - 1) / w, nb), w * T, smem, st>>>(a);
  return cudaGetLastError();
}

template <int M>
static cudaError_t launch_gen_wcol_t(const GenWpmColArgs& a, int nb, cudaStream_t st) {
  constexpr int E = gen_e(M), T = M / E;
  const int w = gen_cols(M);
  const size_t smem = (size_t)M * w * sizeof(float2) + (size_t)a.K * sizeof(float);
  cudaError_t e = set_smem(gen_wpm_col_kernel<M, E>, smem);
  if (e != cudaSuccess) return e;
  count_launch();
  gen_wpm_col_kernel<M, E><<<dim3((a.nx + w - 1) / w, nb), w * T, smem, st>>>(a);
  return cudaGetLastError();
}

template <int M>
static cudaError_t launch_gen_wrow_t(const GenWpmRowArgs& a, int nb, cudaStream_t st) {
  constexpr int E = gen_e(M), T = M / E;
  const int rows = gen_rows(M);
  const size_t smem = (size_t)rows * RowExchange<true>::padded(M) * sizeof(float2) + (size_t)a.K * sizeof(float);
  cudaError_t e = set_smem(gen_wpm_row_kernel<M, E>, smem);
  if (e != cudaSuccess) return e;
  count_launch();
  gen_wpm_row_kernel<M, E><<<dim3((a.ny + rows - 1) / rows, nb), rows * T, smem, st>>>(a);
  return cudaGetLastError();
}

#define WAP_GEN_SIZES(M) M(32) M(64) M(128) M(256) M(512) M(1024) M(2048)
#define WAP_GEN_DISPATCH(FN, m)                               \
  do {                                                        \
    switch (m) {                                              \
      WAP_GEN_SIZES(FN)                                       \
      default: return cudaErrorInvalidValue;                  \
    }                                                         \
  } while (0)
#define WAP_GEN_ROW(M) case M: return launch_gen_row_t<M>(a, nb, st);
#define WAP_GEN_COL(M) case M: return launch_gen_col_t<M>(a, nb, st);
#define WAP_GEN_WCOL(M) case M: return launch_gen_wcol_t<M>(a, nb, st);
#define WAP_GEN_WROW(M) case M: return launch_gen_wrow_t<M>(a, nb, st);

static cudaError_t launch_gen_row(const GenRowArgs& a, int nb, cudaStream_t st) { WAP_GEN_DISPATCH(WAP_GEN_ROW, a.ax.m); }
static cudaError_t launch_gen_col(const GenColArgs& a, int nb, cudaStream_t st) { WAP_GEN_DISPATCH(WAP_GEN_COL, a.ax.m); }
static cudaError_t launch_gen_wcol(const GenWpmColArgs& a, int nb, cudaStream_t st) {
  WAP_GEN_DISPATCH(WAP_GEN_WCOL, a.ax.m);
}
static cudaError_t launch_gen_wrow(const GenWpmRowArgs& a, int nb, cudaStream_t st) {
  WAP_GEN_DISPATCH(WAP_GEN_WROW, a.ax.m);
}

// ----------------------------------------------------------------------------
// host: axis tables
// ----------------------------------------------------------------------------
bool generic_size_supported(int n) { return n >= 17 && n <= 1024; }

// in-place iterative radix-2 FFT in float64 (host; table set-up only)
static void host_fft(std::vector<std::complex<double>>& a) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; ++k) {
        const double ang = -2.0 * M_PI * (double)k / (double)len;
        const std::complex<double> w(std::cos(ang), std::sin(ang));
        const std::complex<double> u = a[i + k], v = a[i + k + len / 2] * w;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
  }
}

static float4 split(std::complex<double> z) {
  const float rh = (float)z.real(), ih = (float)z.imag();
  return make_float4(rh, ih, (float)(z.real() - (double)rh), (float)(z.imag() - (double)ih));
}

template <class T>
static int upload_vec(const T** dst, const std::vector<T>& v) {
  T* d = nullptr;
  cudaError_t e = cudaMalloc(&d, v.size() * sizeof(T));
  if (e == cudaSuccess) e = cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return cuda_fail(e, "generic-axis table upload");
  }
  *dst = d;
  return WAP_OK;
}

int generic_axis_create(GenAxis* ax, int n) {
  *ax = GenAxis{};
  ax->n = n;
  ax->blue = is_pow2(n) ? 0 : 1;
  int m = n;
  if (ax->blue) {
    m = 1;
    while (m < 2 * n - 1) m <<= 1;
  }
  ax->m = m;
  ax->e = gen_e(m);
  int rc = upload_vec(&ax->tw, twiddle_table(m, ax->e));
  if (rc || !ax->blue) return rc;
  // chirp w_q = exp(-i pi q^2 / n) with q^2 reduced mod 2n (exact integers)
  std::vector<float4> chirp(n);
  std::vector<std::complex<double>> bq(m, 0.0);
  for (int q = 0; q < n; ++q) {
    const long long r = ((long long)q * q) % (2LL * n);
    const double ang = M_PI * (double)r / (double)n;
    const std::complex<double> w(std::cos(ang), -std::sin(ang));
    chirp[q] = split(w);
    bq[q] = std::conj(w);
    if (q > 0) bq[m - q] = std::conj(w);
  }
  std::vector<std::complex<double>> bf = bq, bi(m);
  for (int i = 0; i < m; ++i) bi[i] = std::conj(bq[i]);
  host_fft(bf);
  host_fft(bi);
  std::vector<float4> hf(m), hi(m);
  for (int i = 0; i < m; ++i) {
    hf[i] = split(bf[i] / (double)m);
    hi[i] = split(bi[i] / (double)m);
  }
  if ((rc = upload_vec(&ax->chirp, chirp)) || (rc = upload_vec(&ax->bhat_f, hf)) || (rc = upload_vec(&ax->bhat_i, hi)))
    return rc;
  return WAP_OK;
}

void generic_axis_free(GenAxis* ax) {
  cudaFree(const_cast<float4*>(ax->tw));
  cudaFree(const_cast<float4*>(ax->chirp));
  cudaFree(const_cast<float4*>(ax->bhat_f));
  cudaFree(const_cast<float4*>(ax->bhat_i));
  *ax = GenAxis{};
}

// ----------------------------------------------------------------------------
// forward drivers
// ----------------------------------------------------------------------------
int generic_fresnel_forward(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw,
                            const float* psi0, int n_probes, int psi0_per_probe, const int32_t* positions,
                            const float* H, const float* H_lo, double dz, double energy, float* exit, float* dp,
                            float* stack, cudaStream_t st) {
  const Physics ph = physics(energy, dz);
  const long long plane = (long long)p->ny * p->nx;
  GenRowArgs r{};
  r.psi = reinterpret_cast<float2*>(exit);
  r.psi_bstride = plane;
  r.src = reinterpret_cast<const float2*>(psi0);
  r.src_bstride = psi0_per_probe ? plane : 0;
  r.shifts = positions;
  r.V = V;
  r.draw = draw;
  r.v_draw_stride = (long long)n_slices * plane;
  r.ax = p->gen_x;
  r.ny = p->ny;
  r.nx = p->nx;
  r.scale = (float)(1.0 / (double)plane);
  r.ri_a = (float)ph.ri_a;
  r.ri_inv_den = (float)ph.ri_inv_den;
  r.kphase = (float)ph.kphase;
  GenColArgs c{};
  c.psi = r.psi;
  c.psi_bstride = plane;
  c.H = reinterpret_cast<const float2*>(H);
  c.H_lo = reinterpret_cast<const float2*>(H_lo);
  c.dp = dp;
  c.det = p->det.resolved(p->ny, p->nx);
  c.ax = p->gen_y;
  c.ny = p->ny;
  c.nx = p->nx;
  cudaError_t e;
  for (int b0 = 0; b0 < n_probes; b0 += 65535) {
    const int nb = std::min(65535, n_probes - b0);
    r.probe0 = c.probe0 = b0;
    for (int s = 0; s <= n_slices; ++s) {
      r.slice = s;
      r.flags = (s == 0 ? ROW_LOAD_SRC : ROW_IFFT) | (s < n_slices ? (ROW_TRANS | ROW_FFT) : 0);
      r.snap = nullptr;
      if (stack && s >= 1) {
        r.snap = reinterpret_cast<float2*>(stack) + (long long)(s - 1) * plane;
        r.snap_bstride = (long long)n_slices * plane;
      }
      if ((e = launch_gen_row(r, nb, st)) != cudaSuccess) return cuda_fail(e, "generic row pass");
      if (s == n_slices) break;
      c.flags = (s == n_slices - 1 && dp) ? COL_DP : 0;
      if ((e = launch_gen_col(c, nb, st)) != cudaSuccess) return cuda_fail(e, "generic column pass");
    }
  }
  return WAP_OK;
}

int generic_wpm_forward(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw,
                        const float* psi0, int n_probes, int psi0_per_probe, const int32_t* positions, double dz,
                        double energy, double sampling_y, double sampling_x, double power_spacing, float* exit,
                        float* dp, float* stack, cudaStream_t st) {
  const Physics ph = physics(energy, dz);
  const int K = p->n_bins;
  const long long plane = (long long)p->ny * p->nx;
  cudaError_t e;
  WpmBinsArgs bargs{V, p->refs, (int)plane, n_slices, K, (float)ph.ri_a, (float)ph.ri_inv_den, power_spacing};
  count_launch();
  gen_wpm_bins_kernel<<<dim3(n_slices, n_draws), 1024, 0, st>>>(bargs);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "generic wpm bins");
  GenRowArgs r{};
  r.psi = reinterpret_cast<float2*>(exit);
  r.psi_bstride = plane;
  r.src = reinterpret_cast<const float2*>(psi0);
  r.src_bstride = psi0_per_probe ? plane : 0;
  r.shifts = positions;
  r.ax = p->gen_x;
  r.ny = p->ny;
  r.nx = p->nx;
  r.flags = ROW_LOAD_SRC | ROW_FFT;
  GenWpmColArgs c{};
  c.psi = reinterpret_cast<const float2*>(exit);
  c.fields = p->fields;
  c.hvac = p->hvac;
  c.hvac_lo = p->hvac_lo;
  c.ky2 = p->ky2;
  c.kx2 = p->kx2;
  c.refs = p->refs;
  c.draw = draw;
  c.det = p->det.resolved(p->ny, p->nx);
  c.ax = p->gen_y;
  c.ny = p->ny;
  c.nx = p->nx;
  c.K = K;
  c.n_slices = n_slices;
  c.k02 = (float)(ph.k0 * ph.k0);
  c.dz = (float)dz;
  GenWpmRowArgs w{};
  w.psi = reinterpret_cast<float2*>(exit);
  w.fields = p->fields;
  w.dpbuf = p->dpbuf;
  w.V = V;
  w.draw = draw;
  w.v_draw_stride = (long long)n_slices * plane;
  w.refs = p->refs;
  w.ax = p->gen_x;
  w.ny = p->ny;
  w.nx = p->nx;
  w.K = K;
  w.n_slices = n_slices;
  w.scale = (float)(1.0 / (double)plane);
  w.ri_a = (float)ph.ri_a;
  w.ri_inv_den = (float)ph.ri_inv_den;
  w.snap_bstride = (long long)n_slices * plane;
  for (int b0 = 0; b0 < n_probes; b0 += 65535) {
    const int nb = std::min(65535, n_probes - b0);
    r.probe0 = c.probe0 = w.probe0 = b0;
    if ((e = launch_gen_row(r, nb, st)) != cudaSuccess) return cuda_fail(e, "generic wpm row pass");
    for (int s = 0; s < n_slices; ++s) {
      c.slice = s;
      c.dp_mode = 0;
      if ((e = launch_gen_wcol(c, nb, st)) != cudaSuccess) return cuda_fail(e, "generic wpm column pass");
      w.slice = s;
      w.last = (s == n_slices - 1);
      w.snap = stack ? reinterpret_cast<float2*>(stack) + (long long)s * plane : nullptr;
      if ((e = launch_gen_wrow(w, nb, st)) != cudaSuccess) return cuda_fail(e, "generic wpm row pass");
    }
    if (dp) {
      GenWpmColArgs d = c;
      d.psi = p->dpbuf;
      d.dp = dp;
      d.dp_mode = 1;
      if ((e = launch_gen_wcol(d, nb, st)) != cudaSuccess) return cuda_fail(e, "generic wpm pattern pass");
    }
  }
  return WAP_OK;
}

}  // namespace wap
