// Multislice passes built on the register/shared-memory FFT core.
//
// A slice step psi <- ifft2(H * fft2(psi * t_s)) (propagation.py:331-342) is
// split into two passes over the wave, both in place on one (B, ny, nx)
// complex64 buffer:
//
//   row pass  s : [inverse row FFT of slice s-1's result, * 1/(ny nx),
//                  optional snapshot store] -> * t_s -> forward row FFT
//   col pass  s : forward column FFT -> * H -> [dp = |.|^2 on the last
//                  slice] -> inverse column FFT
//
// so the inverse row transform of slice s-1 and the forward row transform of
// slice s share one read and one write of the wave.  The last row pass only
// finishes the inverse transform (exit wave).  fft2(exit) equals the product
// H * fft2(psi * t) the last column pass already holds, so the diffraction
// pattern |fftshift(fft2(exit))|^2 (propagation.py:346-350) is written there
// without another transform.
//
// Thread layout.  Row pass: T = nx/E threads per row, ROWS rows per CTA; thread
// t of a row reads x[t + T e], i.e. a half-warp (T = 16) reads 128 contiguous
// bytes per access.  Column pass: W columns per CTA, lanes run along the
// columns (W consecutive complex64 = 8 W contiguous bytes per row), T = ny/E
// threads per column, the tile is exchanged through shared memory.
//
// The WPM passes (propagation.py:215-256) and the adjoint passes reuse the
// same skeleton; see the comments at each kernel.
#pragma once
#include "wap_fft.cuh"

namespace wap {

// launch-bound ceilings: row-type CTAs hold rows * (nx / E) <= 256 threads,
// column-type CTAs W * (ny / E) <= 512 threads
constexpr int kRowThreads = 256;
constexpr int kColThreads = 512;

enum RowFlags : int {
  ROW_LOAD_SRC = 1,   // read the initial probe (shifted) instead of psi
  ROW_IFFT = 2,       // inverse row FFT first (finishes the previous slice)
  ROW_TRANS = 4,      // multiply by the transmission function of `slice`
  ROW_FFT = 8,        // forward row FFT last
  ROW_ADJOINT = 16,   // adjoint: gradient accumulation + conj(t)
  ROW_SCALE_SRC = 32, // multiply the loaded source by src_scale (adjoint seed)
  ROW_TRANS_TAB = 64, // multiply by the precomputed transmission table ttab
};

enum ColFlags : int {
  COL_CONJ_H = 1,     // multiply by conj(H) (adjoint propagator)
  COL_DP = 2,         // write |H X|^2 (fftshifted) into dp
  COL_SEED = 4,       // adjoint seed: X <- n_px g X (+ fft of second buffer)
  COL_NO_H = 8,       // skip the propagator (pure 2D FFT epilogue)
  COL_NO_FFT = 16,    // the tile is already a spectrum along y: no forward column FFT
  COL_FWD_ONLY = 32,  // store the spectrum after the forward FFT (and H): no inverse FFT
};

struct RowArgs {
  float2* psi;               // (B, ny, nx) in/out
  long long psi_bstride;     // elements between probes in psi
  const float2* src;         // ROW_LOAD_SRC: initial wave(s)
  long long src_bstride;     // 0: one shared probe for every batch entry
  const int* shifts;         // (B, 2) probe centres (row, col), or null
  const float* V;            // (draws, n_slices, ny, nx) volts
  const int* draw;           // (B) potential draw per probe, or null
  long long v_draw_stride;   // n_slices * ny * nx
  const float4* tw;          // twiddle table for nx (hi, lo)
  float2* snap;              // snapshot of the spatial wave entering `slice`
  long long snap_bstride;    //   (after the load / inverse FFT), or null
  const float2* aux;         // ROW_ADJOINT: forward wave psi_s entering slice s
  long long aux_bstride;
  float* grad;               // ROW_ADJOINT: dL/dV, laid out like V, accumulated
  const float2* ttab;        // ROW_TRANS_TAB: exp(i phi(V)) laid out like V
  int ny, nx;
  int slice;
  int flags;
  int probe0;                // batch offset of this launch
  float scale;               // applied after the inverse row FFT
  float src_scale;
  float ri_a, ri_inv_den;    // n^2 - 1 = V (a + V) inv_den
  float kphase;              // 2 pi dz / lambda
  float e_plus_e0;           // E + E0 (for dn/dV)
  int tw_ready;              // tw was not written by a kernel of this stream (a plan's
                             // table): read before the programmatic-launch wait
};

struct ColArgs {
  float2* psi;
  long long psi_bstride;
  const float2* H;           // (ny, nx)
  const float2* H_lo;        // (ny, nx) H - H rounded to complex64, or null
  const float4* tw;          // twiddle table for ny (hi, lo)
  float* dp;                 // COL_DP: (B, det window) or (B, ny, nx)
  const float* g;            // COL_SEED: dL/ddp laid out like dp (zero outside the window)
  Detector det;              // diffraction-pattern window of dp / g
  const float2* seed2;       // COL_SEED: optional row-transformed lambda_exit
  long long seed2_bstride;
  int ny, nx;
  int flags;
  int probe0;
  float seed_scale;          // n_px
  int tw_ready;              // as RowArgs::tw_ready
};

// numpy.fft.fftfreq(n, d)[i] in float64: i * (1/(n d)) with the upper half
// wrapped to negative frequencies
__device__ __forceinline__ double fftfreq_d(int i, int n, double d) {
  const int half = (n - 1) / 2 + 1;
  const double val = 1.0 / ((double)n * d);
  return (double)(i < half ? i : i - n) * val;
}

// ----------------------------------------------------------------------------
// transmission: t = exp(i 2 pi (n-1) dz / lambda), n - 1 without cancellation
// (propagation.py:66-81, :336)
// ----------------------------------------------------------------------------
__device__ __forceinline__ float refr_minus_one(float v, float a, float inv_den) {
  const float r = v * (a + v) * inv_den;   // n^2 - 1
  return r / (sqrtf(1.0f + r) + 1.0f);
}

__device__ __forceinline__ float2 transmission(float v, float a, float inv_den, float kphase) {
  float s, c;
  sincosf(kphase * refr_minus_one(v, a, inv_den), &s, &c);
  return make_float2(c, s);
}

// transmission table: ttab[i] = t(V[i]) for every draw and slice, computed
// once and shared by all probes that see the same potential
// ttab[i] = t(V[i]) * post_scale; post_scale is a power of two (exact), used
// to fold the 1/(ny nx) of the inverse transform into the table
static __global__ void __launch_bounds__(256) trans_table_kernel(const float* __restrict__ V, float2* __restrict__ ttab,
                                                          long long n4, float a, float inv_den, float kphase,
                                                          float post_scale = 1.0f) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n4; i += (long long)gridDim.x * blockDim.x) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(V) + i);
    const float2 t0 = cscale(transmission(v.x, a, inv_den, kphase), post_scale);
    const float2 t1 = cscale(transmission(v.y, a, inv_den, kphase), post_scale);
    const float2 t2 = cscale(transmission(v.z, a, inv_den, kphase), post_scale);
    const float2 t3 = cscale(transmission(v.w, a, inv_den, kphase), post_scale);
    float4* o = reinterpret_cast<float4*>(ttab) + 2 * i;
    o[0] = make_float4(t0.x, t0.y, t1.x, t1.y);
    o[1] = make_float4(t2.x, t2.y, t3.x, t3.y);
  }
}

// hq[i] = (H_hi, H_lo) interleaved: one 16-byte load per element in the
// column pass of the persistent scheduler
static __global__ void __launch_bounds__(256) interleave_h_kernel(const float2* __restrict__ H,
                                                           const float2* __restrict__ H_lo, float4* __restrict__ hq,
                                                           long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 h = __ldg(H + i);
    const float2 l = H_lo ? __ldg(H_lo + i) : make_float2(0.f, 0.f);
    hq[i] = make_float4(h.x, h.y, l.x, l.y);
  }
}

// Programmatic dependent launch of the row and column passes: a pass launched
// with the attribute may become resident while the previous kernel in the
// stream drains; griddepcontrol.wait then blocks until that kernel has
// completed and its writes are visible (a no-op for a normal launch), and
// launch_dependents lets the next pass start the same way.  Both come first
// in the kernel, before any global read.
__device__ __forceinline__ void pdl_wait_then_release() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ----------------------------------------------------------------------------
// row pass
// ----------------------------------------------------------------------------
template <int NX, int E>
struct RowCfg {
  using P = FFTPlan<NX, E>;
  static constexpr int T = P::T;
  static constexpr bool WARP_LOCAL = (T <= 32);
  static constexpr int PADN = RowExchange<true>::padded(NX);
};

// One row tile (rows blockDim.x / T consecutive rows of probe probe0 + by):
// the body of row_pass_kernel and of the single-probe chain kernel.  tw is
// the twiddle table in shared memory, xbuf the exchange buffer.
template <int NX, int E>
__device__ __forceinline__ void row_pass_body(const RowArgs& a, const float4* tw, float2* xbuf, int bx, int by) {
  using C = RowCfg<NX, E>;
  constexpr int T = C::T;
  const int rows = blockDim.x / T;
  const int rl = threadIdx.x / T;
  const int t = threadIdx.x - rl * T;
  const int row = bx * rows + rl;
  const int b = a.probe0 + by;
  const long long plane = (long long)a.ny * NX;
  float2* prow = a.psi + (long long)b * a.psi_bstride + (long long)row * NX;
  const RowExchange<C::WARP_LOCAL> xs{xbuf + rl * C::PADN};
  const int f = a.flags;

  float2 v[E];
  if (f & ROW_LOAD_SRC) {
    // move_probe (propagation.py:263-276): roll by position - (ny//2, nx//2)
    int sy = 0, sx = 0;
    if (a.shifts) {
      sy = (a.shifts[2 * b] - (a.ny >> 1)) & (a.ny - 1);
      sx = (a.shifts[2 * b + 1] - (NX >> 1)) & (NX - 1);
    }
    int srow = row - sy;
    srow += (srow < 0) ? a.ny : 0;
    const float2* s = a.src + (long long)b * a.src_bstride + (long long)srow * NX;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int x = (t + T * e - sx) & (NX - 1);
      v[e] = __ldg(s + x);
    }
    if (f & ROW_SCALE_SRC) {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cscale(v[e], a.src_scale);
    }
  } else {
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = __ldcg(prow + t + T * e);
  }
  // Short-chain shapes (E <= 8, the single-probe launches) fetch the
  // transmission row before the inverse transform, so its L2 latency overlaps
  // the transform instead of following it; E = 16 keeps the registers.
  constexpr bool kEarlyT = E <= 8;
  float2 tpre[kEarlyT ? E : 1];
  if (kEarlyT && (f & ROW_TRANS_TAB)) {
    const int d = a.draw ? a.draw[b] : 0;
    const float2* trow = a.ttab + (long long)d * a.v_draw_stride + (long long)a.slice * plane + (long long)row * NX;
#pragma unroll
    for (int e = 0; e < (kEarlyT ? E : 1); ++e) tpre[e] = __ldg(trow + t + T * e);
  }

  if (f & ROW_IFFT) {
    fft<NX, E, true>(v, t, xs, tw);
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = cscale(v[e], a.scale);
  }
  // snapshot of the spatial wave entering this slice (or the exit wave)
  if (a.snap) {
    float2* sp = a.snap + (long long)b * a.snap_bstride + (long long)row * NX;
#pragma unroll
    for (int e = 0; e < E; ++e) __stcs(sp + t + T * e, v[e]);
  }

  if (f & ROW_TRANS_TAB) {
    if constexpr (kEarlyT) {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmul(v[e], tpre[e]);
    } else {
      const int d = a.draw ? a.draw[b] : 0;
      const float2* trow = a.ttab + (long long)d * a.v_draw_stride + (long long)a.slice * plane + (long long)row * NX;
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmul(v[e], __ldg(trow + t + T * e));
    }
  } else if (f & (ROW_TRANS | ROW_ADJOINT)) {
    const int d = a.draw ? a.draw[b] : 0;
    const float* vrow = a.V + (long long)d * a.v_draw_stride + (long long)a.slice * plane + (long long)row * NX;
    if (f & ROW_ADJOINT) {
      // v holds lambda_a = dL/da* for a_s = psi_s t_s.
      //   dL/dV = 2 Re(conj(lambda_a) i a_s) dphi/dV,
      //   dphi/dV = kphase (E + E0 + V) inv_den / n
      //   lambda_psi_s = conj(t_s) lambda_a
      const float2* arow = a.aux + (long long)b * a.aux_bstride + (long long)row * NX;
      float* grow = a.grad + (long long)d * a.v_draw_stride + (long long)a.slice * plane + (long long)row * NX;
      const float2* trow =
          a.ttab ? a.ttab + (long long)d * a.v_draw_stride + (long long)a.slice * plane + (long long)row * NX : nullptr;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const int x = t + T * e;
        const float vv = __ldg(vrow + x);
        const float dn = refr_minus_one(vv, a.ri_a, a.ri_inv_den);
        float2 tt;
        if (trow) {
          tt = __ldg(trow + x);   // shared transmission table (unscaled)
        } else {
          float s, c;
          sincosf(a.kphase * dn, &s, &c);
          tt = make_float2(c, s);
        }
        const float2 as = cmul(__ldcg(arow + x), tt);
        const float dphidv = a.kphase * (a.e_plus_e0 + vv) * a.ri_inv_den / (1.0f + dn);
        const float gre = 2.0f * (v[e].y * as.x - v[e].x * as.y) * dphidv;
        atomicAdd(grow + x, gre);
        v[e] = cmulc(v[e], tt);
      }
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) {
        const float vv = __ldg(vrow + t + T * e);
        v[e] = cmul(v[e], transmission(vv, a.ri_a, a.ri_inv_den, a.kphase));
      }
    }
  }

  if (f & ROW_FFT) fft<NX, E, false>(v, t, xs, tw);

#pragma unroll
  for (int e = 0; e < E; ++e) __stcg(prow + t + T * e, v[e]);
}

template <int NX, int E>
__global__ void __launch_bounds__(kRowThreads)
row_pass_kernel(const RowArgs a) {
  using C = RowCfg<NX, E>;
  extern __shared__ float4 smem_raw[];
  float4* tw = smem_raw;
  float2* xbuf = reinterpret_cast<float2*>(tw + C::P::TW_SIZE);
  // a plan's twiddles do not depend on the previous pass: their load overlaps
  // its tail (one L2 round trip less on the chain of a single probe)
  if (a.tw_ready)
    for (int i = threadIdx.x; i < C::P::TW_SIZE; i += blockDim.x) tw[i] = __ldg(a.tw + i);
  pdl_wait_then_release();
  if (!a.tw_ready)
    for (int i = threadIdx.x; i < C::P::TW_SIZE; i += blockDim.x) tw[i] = a.tw[i];
  __syncthreads();
  row_pass_body<NX, E>(a, tw, xbuf, blockIdx.x, blockIdx.y);
}

// ----------------------------------------------------------------------------
// column tile load: [NY][W] complex64 from global memory (row stride nx) into
// shared memory, 16 bytes per access; consecutive threads take consecutive
// 16-byte words of a row segment, so a warp moves 512 contiguous-by-row bytes
// (the adjoint seed's second input; the column passes themselves move their
// columns between registers and global memory directly)
// ----------------------------------------------------------------------------
template <int NY>
__device__ __forceinline__ void tile_load(float2* tile, const float2* __restrict__ g, int W, int nx) {
  const int w2 = W >> 1;
  const int sh = __ffs(w2) - 1;
  float4* t4 = reinterpret_cast<float4*>(tile);
  for (int i = threadIdx.x; i < NY * w2; i += blockDim.x) {
    const int r = i >> sh, c2 = i & (w2 - 1);
    t4[i] = __ldcg(reinterpret_cast<const float4*>(g + (long long)r * nx) + c2);
  }
}

// ----------------------------------------------------------------------------
// column pass
// ----------------------------------------------------------------------------
// One column tile (W = blockDim.x / T columns of probe probe0 + by): the body
// of col_pass_kernel and of the single-probe chain kernel.
template <int NY, int E, bool SEED>
__device__ __forceinline__ void col_pass_body(const ColArgs& a, const float4* tw, float2* tile, int bx, int by) {
  using P = FFTPlan<NY, E>;
  constexpr int T = P::T;
  const int W = blockDim.x / T;
  const int c = threadIdx.x % W;
  const int t = threadIdx.x / W;
  const int col = bx * W + c;
  const int b = a.probe0 + by;
  const int nx = a.nx;
  const long long plane = (long long)NY * nx;
  // the column straight between global memory and registers (a warp moves W
  // consecutive columns of each of its rows; the tile serves the transforms)
  float2* pcol = a.psi + (long long)b * a.psi_bstride + col;
  const ColExchange<> xs{tile, W, c};
  const int f = a.flags;

  float2 v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = __ldcg(pcol + (long long)(t + T * e) * nx);
  // short-chain shapes fetch H (hi and lo) before the forward transform, as
  // the row pass does with the transmission
  constexpr bool kEarlyH = E <= 8;
  float2 hpre[kEarlyH ? E : 1], lpre[kEarlyH ? E : 1];
  if (kEarlyH && !(f & COL_NO_H)) {
#pragma unroll
    for (int e = 0; e < (kEarlyH ? E : 1); ++e) {
      const long long o = (long long)(t + T * e) * nx + col;
      hpre[e] = __ldg(a.H + o);
      lpre[e] = a.H_lo ? __ldg(a.H_lo + o) : make_float2(0.f, 0.f);
    }
  }

  if (!(f & COL_NO_FFT)) fft<NY, E, false>(v, t, xs, tw);

  // fftshift of (ky, kx) for dp / g
  const int sx = (col + (nx >> 1)) & (nx - 1);
  // position of this column in the detector window (rows are tested per element)
  const int drx = sx - a.det.x0;
  const bool dcol = (unsigned)drx < (unsigned)a.det.nx;
  if constexpr (SEED) {
    const float* gp = a.g + (long long)b * a.det.plane() + drx;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int ky = t + T * e;
      const int ry = ((ky + (NY >> 1)) & (NY - 1)) - a.det.y0;
      const bool in = a.g && dcol && (unsigned)ry < (unsigned)a.det.ny;
      v[e] = in ? cscale(v[e], a.seed_scale * __ldg(gp + ry * a.det.nx)) : make_float2(0.f, 0.f);
    }
    if (a.seed2) {
      float2 u[E];
      __syncthreads();
      tile_load<NY>(tile, a.seed2 + (long long)b * a.seed2_bstride + (long long)bx * W, W, nx);
      __syncthreads();
#pragma unroll
      for (int e = 0; e < E; ++e) u[e] = xs.ld(t + T * e);
      fft<NY, E, false>(u, t, xs, tw);
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cadd(v[e], u[e]);
    }
  }

  if (kEarlyH && !(f & COL_NO_H)) {
    if (f & COL_CONJ_H) {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmulc_hl(v[e], hpre[e], lpre[e]);
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmul_hl(v[e], hpre[e], lpre[e]);
    }
  } else if (!(f & COL_NO_H)) {
    const float2* hcol = a.H + col;
    if (a.H_lo) {
      const float2* lcol = a.H_lo + col;
      if (f & COL_CONJ_H) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const long long o = (long long)(t + T * e) * nx;
          v[e] = cmulc_hl(v[e], __ldg(hcol + o), __ldg(lcol + o));
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const long long o = (long long)(t + T * e) * nx;
          v[e] = cmul_hl(v[e], __ldg(hcol + o), __ldg(lcol + o));
        }
      }
    } else if (f & COL_CONJ_H) {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmulc(v[e], __ldg(hcol + (long long)(t + T * e) * nx));
    } else {
#pragma unroll
      for (int e = 0; e < E; ++e) v[e] = cmul(v[e], __ldg(hcol + (long long)(t + T * e) * nx));
    }
  }

  if (f & COL_DP) {
    float* dp = a.dp + (long long)b * a.det.plane() + drx;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int ky = t + T * e;
      const int ry = ((ky + (NY >> 1)) & (NY - 1)) - a.det.y0;
      if (dcol && (unsigned)ry < (unsigned)a.det.ny) __stcs(dp + ry * a.det.nx, fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
    }
    if (f & COL_NO_H) return;  // pure diffraction epilogue: no inverse transform
  }

  if (!(f & COL_FWD_ONLY)) fft<NY, E, true>(v, t, xs, tw);
#pragma unroll
  for (int e = 0; e < E; ++e) __stcg(pcol + (long long)(t + T * e) * nx, v[e]);
}

template <int NY, int E, bool SEED>
__global__ void __launch_bounds__(kColThreads)
col_pass_kernel(const ColArgs a) {
  using P = FFTPlan<NY, E>;
  extern __shared__ float4 smem_raw[];
  float4* tw = smem_raw;
  float2* tile = reinterpret_cast<float2*>(tw + P::TW_SIZE);
  if (a.tw_ready)
    for (int i = threadIdx.x; i < P::TW_SIZE; i += blockDim.x) tw[i] = __ldg(a.tw + i);
  pdl_wait_then_release();
  if (!a.tw_ready)
    for (int i = threadIdx.x; i < P::TW_SIZE; i += blockDim.x) tw[i] = a.tw[i];
  __syncthreads();
  col_pass_body<NY, E, SEED>(a, tw, tile, blockIdx.x, blockIdx.y);
}

// The WPM bin propagator applied to v = X * Hvac by the direct formulas, for
// the pixels outside the series' range (near or beyond the evanescent edge).
// Rarely taken, so kept out of line: the unrolled bin loop stays small.
static __device__ __noinline__ float2 wpm_bin_direct(float2 v, float pr, float ak, float dz, const float2* hvac) {
  const float q0 = 1.0f / pr;
  const float sq0 = sqrtf(fabsf(q0));
  const float qk = q0 + ak;
  if (q0 >= 0.0f && qk >= 0.0f) {
    float s, c;
    sincosf(dz * ak / (sqrtf(qk) + sq0), &s, &c);
    return cmul(v, make_float2(c, s));
  }
  if (q0 < 0.0f && qk < 0.0f) return cscale(v, expf(dz * ak / (sqrtf(-qk) + sq0)));
  // one side evanescent: exact H_k; undo the vacuum factor on X.  v = X * hv;
  // |hv| is 1 (propagating vacuum) or a decay factor: divide it out explicitly
  const float2 hv = __ldg(hvac);
  float2 hk;
  if (qk >= 0.0f) {
    float s, c;
    sincosf(dz * sqrtf(qk), &s, &c);
    hk = make_float2(c, s);
  } else {
    hk = make_float2(expf(-dz * sqrtf(-qk)), 0.0f);
  }
  const float n2 = fmaf(hv.x, hv.x, hv.y * hv.y);
  const float2 x = n2 > 0.0f ? cscale(cmulc(v, hv), 1.0f / n2) : make_float2(0.f, 0.f);
  return cmul(x, hk);
}

// exp(i phi) for phases beyond the Taylor range, out of line for the same reason
static __device__ __noinline__ float2 cis_large(float ph) {
  float s, c;
  sincosf(ph, &s, &c);
  return make_float2(c, s);
}

// exp(i phi) = (cos phi, sin phi) by the Taylor series of cos and sin in Horner
// form, for |phi| <= 0.5 (truncation below 1e-10, under float rounding);
// larger phases go to sincosf.  The WPM bin phases are small (dz |n_k - 1| k0).
__device__ __forceinline__ float2 cis_small(float ph) {
  if (fabsf(ph) > 0.5f) return cis_large(ph);
  const float p2 = ph * ph;
  // Taylor coefficients (-1)^j / (2j+1)! and (-1)^j / (2j)!
  const float sn = ph * fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, 2.7557319e-06f, -1.9841270e-04f), 8.3333333e-03f),
                                      -1.6666667e-01f), 1.0f);
  const float cs = fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, fmaf(p2, -2.7557319e-07f, 2.4801587e-05f), -1.3888889e-03f),
                                           4.1666667e-02f), -0.5f), 1.0f);
  return make_float2(cs, sn);
}

// ----------------------------------------------------------------------------
// WPM (propagation.py:215-256)
// ----------------------------------------------------------------------------
// Per slice the reference forms K reference fields u_k = ifft2(H_k fft2(psi))
// with H_k = exp(i dz sqrt(n_k^2 k0^2 - k_perp^2)) and blends, per pixel, the
// two fields that bracket the pixel's n with smoothstep weights.  Here:
//   * bins live in delta = n - 1 (n_refs - 1 = dmin + (dmax - dmin) t^p,
//     the same points), computed for all slices up front (wpm_bins_kernel);
//   * H_k = Hvac * exp(i dz a_k / (kz_k + kz_0)), a_k = k0^2 dk (2 + dk),
//     with Hvac = exp(i dz sqrt(k0^2 - k_perp^2)) tabulated in float64 on the
//     device and rounded once; the small residual phase is formed in float32
//     without cancellation.  Evanescent components use the complex-sqrt
//     branch of the reference directly;
//   * wpm_col_kernel writes the K column-transformed fields, wpm_row_kernel
//     finishes each field's inverse row transform and accumulates the blend.

struct WpmBinsArgs {
  const float* V;            // (draws, n_slices, ny, nx)
  float* refs;               // (draws, n_slices, K) delta reference values
  int n_px, n_slices, K;
  float ri_a, ri_inv_den;
  double power;
};

// one CTA per (slice, draw): min/max of delta over the slice, then the K
// reference values delta_min + (delta_max - delta_min) t_k^p in float64.
// Each thread keeps eight 16-byte loads in flight per trip: with one, the
// slice's reduction is a chain of 64 memory latencies at 512^2.
static __global__ void __launch_bounds__(1024) wpm_bins_kernel(const WpmBinsArgs a) {
  constexpr int kInFlight = 8;
  const int s = blockIdx.x, d = blockIdx.y;
  const float4* v4 = reinterpret_cast<const float4*>(a.V + ((long long)d * a.n_slices + s) * a.n_px);
  const int n4 = a.n_px >> 2, step = blockDim.x;
  float lo = 3.0e38f, hi = -3.0e38f;
  auto fold = [&](const float4 q) {
    const float d0 = refr_minus_one(q.x, a.ri_a, a.ri_inv_den);
    const float d1 = refr_minus_one(q.y, a.ri_a, a.ri_inv_den);
    const float d2 = refr_minus_one(q.z, a.ri_a, a.ri_inv_den);
    const float d3 = refr_minus_one(q.w, a.ri_a, a.ri_inv_den);
    lo = fminf(lo, fminf(fminf(d0, d1), fminf(d2, d3)));
    hi = fmaxf(hi, fmaxf(fmaxf(d0, d1), fmaxf(d2, d3)));
  };
  int i = threadIdx.x;
  for (; i + (kInFlight - 1) * step < n4; i += kInFlight * step) {
    float4 q[kInFlight];
#pragma unroll
    for (int u = 0; u < kInFlight; ++u) q[u] = __ldg(v4 + i + u * step);
#pragma unroll
    for (int u = 0; u < kInFlight; ++u) fold(q[u]);
  }
  for (; i < n4; i += step) fold(__ldg(v4 + i));
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
      // numpy linspace(0, 1, K): k * (1/(K-1)), last point exactly 1
      const double tk = (k == a.K - 1) ? 1.0 : (double)k * (1.0 / (double)(a.K - 1));
      const double tp = (a.power == 1.0) ? tk : pow(tk, a.power);
      out[k] = (float)(dlo + (dhi - dlo) * tp);
    }
  }
}

struct WpmColArgs {
  const float2* psi;         // (B, ny, nx) row-transformed wave
  float2* fields;            // (B, K, ny, nx) column-transformed reference fields
  const float2* hvac;        // (ny, nx)  exp(i dz kz_vac): complex64 hi part
  const float2* hvac_lo;     // (ny, nx)  and lo part of the float64 value
  const float* ky2;          // (ny) (2 pi fy)^2
  const float* kx2;          // (nx) (2 pi fx)^2
  const float* refs;         // (draws, n_slices, K)
  const int* draw;
  const float4* tw;
  float* dp;                 // dp mode: |fft2|^2 (fftshifted, detector window), no fields
  Detector det;
  int ny, nx, K, slice, n_slices, probe0, dp_mode;
  int kpg;                   // bins per CTA group (blockIdx.z): bins [z kpg, min(z kpg + kpg, K))
  float k02;                 // k0^2
  float dz;
};

template <int NY, int E>
__global__ void __launch_bounds__(kColThreads)
wpm_col_kernel(const WpmColArgs a) {
  using P = FFTPlan<NY, E>;
  constexpr int T = P::T;
  const int W = blockDim.x / T;
  extern __shared__ float4 smem_raw[];
  float4* tw = smem_raw;
  float2* tile = reinterpret_cast<float2*>(tw + P::TW_SIZE);
  float* srefs = reinterpret_cast<float*>(tile + NY * W);
  for (int i = threadIdx.x; i < P::TW_SIZE; i += blockDim.x) tw[i] = a.tw[i];
  const int c = threadIdx.x % W;
  const int t = threadIdx.x / W;
  const int col = blockIdx.x * W + c;
  const int b = a.probe0 + blockIdx.y;
  if (!a.dp_mode) {
    const int d = a.draw ? a.draw[b] : 0;
    const float* r = a.refs + ((long long)d * a.n_slices + a.slice) * a.K;
    for (int i = threadIdx.x; i < a.K; i += blockDim.x) srefs[i] = r[i];
  }
  __syncthreads();
  const int nx = a.nx;
  const long long plane = (long long)NY * nx;
  const ColExchange<> xs{tile, W, c};

  // the column straight from global memory (a warp reads W consecutive
  // columns of each of its rows; the tile serves the transforms only)
  float2 v[E];
  const float2* pcol = a.psi + (long long)b * plane + col;
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = __ldcg(pcol + (long long)(t + T * e) * nx);
  fft<NY, E, false>(v, t, xs, tw);

  if (a.dp_mode) {
    const int drx = ((col + (nx >> 1)) & (nx - 1)) - a.det.x0;
    if ((unsigned)drx >= (unsigned)a.det.nx) return;   // column outside the detector window
    float* dp = a.dp + (long long)b * a.det.plane() + drx;
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const int ry = ((t + T * e + (NY >> 1)) & (NY - 1)) - a.det.y0;
      if ((unsigned)ry < (unsigned)a.det.ny) __stcs(dp + ry * a.det.nx, fmaf(v[e].x, v[e].x, v[e].y * v[e].y));
    }
    return;
  }

  // per element: q0 = k0^2 - k_perp^2, X * Hvac
  float q0[E];
  const float kx2 = __ldg(a.kx2 + col);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const int ky = t + T * e;
    q0[e] = a.k02 - (__ldg(a.ky2 + ky) + kx2);
    v[e] = cmul_hl(v[e], __ldg(a.hvac + (long long)ky * nx + col), __ldg(a.hvac_lo + (long long)ky * nx + col));
  }
  // Bin phase dz a_k / (sqrt(q0 + a_k) + sqrt(q0)) = (dz a_k / (2 sqrt(q0))) f(a_k / q0)
  // with f(x) = 2 / (1 + sqrt(1 + x)) = 1 - x/4 + x^2/8 - 5 x^3/64 + O(x^4): to
  // float rounding while |a_k| <= q0 / 128 (the x^4 term is below 1e-9), which
  // holds away from the evanescent edge (|a_k| / k0^2 is 2|n_k - 1|, ~1e-4).
  // pa = dz / (2 sqrt(q0)) (0 when q0 <= 0), pr = 1 / q0; other elements take
  // the direct formulas below.
  float pa[E], pr[E];
#pragma unroll
  for (int e = 0; e < E; ++e) {
    pr[e] = 1.0f / q0[e];
    pa[e] = q0[e] > 0.0f ? 0.5f * a.dz * sqrtf(pr[e]) : 0.0f;
  }

  float2* fcol = a.fields + (long long)b * a.K * plane + col;
  const int kb = blockIdx.z * a.kpg, ke = min(kb + a.kpg, a.K);
  for (int k = kb; k < ke; ++k) {
    const float dk = srefs[k];
    const float ak = a.k02 * dk * (2.0f + dk);   // n_k^2 k0^2 - k0^2
    float2 u[E];
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const float x = ak * pr[e];
      if (pa[e] > 0.0f && fabsf(x) <= 0.0078125f) {
        const float ph = ak * pa[e] * fmaf(x, fmaf(x, fmaf(x, -0.078125f, 0.125f), -0.25f), 1.0f);
        u[e] = cmul(v[e], cis_small(ph));
        continue;
      }
      u[e] = wpm_bin_direct(v[e], pr[e], ak, a.dz, a.hvac + (long long)(t + T * e) * nx + col);
    }
    fft<NY, E, true>(u, t, xs, tw);
    // field k straight from the registers (no staging through the tile: the
    // next transform's first exchange waits for every thread's reads)
    float2* fk = fcol + (long long)k * plane;
#pragma unroll
    for (int e = 0; e < E; ++e) __stcg(fk + (long long)(t + T * e) * nx, u[e]);
  }
}

struct WpmRowArgs {
  float2* psi;               // (B, ny, nx): out (row-transformed next wave)
  const float2* fields;      // (B, K, ny, nx)
  float2* dpbuf;             // last slice: row FFT of the exit wave goes here
  long long dpbuf_bstride;
  const float* V;
  const int* draw;
  long long v_draw_stride;
  const float* refs;
  const float4* tw;
  float2* snap;              // wavefront after this slice (spatial)
  long long snap_bstride;
  int ny, nx, K, slice, n_slices, probe0, last;
  float scale;               // 1/(ny nx)
  float ri_a, ri_inv_den;
  // Bin-split mode (blend != null): CTA group z owns the pixels whose left
  // bin lies in [z kpg, min(z kpg + kpg, K - 1)), transforms the bins it needs
  // (its own and the next group's first), and stores the owned pixels' blend
  // into `blend`; a row pass then applies the forward row FFT.
  float2* blend;
  int kpg;
};

template <int NX, int E>
__global__ void __launch_bounds__(kRowThreads, E <= 8 ? 3 : 1)
wpm_row_kernel(const WpmRowArgs a) {
  using C = RowCfg<NX, E>;
  constexpr int T = C::T;
  const int rows = blockDim.x / T;
  extern __shared__ float4 smem_raw[];
  float4* tw = smem_raw;
  float2* xbuf = reinterpret_cast<float2*>(tw + C::P::TW_SIZE);
  float* srefs = reinterpret_cast<float*>(xbuf + rows * C::PADN);
  unsigned* used = reinterpret_cast<unsigned*>(srefs + a.K);
  const int b = a.probe0 + blockIdx.y;
  const int d = a.draw ? a.draw[b] : 0;
  for (int i = threadIdx.x; i < C::P::TW_SIZE; i += blockDim.x) tw[i] = a.tw[i];
  {
    const float* r = a.refs + ((long long)d * a.n_slices + a.slice) * a.K;
    for (int i = threadIdx.x; i < a.K; i += blockDim.x) srefs[i] = r[i];
    for (int i = threadIdx.x; i < (a.K + 31) / 32; i += blockDim.x) used[i] = 0u;
  }
  __syncthreads();

  const int rl = threadIdx.x / T;
  const int t = threadIdx.x - rl * T;
  const int row = blockIdx.x * rows + rl;
  const long long plane = (long long)a.ny * NX;
  const RowExchange<C::WARP_LOCAL> xs{xbuf + rl * C::PADN};
  const int K = a.K;

  // bracketing bins and smoothstep weights (propagation.py:239-249)
  const bool split = a.blend != nullptr;
  const int kb = split ? blockIdx.z * a.kpg : 0;           // owned left bins [kb, kl)
  const int kl = split ? min(kb + a.kpg, K - 1) : K - 1;
  int il[E];
  float wr[E];
  const float* vrow = a.V + (long long)d * a.v_draw_stride + (long long)a.slice * plane + (long long)row * NX;
#pragma unroll
  for (int e = 0; e < E; ++e) {
    const float dn = refr_minus_one(__ldg(vrow + t + T * e), a.ri_a, a.ri_inv_den);
    // searchsorted(side='left'): first index with refs[i] >= dn
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
    if (ir - 1 >= kb && ir - 1 < kl) {
      atomicOr(used + ((ir - 1) >> 5), 1u << ((ir - 1) & 31));
      atomicOr(used + (ir >> 5), 1u << (ir & 31));
    }
  }
  __syncthreads();

  float2 acc[E];
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = make_float2(0.f, 0.f);
  const float2* frow = a.fields + (long long)b * K * plane + (long long)row * NX;
  for (int k = kb; k <= kl; ++k) {
    if (!(used[k >> 5] & (1u << (k & 31)))) continue;   // CTA-uniform
    float2 u[E];
    const float2* fk = frow + (long long)k * plane;
#pragma unroll
    for (int e = 0; e < E; ++e) u[e] = __ldcg(fk + t + T * e);
    fft<NX, E, true>(u, t, xs, tw);
#pragma unroll
    for (int e = 0; e < E; ++e) {
      const float cw = (il[e] == k) ? (1.0f - wr[e]) : ((il[e] + 1 == k) ? wr[e] : 0.0f);
      acc[e] = make_float2(fmaf(cw, u[e].x, acc[e].x), fmaf(cw, u[e].y, acc[e].y));
    }
  }
#pragma unroll
  for (int e = 0; e < E; ++e) acc[e] = cscale(acc[e], a.scale);

  if (split) {
    float2* brow = a.blend + (long long)b * plane + (long long)row * NX;
#pragma unroll
    for (int e = 0; e < E; ++e)
      if (il[e] >= kb && il[e] < kl) __stcg(brow + t + T * e, acc[e]);
    return;
  }

  if (a.snap) {
    float2* sp = a.snap + (long long)b * a.snap_bstride + (long long)row * NX;
#pragma unroll
    for (int e = 0; e < E; ++e) __stcs(sp + t + T * e, acc[e]);
  }
  float2* prow = a.psi + (long long)b * plane + (long long)row * NX;
  if (a.last) {
#pragma unroll
    for (int e = 0; e < E; ++e) __stcg(prow + t + T * e, acc[e]);
  }
  fft<NX, E, false>(acc, t, xs, tw);
  float2* orow = a.last ? a.dpbuf + (long long)b * a.dpbuf_bstride + (long long)row * NX : prow;
#pragma unroll
  for (int e = 0; e < E; ++e) __stcg(orow + t + T * e, acc[e]);
}

}  // namespace wap
