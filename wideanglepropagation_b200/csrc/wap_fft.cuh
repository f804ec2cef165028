// In-house complex64 FFT core for the multislice passes (sm_100a).
//
// One N-point transform is computed by T = N/E threads; thread t holds the E
// elements x[t + T*e] (e = 0..E-1) in registers.  The transform is a radix-E
// Stockham autosort (plus one smaller remainder radix), numpy.fft sign and
// normalisation conventions: forward exp(-2 pi i jk/N) unnormalised, inverse
// exp(+2 pi i jk/N) unnormalised (callers apply 1/N).
//
// Stage s (radix R, span L = product of earlier radices), butterfly
// b = t + T*q, k = b mod L:
//   inputs  x[b + (N/R) j] = register slot q + (E/R) j
//   twiddle W_{LR}^{jk}, from a per-stage table laid out [j][k] so that
//           consecutive threads read consecutive words; each entry holds
//           the float64 value as float hi + lo parts (systematic rounding
//           of a float-only table would repeat identically every slice);
//           the hi parts alone (float2) are the cheaper format for waves
//           that pass through few enough transforms
//   outputs y_m -> position (b - k) R + k + m L, exchanged through shared
//           memory for every stage but the last.
// After the last stage thread t again holds X[t + T*e] in slot e, so a forward
// transform, a pointwise multiply and an inverse transform chain in registers.
// The in-register radix-2/4/8/16 butterflies use split-radix-free 4x4 / 2x4
// decompositions with exact constants of the 16th roots of unity.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace wap {

// ----------------------------------------------------------------------------
// plan arithmetic, shared by host (twiddle tables) and device (stages)
// ----------------------------------------------------------------------------
__host__ __device__ constexpr int ilog2c(int n) { return n <= 1 ? 0 : 1 + ilog2c(n >> 1); }

template <int N, int E>
struct FFTPlan {
  static_assert((N & (N - 1)) == 0 && (E & (E - 1)) == 0, "powers of two");
  static_assert(E >= 2 && E <= 16 && N >= E, "2 <= E <= 16 <= N");
  static constexpr int T = N / E;
  static constexpr int LOGN = ilog2c(N);
  static constexpr int LOGE = ilog2c(E);
  static constexpr int NFULL = LOGN / LOGE;
  static constexpr int REM = 1 << (LOGN % LOGE);
  static constexpr int S = NFULL + (REM > 1 ? 1 : 0);
  __host__ __device__ static constexpr int radix(int s) { return s < NFULL ? E : REM; }
  __host__ __device__ static constexpr int span(int s) {
    int L = 1;
    for (int i = 0; i < s; ++i) L *= radix(i);
    return L;
  }
  // offset of stage s in the concatenated twiddle table (stages s >= 1; a
  // stage holds rows j = 1 .. R-1 of its [j][k] table, row 0 being all ones)
  __host__ __device__ static constexpr int tw_offset(int s) {
    int off = 0;
    for (int i = 1; i < s; ++i) off += (radix(i) - 1) * span(i);
    return off;
  }
  static constexpr int TW_SIZE = tw_offset(S) > 0 ? tw_offset(S) : 1;
};

// Runtime mirror of FFTPlan for the host-side table builder.
struct PlanShape {
  int n, e, nfull, rem, stages;
  __host__ __device__ int radix(int s) const { return s < nfull ? e : rem; }
  __host__ __device__ int span(int s) const {
    int L = 1;
    for (int i = 0; i < s; ++i) L *= radix(i);
    return L;
  }
  __host__ __device__ int tw_offset(int s) const {
    int off = 0;
    for (int i = 1; i < s; ++i) off += (radix(i) - 1) * span(i);
    return off;
  }
  __host__ __device__ int tw_size() const { int t = tw_offset(stages); return t > 0 ? t : 1; }
};

__host__ __device__ inline PlanShape make_plan_shape(int n, int e) {
  PlanShape p{};
  int logn = ilog2c(n), loge = ilog2c(e);
  p.n = n;
  p.e = e;
  p.nfull = logn / loge;
  p.rem = 1 << (logn % loge);
  p.stages = p.nfull + (p.rem > 1 ? 1 : 0);
  return p;
}

// ----------------------------------------------------------------------------
// complex helpers
// ----------------------------------------------------------------------------
// Complex add / subtract as one packed FP32x2 instruction (sm_100 add/sub
// .f32x2: both lanes rounded exactly like two scalar adds), halving the issue
// slots of the butterflies' additions.
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) {
  float2 r;
  asm("{\n\t.reg .b64 pa, pb, pr;\n\tmov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\t"
      "sub.rn.f32x2 pr, pa, pb;\n\tmov.b64 {%0, %1}, pr;\n\t}"
      : "=f"(r.x), "=f"(r.y)
      : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
  return r;
}
// a + (-i) b and a - (-i) b (forward sign; INV: +i), the rotated pair of a
// radix-4 butterfly: scalar adds, since the rotation swaps the lanes
template <bool INV>
__device__ __forceinline__ float2 cadd_rot(float2 a, float2 b) {
  return INV ? make_float2(a.x - b.y, a.y + b.x) : make_float2(a.x + b.y, a.y - b.x);
}
template <bool INV>
__device__ __forceinline__ float2 csub_rot(float2 a, float2 b) {
  return INV ? make_float2(a.x + b.y, a.y - b.x) : make_float2(a.x - b.y, a.y + b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }

// multiply by -i (forward sign) or +i (inverse sign)
template <bool INV>
__device__ __forceinline__ float2 mul_mi(float2 a) {
  return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

// cos / sin of 2 pi m / 16 as an unevaluated float sum hi + lo (|lo| < ulp(hi)/2).
// The hi parts alone carry a systematic rounding error that every slice
// applies again; the lo parts remove it (see tw16).
struct Pair {
  float hi, lo;
};
__device__ __forceinline__ Pair cos16p(int m) {
  constexpr float C8H = 0.9238795042037964f, C8L = 2.830748968563057e-08f;
  constexpr float R2H = 0.7071067690849304f, R2L = 1.2101617485882343e-08f;
  constexpr float S8H = 0.3826834261417389f, S8L = 6.2233507236442165e-09f;
  switch (m & 15) {
    case 0: return {1.0f, 0.0f};
    case 1: return {C8H, C8L};
    case 2: return {R2H, R2L};
    case 3: return {S8H, S8L};
    case 4: return {0.0f, 0.0f};
    case 5: return {-S8H, -S8L};
    case 6: return {-R2H, -R2L};
    case 7: return {-C8H, -C8L};
    case 8: return {-1.0f, 0.0f};
    case 9: return {-C8H, -C8L};
    case 10: return {-R2H, -R2L};
    case 11: return {-S8H, -S8L};
    case 12: return {0.0f, 0.0f};
    case 13: return {S8H, S8L};
    case 14: return {R2H, R2L};
    default: return {C8H, C8L};
  }
}
__device__ __forceinline__ Pair sin16p(int m) { return cos16p(m - 4); }

// a * W16^m with W16 = exp(-+2 pi i / 16); m is a compile-time constant after
// unrolling, so the branches fold away.  Non-trivial constants are applied as
// hi + lo through FMAs.
template <bool INV>
__device__ __forceinline__ float2 tw16(float2 a, int m) {
  m &= 15;
  if (m == 0) return a;
  if (m == 8) return make_float2(-a.x, -a.y);
  if (m == 4) return mul_mi<INV>(a);
  if (m == 12) return mul_mi<!INV>(a);
  const Pair c = cos16p(m);
  Pair s = sin16p(m);
  if (!INV) s = {-s.hi, -s.lo};  // twiddle = c + i s
  if ((m & 3) == 2) {
    // |c| == |s|: one rounded sum, then c (hi + lo)
    const float d0 = (c.hi == s.hi) ? a.x - a.y : a.x + a.y;
    const float d1 = (c.hi == s.hi) ? a.y + a.x : a.y - a.x;
    return make_float2(fmaf(c.hi, d0, c.lo * d0), fmaf(c.hi, d1, c.lo * d1));
  }
  return make_float2(fmaf(c.hi, a.x, fmaf(-s.hi, a.y, fmaf(c.lo, a.x, -s.lo * a.y))),
                     fmaf(c.hi, a.y, fmaf(s.hi, a.x, fmaf(c.lo, a.y, s.lo * a.x))));
}

// complex multiply by a twiddle stored as (re_hi, im_hi, re_lo, im_lo)
__device__ __forceinline__ float2 cmul_tw(float2 a, float4 w) {
  return make_float2(fmaf(a.x, w.x, fmaf(-a.y, w.y, fmaf(a.x, w.z, -a.y * w.w))),
                     fmaf(a.x, w.y, fmaf(a.y, w.x, fmaf(a.x, w.w, a.y * w.z))));
}
// a * conj(twiddle)
__device__ __forceinline__ float2 cmulc_tw(float2 a, float4 w) {
  return make_float2(fmaf(a.x, w.x, fmaf(a.y, w.y, fmaf(a.x, w.z, a.y * w.w))),
                     fmaf(a.y, w.x, fmaf(-a.x, w.y, fmaf(a.y, w.z, -a.x * w.w))));
}
// stage-twiddle multiply for the two table formats: float4 (hi + lo, exact to
// float64 rounding) or float2 (hi only: one rounding per entry, which repeats
// identically in every transform - cheaper, with a systematic error that grows
// with the number of transforms a wave goes through)
template <bool INV>
__device__ __forceinline__ float2 tw_mul(float2 a, float4 w) { return INV ? cmulc_tw(a, w) : cmul_tw(a, w); }
template <bool INV>
__device__ __forceinline__ float2 tw_mul(float2 a, float2 w) { return INV ? cmulc(a, w) : cmul(a, w); }

// a * (h + hl) for a propagator value split into complex64 hi and lo parts
__device__ __forceinline__ float2 cmul_hl(float2 a, float2 h, float2 hl) {
  return make_float2(fmaf(a.x, h.x, fmaf(-a.y, h.y, fmaf(a.x, hl.x, -a.y * hl.y))),
                     fmaf(a.x, h.y, fmaf(a.y, h.x, fmaf(a.x, hl.y, a.y * hl.x))));
}
__device__ __forceinline__ float2 cmulc_hl(float2 a, float2 h, float2 hl) {
  return make_float2(fmaf(a.x, h.x, fmaf(a.y, h.y, fmaf(a.x, hl.x, a.y * hl.y))),
                     fmaf(a.y, h.x, fmaf(-a.x, h.y, fmaf(a.y, hl.x, -a.x * hl.y))));
}

// ----------------------------------------------------------------------------
// in-register DFT codelets, natural order in and out
// ----------------------------------------------------------------------------
template <bool INV>
__device__ __forceinline__ void dft2(float2& a0, float2& a1) {
  float2 t = a0;
  a0 = cadd(t, a1);
  a1 = csub(t, a1);
}

template <bool INV>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
  float2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
  float2 t2 = cadd(a1, a3), d = csub(a1, a3);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd_rot<INV>(t1, d);   // t1 + (-+i) d
  a3 = csub_rot<INV>(t1, d);
}

// dft4 whose input a2 still carries a factor -+i (W16^4 of the radix-16
// codelet): the rotation is folded into the additions that use a2
template <bool INV>
__device__ __forceinline__ void dft4_rot2(float2& a0, float2& a1, float2& a2, float2& a3) {
  float2 t0 = cadd_rot<INV>(a0, a2), t1 = csub_rot<INV>(a0, a2);
  float2 t2 = cadd(a1, a3), d = csub(a1, a3);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  a1 = cadd_rot<INV>(t1, d);
  a3 = csub_rot<INV>(t1, d);
}

template <int R, bool INV>
__device__ __forceinline__ void dft(float2 (&a)[R]) {
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2<INV>(a[0], a[1]);
  } else if constexpr (R == 4) {
    dft4<INV>(a[0], a[1], a[2], a[3]);
  } else if constexpr (R == 8) {
    // n = n1 + 2 n2, k = 4 k1 + k2
#pragma unroll
    for (int n1 = 0; n1 < 2; ++n1) dft4<INV>(a[n1], a[n1 + 2], a[n1 + 4], a[n1 + 6]);
    // Y[n1][k2] sits in a[n1 + 2 k2]; W16^4 (k2 = 2) is folded into its additions
    a[3] = tw16<INV>(a[3], 2);
    a[7] = tw16<INV>(a[7], 6);
    float2 o[8];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      float2 y0 = a[2 * k2], y1 = a[1 + 2 * k2];
      if (k2 == 2) {
        o[k2] = cadd_rot<INV>(y0, y1);
        o[4 + k2] = csub_rot<INV>(y0, y1);
      } else {
        o[k2] = cadd(y0, y1);
        o[4 + k2] = csub(y0, y1);
      }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = o[i];
  } else if constexpr (R == 16) {
    // n = n1 + 4 n2, k = 4 k1 + k2
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) dft4<INV>(a[n1], a[n1 + 4], a[n1 + 8], a[n1 + 12]);
    // Y[n1][k2] sits in a[n1 + 4 k2]; W16^4 (n1 = k2 = 2) is folded into the
    // additions of its dft4
#pragma unroll
    for (int n1 = 1; n1 < 4; ++n1)
#pragma unroll
      for (int k2 = 1; k2 < 4; ++k2)
        if (n1 * k2 != 4) a[n1 + 4 * k2] = tw16<INV>(a[n1 + 4 * k2], n1 * k2);
    float2 o[16];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
      float2 y0 = a[4 * k2], y1 = a[1 + 4 * k2], y2 = a[2 + 4 * k2], y3 = a[3 + 4 * k2];
      if (k2 == 2) dft4_rot2<INV>(y0, y1, y2, y3);
      else dft4<INV>(y0, y1, y2, y3);
      o[k2] = y0;
      o[4 + k2] = y1;
      o[8 + k2] = y2;
      o[12 + k2] = y3;
    }
#pragma unroll
    for (int i = 0; i < 16; ++i) a[i] = o[i];
  } else {
    static_assert(R <= 16, "radix");
  }
}

// ----------------------------------------------------------------------------
// shared-memory exchange policies
// ----------------------------------------------------------------------------
// Block-level barrier: __syncthreads, or named barrier BAR over NT threads
// when only part of the block (e.g. the compute warps of a warp-specialised
// kernel) takes part in the transform.
template <int BAR, int NT>
__device__ __forceinline__ void block_sync() {
  if constexpr (BAR == 0) {
    __syncthreads();
  } else {
    asm volatile("bar.sync %0, %1;" ::"n"(BAR), "n"(NT) : "memory");
  }
}

// One transform per row segment of shared memory; index p padded by one word
// per 16 so that radix-R Stockham scatters are bank-conflict free.
template <bool WARP_LOCAL, int BAR = 0, int NT = 0>
struct RowExchange {
  float2* base;
  __device__ __forceinline__ void st(int p, float2 v) const { base[p + (p >> 4)] = v; }
  __device__ __forceinline__ float2 ld(int p) const { return base[p + (p >> 4)]; }
  // position b + o, b a run-time value and o a compile-time offset
  __device__ __forceinline__ void st2(int b, int o, float2 v) const { st(b + o, v); }
  __device__ __forceinline__ float2 ld2(int b, int o) const { return ld(b + o); }
  __device__ __forceinline__ void sync() const {
    if constexpr (WARP_LOCAL) __syncwarp();
    else block_sync<BAR, NT>();
  }
  __host__ __device__ static constexpr int padded(int n) { return n + (n >> 4); }
};

// One transform per column of a row-major [N][W] tile (lanes run along the
// columns, so stores of one Stockham position by a warp are contiguous).
template <int BAR = 0, int NT = 0>
struct ColExchange {
  float2* base;
  int w, c;
  __device__ __forceinline__ void st(int p, float2 v) const { base[p * w + c] = v; }
  __device__ __forceinline__ float2 ld(int p) const { return base[p * w + c]; }
  __device__ __forceinline__ void st2(int b, int o, float2 v) const { st(b + o, v); }
  __device__ __forceinline__ float2 ld2(int b, int o) const { return ld(b + o); }
  __device__ __forceinline__ void sync() const { block_sync<BAR, NT>(); }
};

// ColExchange with one padding row per 16: position p lives in row
// p + p / 16 of a [N + N/16][W] buffer.  With W = 8 (512-point columns) the
// radix-16 scatter of the first stage sends the two positions 16 rows apart
// that a half-warp stores to the same banks of an unpadded [N][8] tile; the
// padding row moves every other 16-row block to the other half of the banks.
// The padded row is formed from the stage's run-time base b and compile-time
// offset o separately - pad(b + o) = pad(b) + pad(o) - which holds when the
// low four bits of b and o do not carry: true of every E = 16 Stockham stage
// (first stage: b a multiple of 16, o < 16; later stages and the reads: o a
// multiple of 16).
template <int BAR = 0, int NT = 0>
struct ColExchangePad {
  float2* base;
  int w, c;
  __device__ __forceinline__ static int pad(int p) { return p + (p >> 4); }
  __device__ __forceinline__ void st2(int b, int o, float2 v) const { base[(pad(b) + pad(o)) * w + c] = v; }
  __device__ __forceinline__ float2 ld2(int b, int o) const { return base[(pad(b) + pad(o)) * w + c]; }
  __device__ __forceinline__ void sync() const { block_sync<BAR, NT>(); }
};

// ----------------------------------------------------------------------------
// Stockham stages
// ----------------------------------------------------------------------------
template <int N, int E, int SI, bool INV, class X, class TW>
__device__ __forceinline__ void fft_stage(float2 (&v)[E], int t, const X& xs, const TW* __restrict__ tw) {
  using P = FFTPlan<N, E>;
  constexpr int R = P::radix(SI);
  constexpr int L = P::span(SI);
  constexpr int B = E / R;
  constexpr int T = P::T;
  constexpr bool LAST = (SI == P::S - 1);
  constexpr int OFF = P::tw_offset(SI);
#pragma unroll
  for (int q = 0; q < B; ++q) {
    const int b = t + T * q;
    const int k = b & (L - 1);
    float2 a[R];
#pragma unroll
    for (int j = 0; j < R; ++j) a[j] = v[q + B * j];
    if constexpr (L > 1) {
#pragma unroll
      for (int j = 1; j < R; ++j) {
        a[j] = tw_mul<INV>(a[j], tw[OFF + (j - 1) * L + k]);
      }
    }
    dft<R, INV>(a);
#pragma unroll
    for (int m = 0; m < R; ++m) v[q + B * m] = a[m];
  }
  if constexpr (!LAST) {
    xs.sync();  // every thread has finished reading the previous contents
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int b = t + T * q;
      const int k = b & (L - 1);
      const int base = (b - k) * R + k;
#pragma unroll
      for (int m = 0; m < R; ++m) xs.st2(base, m * L, v[q + B * m]);
    }
    xs.sync();
#pragma unroll
    for (int e = 0; e < E; ++e) v[e] = xs.ld2(t, T * e);
  }
}

// TW: float4 (hi + lo) or float2 (hi only) stage-twiddle table
template <int N, int E, bool INV, class X, int SI = 0, class TW>
__device__ __forceinline__ void fft(float2 (&v)[E], int t, const X& xs, const TW* __restrict__ tw) {
  if constexpr (SI < FFTPlan<N, E>::S) {
    fft_stage<N, E, SI, INV>(v, t, xs, tw);
    fft<N, E, INV, X, SI + 1>(v, t, xs, tw);
  }
}

}  // namespace wap
