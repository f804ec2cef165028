// C ABI of libwap.so: plans, dispatch of the multislice passes, transfer
// functions.  See include/wap.h for the contract of every entry point.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/wap.h"
#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

// ----------------------------------------------------------------------------
// errors
// ----------------------------------------------------------------------------
static thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  return fail(WAP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

void clear_error() { g_err.clear(); }
const char* last_error() { return g_err.c_str(); }

// ----------------------------------------------------------------------------
// physics scalars (propagation.py:14-81), float64 on the host
// ----------------------------------------------------------------------------
Physics physics(double energy, double dz) {
  const double h = 6.626070040e-34, c = 299792458.0, me = 9.10938356e-31, e = 1.6021766208e-19;
  Physics p;
  p.e0 = me * c * c / e;
  p.lambda = h * c / std::sqrt(energy * (2 * me * c * c / e + energy)) / e * 1.0e10;
  p.ri_a = 2 * p.e0 + 2 * energy;
  p.ri_inv_den = 1.0 / (energy * (2 * p.e0 + energy));
  p.kphase = 2 * M_PI * dz / p.lambda;
  p.k0 = 2 * M_PI / p.lambda;
  p.e_plus_e0 = energy + p.e0;
  return p;
}

// ----------------------------------------------------------------------------
// twiddle tables: per Stockham stage s >= 1, W_{L R}^{j k} for j = 1 .. R-1
// laid out [j-1][k] (row j = 0 is all ones and is not stored), each float64
// value stored as float hi + lo parts (re_hi, im_hi, re_lo, im_lo)
// ----------------------------------------------------------------------------
std::vector<float4> twiddle_table(int n, int e) {
  const PlanShape p = make_plan_shape(n, e);
  std::vector<float4> tw(p.tw_size(), make_float4(1.f, 0.f, 0.f, 0.f));
  for (int s = 1; s < p.stages; ++s) {
    const int R = p.radix(s), L = p.span(s), off = p.tw_offset(s);
    const long long LR = (long long)L * R;
    for (int j = 1; j < R; ++j)
      for (int k = 0; k < L; ++k) {
        const long long m = ((long long)j * k) % LR;
        const double ang = -2.0 * M_PI * (double)m / (double)LR;
        const double c = std::cos(ang), sn = std::sin(ang);
        const float ch = (float)c, sh = (float)sn;
        tw[off + (j - 1) * L + k] = make_float4(ch, sh, (float)(c - (double)ch), (float)(sn - (double)sh));
      }
  }
  return tw;
}

// ----------------------------------------------------------------------------
// launch helpers: one template instance per (size, elements per thread)
// ----------------------------------------------------------------------------
template <class K>
static cudaError_t prep_smem(K kern, size_t smem) {
  if (smem > 48 * 1024) return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  return cudaSuccess;
}

template <int N, int E>
size_t row_smem_bytes(int rows, int extra_bytes) {
  return (size_t)rows * RowCfg<N, E>::PADN * sizeof(float2) + FFTPlan<N, E>::TW_SIZE * sizeof(float4) + extra_bytes;
}

template <int N, int E>
size_t col_smem_bytes(int w, int extra_bytes) {
  return (size_t)N * w * sizeof(float2) + FFTPlan<N, E>::TW_SIZE * sizeof(float4) + extra_bytes;
}

// Row and column passes go out with programmatic dependent launch (the
// kernels wait for their predecessor first thing): in a chain of short,
// latency-bound passes the next pass is already resident when one finishes
// (C1 0.26 -> 0.19 ms per call).  The WPM passes launch normally: their large
// CTAs parked early cost more than the launch latency saved (C3 12.5 vs 13.1 ms).
template <class K, class A>
static cudaError_t launch_pdl(K kern, dim3 grid, int threads, size_t smem, cudaStream_t st, const A& args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, args);
}

template <int N, int E>
static cudaError_t launch_row_t(const RowArgs& a, int nb, int rows, cudaStream_t st) {
  const size_t smem = row_smem_bytes<N, E>(rows, 0);
  cudaError_t err = prep_smem(row_pass_kernel<N, E>, smem);
  if (err != cudaSuccess) return err;
  count_launch();
  return launch_pdl(row_pass_kernel<N, E>, dim3(a.ny / rows, nb), rows * FFTPlan<N, E>::T, smem, st, a);
}

template <int N, int E>
static cudaError_t launch_col_t(const ColArgs& a, int nb, int w, cudaStream_t st) {
  const size_t smem = col_smem_bytes<N, E>(w, 0);
  const dim3 grid(a.nx / w, nb);
  const int threads = w * FFTPlan<N, E>::T;
  cudaError_t err;
  count_launch();
  if (a.flags & COL_SEED) {
    if ((err = prep_smem(col_pass_kernel<N, E, true>, smem)) != cudaSuccess) return err;
    return launch_pdl(col_pass_kernel<N, E, true>, grid, threads, smem, st, a);
  }
  if ((err = prep_smem(col_pass_kernel<N, E, false>, smem)) != cudaSuccess) return err;
  return launch_pdl(col_pass_kernel<N, E, false>, grid, threads, smem, st, a);
}

template <int N, int E>
static cudaError_t launch_wpm_col_t(const WpmColArgs& a, int nb, int w, cudaStream_t st) {
  const size_t smem = col_smem_bytes<N, E>(w, a.K * (int)sizeof(float));
  cudaError_t err = prep_smem(wpm_col_kernel<N, E>, smem);
  if (err != cudaSuccess) return err;
  count_launch();
  const int groups = a.dp_mode ? 1 : (a.K + a.kpg - 1) / a.kpg;
  wpm_col_kernel<N, E><<<dim3(a.nx / w, nb, groups), w * FFTPlan<N, E>::T, smem, st>>>(a);
  return cudaGetLastError();
}

template <int N, int E>
static cudaError_t launch_wpm_row_t(const WpmRowArgs& a, int nb, int rows, cudaStream_t st) {
  const int extra = a.K * (int)sizeof(float) + ((a.K + 31) / 32) * (int)sizeof(unsigned);
  const size_t smem = row_smem_bytes<N, E>(rows, extra);
  cudaError_t err = prep_smem(wpm_row_kernel<N, E>, smem);
  if (err != cudaSuccess) return err;
  count_launch();
  const int groups = a.blend ? (a.K - 1 + a.kpg - 1) / a.kpg : 1;
  wpm_row_kernel<N, E><<<dim3(a.ny / rows, nb, groups), rows * FFTPlan<N, E>::T, smem, st>>>(a);
  return cudaGetLastError();
}

// resident CTAs per SM of the WPM kernels at a launch shape (0 on error)
template <int N, int E>
static int occ_wpm_col_t(int w, int K) {
  const size_t smem = col_smem_bytes<N, E>(w, K * (int)sizeof(float));
  int n = 0;
  if (prep_smem(wpm_col_kernel<N, E>, smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wpm_col_kernel<N, E>, w * FFTPlan<N, E>::T, smem) !=
      cudaSuccess)
    return 0;
  return n;
}

template <int N, int E>
static int occ_wpm_row_t(int rows, int K) {
  const int extra = K * (int)sizeof(float) + ((K + 31) / 32) * (int)sizeof(unsigned);
  const size_t smem = row_smem_bytes<N, E>(rows, extra);
  int n = 0;
  if (prep_smem(wpm_row_kernel<N, E>, smem) != cudaSuccess) return 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, wpm_row_kernel<N, E>, rows * FFTPlan<N, E>::T, smem) !=
      cudaSuccess)
    return 0;
  return n;
}

#define WAP_SIZE_CASES(M, E) \
  M(32, E) M(64, E) M(128, E) M(256, E) M(512, E) M(1024, E) M(2048, E)

#define WAP_DISPATCH(FN, n, e, ...)                                     \
  do {                                                                  \
    switch ((e) * 100000 + (n)) {                                       \
      WAP_SIZE_CASES(WAP_CASE_##FN, 8)                                  \
      WAP_SIZE_CASES(WAP_CASE_##FN, 16)                                 \
      default: return cudaErrorInvalidValue;                            \
    }                                                                   \
  } while (0)

// the row and column passes also come with 4 elements per thread (grids up to
// 1024): short per-thread chains for calls of one or two probes, whose few
// CTAs per pass are latency-bound
#define WAP_SIZE_CASES_E4(M) M(32, 4) M(64, 4) M(128, 4) M(256, 4) M(512, 4) M(1024, 4)
#define WAP_DISPATCH_RC(FN, n, e)                                       \
  do {                                                                  \
    switch ((e) * 100000 + (n)) {                                       \
      WAP_SIZE_CASES_E4(WAP_CASE_##FN)                                  \
      WAP_SIZE_CASES(WAP_CASE_##FN, 8)                                  \
      WAP_SIZE_CASES(WAP_CASE_##FN, 16)                                 \
      default: return cudaErrorInvalidValue;                            \
    }                                                                   \
  } while (0)

#define WAP_CASE_row(N, E) case E * 100000 + N: return launch_row_t<N, E>(a, nb, k, st);
#define WAP_CASE_col(N, E) case E * 100000 + N: return launch_col_t<N, E>(a, nb, k, st);
#define WAP_CASE_wcol(N, E) case E * 100000 + N: return launch_wpm_col_t<N, E>(a, nb, k, st);
#define WAP_CASE_wrow(N, E) case E * 100000 + N: return launch_wpm_row_t<N, E>(a, nb, k, st);
#define WAP_CASE_wcolocc(N, E) case E * 100000 + N: return occ_wpm_col_t<N, E>(k, K);
#define WAP_CASE_wrowocc(N, E) case E * 100000 + N: return occ_wpm_row_t<N, E>(k, K);

#define WAP_DISPATCH_INT(FN, n, e)                                      \
  do {                                                                  \
    switch ((e) * 100000 + (n)) {                                       \
      WAP_SIZE_CASES(WAP_CASE_##FN, 8)                                  \
      WAP_SIZE_CASES(WAP_CASE_##FN, 16)                                 \
      default: return 0;                                                \
    }                                                                   \
  } while (0)

cudaError_t launch_row(int n, int e, const RowArgs& a, int nb, int k, cudaStream_t st) { WAP_DISPATCH_RC(row, n, e); }
cudaError_t launch_col(int n, int e, const ColArgs& a, int nb, int k, cudaStream_t st) { WAP_DISPATCH_RC(col, n, e); }
cudaError_t launch_wpm_col(int n, int e, const WpmColArgs& a, int nb, int k, cudaStream_t st) { WAP_DISPATCH(wcol, n, e); }
cudaError_t launch_wpm_row(int n, int e, const WpmRowArgs& a, int nb, int k, cudaStream_t st) { WAP_DISPATCH(wrow, n, e); }
int wpm_col_occupancy(int n, int e, int k, int K) { WAP_DISPATCH_INT(wcolocc, n, e); }
int wpm_row_occupancy(int n, int e, int k, int K) { WAP_DISPATCH_INT(wrowocc, n, e); }

bool size_supported(int n) { return n >= 32 && n <= 2048 && (n & (n - 1)) == 0; }

// rows per row-type CTA: fill kRowThreads, at most the grid height
int rows_per_cta(int nx, int e, int ny) {
  const int T = nx / e;
  int rows = kRowThreads / T;
  if (rows < 1) rows = 1;
  if (rows > ny) rows = ny;
  return rows;
}

// ----------------------------------------------------------------------------
// transfer functions in float64 (propagation.py:102-107, :139-156, :224-228)
// ----------------------------------------------------------------------------
struct TfArgs {
  int kind, n, m, c128;
  double ps0, ps1, z, lambda;
  void* out;
  float2* out_lo;   // complex64 output only: value - (complex64)value, or null
};

// out[i, j], i < n (axis 0, fftfreq(n, ps0)), j < m (axis 1, fftfreq(m, ps1))
__global__ void transfer_kernel(const TfArgs a) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)a.n * a.m) return;
  const int i = (int)(idx / a.m), j = (int)(idx % a.m);
  const double fx = fftfreq_d(i, a.n, a.ps0), fy = fftfreq_d(j, a.m, a.ps1);
  double re, im;
  if (a.kind == WAP_TF_FRESNEL) {
    // exp(i 2 pi z / lam) * exp(-i pi lam z (fx^2 + fy^2)), as two factors
    double s1, c1, s2, c2;
    sincos(2.0 * M_PI / a.lambda * a.z, &s1, &c1);
    sincos(-M_PI * a.lambda * a.z * (fx * fx + fy * fy), &s2, &c2);
    re = c1 * c2 - s1 * s2;
    im = c1 * s2 + s1 * c2;
  } else {
    const double q = 1.0 / (a.lambda * a.lambda) - fx * fx - fy * fy;
    if (q >= 0.0) {
      sincos(2.0 * M_PI * a.z * sqrt(q), &im, &re);
    } else {
      re = exp(-2.0 * M_PI * a.z * sqrt(-q));
      im = 0.0;
    }
  }
  if (a.c128) {
    reinterpret_cast<double2*>(a.out)[idx] = make_double2(re, im);
  } else {
    const float rh = (float)re, ih = (float)im;
    reinterpret_cast<float2*>(a.out)[idx] = make_float2(rh, ih);
    if (a.out_lo) a.out_lo[idx] = make_float2((float)(re - (double)rh), (float)(im - (double)ih));
  }
}

}  // namespace wap

using namespace wap;

// ----------------------------------------------------------------------------
// plan
// ----------------------------------------------------------------------------
static int upload_twiddles(wap_plan* p) {
  for (int which = 0; which < 2; ++which) {
    const int n = which == 0 ? p->nx : p->ny;
    const int e = which == 0 ? p->row_e : p->col_e;
    std::vector<float4> h = twiddle_table(n, e);
    float4*& d = which == 0 ? p->tw_row : p->tw_col;
    if (d) cudaFree(d);
    d = nullptr;
    cudaError_t err = cudaMalloc(&d, h.size() * sizeof(float4));
    if (err != cudaSuccess) return cuda_fail(err, "cudaMalloc(twiddles)");
    err = cudaMemcpy(d, h.data(), h.size() * sizeof(float4), cudaMemcpyHostToDevice);
    if (err != cudaSuccess) return cuda_fail(err, "cudaMemcpy(twiddles)");
  }
  return WAP_OK;
}

static int default_col_w(int ny, int e, int nx) {
  const int T = ny / e;
  int w = 16;
  while (w > 1 && (w * T > kColThreads || (size_t)ny * w * 8 > 96 * 1024)) w >>= 1;
  if (w > nx) w = nx;
  return w;
}

static bool config_valid(const wap_plan* p, int row_e, int col_e, int col_w) {
  // 4 elements per thread: Fresnel/AS passes on grids up to 1024 (the WPM
  // passes come with 8 and 16 only)
  auto e_ok = [&](int e, int n) {
    return e == 8 || e == 16 || (e == 4 && p->op == WAP_OP_FRESNEL_AS && n <= 1024);
  };
  if (!e_ok(row_e, p->nx) || !e_ok(col_e, p->ny)) return false;
  if (p->nx / row_e > kRowThreads) return false;
  if (col_w < 1 || (col_w & (col_w - 1)) || col_w > p->nx) return false;
  if (col_w * (p->ny / col_e) > kColThreads) return false;
  if ((size_t)p->ny * col_w * 8 > 160 * 1024) return false;
  return true;
}

static void plan_free(wap_plan* p) {
  if (!p) return;
  cudaFree(p->tw_row);
  cudaFree(p->tw_col);
  cudaFree(p->fields);
  cudaFree(p->dpbuf);
  cudaFree(p->blend);
  cudaFree(p->hvac);
  cudaFree(p->hvac_lo);
  cudaFree(p->ky2);
  cudaFree(p->kx2);
  cudaFree(p->refs);
  cudaFree(p->ttab);
  cudaFree(p->counter);
  cudaFree(p->chain_tw);
  cudaFree(p->chain_count);
  cudaFree(p->chain_status);
  cudaFree(p->cl_tw);
  if (p->generic) {
    generic_axis_free(&p->gen_x);
    generic_axis_free(&p->gen_y);
  }
  delete p;
}

extern "C" {

const char* wap_version(void) { return "wap-b200 0.1 (sm_100a)"; }

const char* wap_last_error(void) { return wap::last_error(); }

int wap_plan_create(wap_plan** out, int ny, int nx, int max_batch, int op, int n_bins) {
  clear_error();
  if (!out) return fail(WAP_ERR_ARG, "plan pointer is NULL");
  *out = nullptr;
  // power-of-two grids in [32, 2048] take the fast path; a grid with another
  // side (17 .. 1024) runs the Bluestein transforms of wap_generic.cu
  const bool generic = !size_supported(ny) || !size_supported(nx);
  auto axis_ok = [](int n) { return size_supported(n) || generic_size_supported(n); };
  if (!axis_ok(ny) || !axis_ok(nx))
    return fail(WAP_ERR_UNSUPPORTED,
                "unsupported grid %d x %d: each axis must be a power of two in [32, 2048] or a size in [17, 1024]", ny,
                nx);
  if (max_batch < 1) return fail(WAP_ERR_ARG, "max_batch must be >= 1 (got %d)", max_batch);
  if (op != WAP_OP_FRESNEL_AS && op != WAP_OP_WPM) return fail(WAP_ERR_ARG, "unknown op %d", op);
  if (op == WAP_OP_WPM && (n_bins < 2 || n_bins > 4096))
    return fail(WAP_ERR_ARG, "n_bins must be in [2, 4096] (got %d)", n_bins);
  wap_plan* p = new wap_plan();
  cudaGetDevice(&p->device);
  p->ny = ny;
  p->nx = nx;
  p->max_batch = max_batch;
  p->op = op;
  p->n_bins = op == WAP_OP_WPM ? n_bins : 0;
  p->row_e = nx >= 64 ? 16 : 8;
  p->col_e = ny >= 64 ? 16 : 8;
  p->col_w = default_col_w(ny, p->col_e, nx);
  p->generic = generic;
  int rc = generic ? generic_axis_create(&p->gen_x, nx) : upload_twiddles(p);
  if (rc == WAP_OK && generic) rc = generic_axis_create(&p->gen_y, ny);
  if (rc != WAP_OK) {
    plan_free(p);   // keeps the failure's message
    return rc;
  }
  if (op == WAP_OP_WPM) {
    const size_t plane = (size_t)ny * nx;
    cudaError_t err = cudaMalloc(&p->fields, (size_t)max_batch * n_bins * plane * sizeof(float2));
    if (err == cudaSuccess) err = cudaMalloc(&p->dpbuf, (size_t)max_batch * plane * sizeof(float2));
    if (err == cudaSuccess) err = cudaMalloc(&p->blend, (size_t)max_batch * plane * sizeof(float2));
    if (err == cudaSuccess) err = cudaMalloc(&p->hvac, plane * sizeof(float2));
    if (err == cudaSuccess) err = cudaMalloc(&p->hvac_lo, plane * sizeof(float2));
    if (err == cudaSuccess) err = cudaMalloc(&p->ky2, ny * sizeof(float));
    if (err == cudaSuccess) err = cudaMalloc(&p->kx2, nx * sizeof(float));
    if (err != cudaSuccess) {
      plan_free(p);
      return cuda_fail(err, "cudaMalloc(WPM workspace)");
    }
  }
  *out = p;
  return WAP_OK;
}

int wap_plan_destroy(wap_plan* p) {
  clear_error();
  plan_free(p);
  return WAP_OK;
}

int wap_plan_set_config(wap_plan* p, int row_e, int col_e, int col_w) {
  clear_error();
  if (!p) return fail(WAP_ERR_ARG, "plan is NULL");
  if (p->generic) return fail(WAP_ERR_UNSUPPORTED, "grids that are not powers of two have a fixed launch shape");
  if (!config_valid(p, row_e, col_e, col_w))
    return fail(WAP_ERR_ARG, "invalid launch configuration row_e=%d col_e=%d col_w=%d for %d x %d", row_e, col_e, col_w,
                p->ny, p->nx);
  p->row_e = row_e;
  p->col_e = col_e;
  p->col_w = col_w;
  return upload_twiddles(p);
}

int wap_plan_set_detector(wap_plan* p, int y0, int x0, int ny, int nx) {
  clear_error();
  if (!p) return fail(WAP_ERR_ARG, "plan is NULL");
  if (ny == 0 && nx == 0) {
    p->det = Detector{};
    return WAP_OK;
  }
  if (ny < 1 || nx < 1 || y0 < 0 || x0 < 0 || y0 + ny > p->ny || x0 + nx > p->nx)
    return fail(WAP_ERR_ARG, "detector window rows %d+%d, columns %d+%d outside the %d x %d grid", y0, ny, x0, nx,
                p->ny, p->nx);
  p->det = Detector{y0, x0, ny, nx};
  return WAP_OK;
}

int wap_plan_get_config(const wap_plan* p, int* row_e, int* col_e, int* col_w) {
  clear_error();
  if (!p || !row_e || !col_e || !col_w) return fail(WAP_ERR_ARG, "NULL argument");
  *row_e = p->row_e;
  *col_e = p->col_e;
  *col_w = p->col_w;
  return WAP_OK;
}

int wap_transfer_function(int kind, int n, int m, double ps0, double ps1, double z, double energy, void* out,
                          int out_c128, void* out_lo, void* stream) {
  clear_error();
  if (!out) return fail(WAP_ERR_ARG, "out is NULL");
  if (kind != WAP_TF_FRESNEL && kind != WAP_TF_ANGULAR) return fail(WAP_ERR_ARG, "unknown transfer function %d", kind);
  if (n < 1 || m < 1) return fail(WAP_ERR_ARG, "bad shape %d x %d", n, m);
  if (!(energy > 0) || !(ps0 > 0) || !(ps1 > 0)) return fail(WAP_ERR_ARG, "energy and sampling must be positive");
  if (out_c128 && out_lo) return fail(WAP_ERR_ARG, "out_lo is only produced with a complex64 out");
  TfArgs a{kind, n, m, out_c128 ? 1 : 0, ps0, ps1, z, physics(energy, 1.0).lambda, out,
           reinterpret_cast<float2*>(out_lo)};
  const long long total = (long long)n * m;
  count_launch();
  transfer_kernel<<<(unsigned)((total + 255) / 256), 256, 0, (cudaStream_t)stream>>>(a);
  cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? WAP_OK : cuda_fail(err, "transfer_kernel");
}

}  // extern "C"

// ----------------------------------------------------------------------------
// Fresnel / angular-spectrum forward
// ----------------------------------------------------------------------------
namespace wap {

int check_common(const wap_plan* p, const float* V, int n_slices, int n_draws, const float* psi0, int n_probes,
                 float* exit) {
  if (!p) return fail(WAP_ERR_ARG, "plan is NULL");
  if (!V || !psi0 || !exit) return fail(WAP_ERR_ARG, "V, psi0 and exit must be non-NULL device pointers");
  if (n_slices < 1) return fail(WAP_ERR_ARG, "need at least one slice (got %d)", n_slices);
  if (n_draws < 1) return fail(WAP_ERR_ARG, "n_draws must be >= 1");
  if (n_probes < 1 || n_probes > p->max_batch)
    return fail(WAP_ERR_ARG, "n_probes=%d outside [1, max_batch=%d]", n_probes, p->max_batch);
  int dev = -1;
  cudaGetDevice(&dev);
  if (dev != p->device) return fail(WAP_ERR_ARG, "plan was created on device %d, current device is %d", p->device, dev);
  return WAP_OK;
}

RowArgs base_row_args(const wap_plan* p, const Physics& ph, const float* V, int n_slices, const int32_t* draw) {
  RowArgs r{};
  r.V = V;
  r.draw = draw;
  r.v_draw_stride = (long long)n_slices * p->ny * p->nx;
  r.tw = p->tw_row;
  r.ny = p->ny;
  r.nx = p->nx;
  r.scale = (float)(1.0 / ((double)p->ny * p->nx));
  r.src_scale = 1.0f;
  r.ri_a = (float)ph.ri_a;
  r.ri_inv_den = (float)ph.ri_inv_den;
  r.kphase = (float)ph.kphase;
  r.e_plus_e0 = (float)ph.e_plus_e0;
  r.tw_ready = 1;   // uploaded at plan creation
  return r;
}

ColArgs base_col_args(const wap_plan* p, const float* H, const float* H_lo) {
  ColArgs c{};
  c.H = reinterpret_cast<const float2*>(H);
  c.H_lo = reinterpret_cast<const float2*>(H_lo);
  c.tw = p->tw_col;
  c.ny = p->ny;
  c.nx = p->nx;
  c.seed_scale = (float)((double)p->ny * p->nx);
  c.det = p->det.resolved(p->ny, p->nx);
  c.tw_ready = 1;
  return c;
}

// algorithmic bytes of one pass over n_probes waves (per pixel: wave in 8,
// wave out 8, potential 4, snapshot 8, forward wave 8, gradient RMW 8; the
// transfer function is counted once per launch)
static double row_bytes(const wap_plan* p, const RowArgs& r, int n_probes) {
  double per = 16;
  if (r.flags & (ROW_TRANS | ROW_ADJOINT)) per += 4;
  if (r.flags & ROW_TRANS_TAB) per += 8;
  if (r.snap) per += 8;
  if (r.flags & ROW_ADJOINT) per += 16;
  return per * (double)p->ny * p->nx * n_probes;
}

static double col_bytes(const wap_plan* p, const ColArgs& c, int n_probes) {
  double per = 16;
  if (c.flags & COL_DP) per += 4;
  if (c.flags & COL_SEED) per += 4 + (c.seed2 ? 8 : 0);
  return per * (double)p->ny * p->nx * n_probes + ((c.flags & COL_NO_H) ? 0.0 : 8.0 * p->ny * p->nx);
}

// batch chunks of at most 65535 probes (grid.y limit)
cudaError_t row_chunks(const wap_plan* p, RowArgs r, int n_probes, cudaStream_t st) {
  const int rows = rows_per_cta(p->nx, p->row_e, p->ny);
  const ProfToken tok = prof_begin(WAP_KIND_ROW, st);
  for (int b0 = 0; b0 < n_probes; b0 += 65535) {
    r.probe0 = b0;
    cudaError_t e = launch_row(p->nx, p->row_e, r, std::min(65535, n_probes - b0), rows, st);
    if (e != cudaSuccess) return e;
  }
  prof_end(tok, st, row_bytes(p, r, n_probes));
  return cudaSuccess;
}

cudaError_t col_chunks(const wap_plan* p, ColArgs c, int n_probes, cudaStream_t st) {
  const ProfToken tok = prof_begin(WAP_KIND_COL, st);
  for (int b0 = 0; b0 < n_probes; b0 += 65535) {
    c.probe0 = b0;
    cudaError_t e = launch_col(p->ny, p->col_e, c, std::min(65535, n_probes - b0), p->col_w, st);
    if (e != cudaSuccess) return e;
  }
  prof_end(tok, st, col_bytes(p, c, n_probes));
  return cudaSuccess;
}

// Whether a call tabulates exp(i phi(V)) (one elementwise kernel, bit for
// bit the values the row pass would compute inline): when several probes see
// each potential slice, and for one probe per draw while the table stays
// within kSmallTransTable bytes of plan workspace - computed by a fully
// occupied elementwise kernel it takes a long serial step out of the
// latency-bound row pass of a single probe (512^2 x 100 slices: 2.07 -> 1.55 ms)
constexpr size_t kSmallTransTable = size_t(1) << 30;
static bool use_trans_table(const wap_plan* p, int n_probes, int n_slices, int n_draws) {
  if (n_probes >= 2 * n_draws) return true;
  return (size_t)n_draws * n_slices * p->ny * p->nx * sizeof(float2) <= kSmallTransTable;
}

// exp(i phi(V)) for every draw and slice into the plan's grow-only table
int build_trans_table(wap_plan* p, const float* V, int n_slices, int n_draws, const RowArgs& r, cudaStream_t st) {
  const size_t need = (size_t)n_draws * n_slices * p->ny * p->nx;
  cudaError_t e = cudaSuccess;
  if (need > p->ttab_cap) {
    cudaFree(p->ttab);
    p->ttab = nullptr;
    p->ttab_cap = 0;
    e = cudaMalloc(&p->ttab, need * sizeof(float2));
    if (e != cudaSuccess) {
      cudaGetLastError();
      return cuda_fail(e, "cudaMalloc(transmission table)");
    }
    p->ttab_cap = need;
  }
  const long long n4 = (long long)need / 4;
  const ProfToken tok = prof_begin(WAP_KIND_TRANS, st);
  count_launch();
  trans_table_kernel<<<(unsigned)std::min<long long>((n4 + 255) / 256, 148LL * 16), 256, 0, st>>>(
      V, p->ttab, n4, r.ri_a, r.ri_inv_den, r.kphase);
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "trans_table_kernel");
  prof_end(tok, st, 12.0 * (double)need);
  return WAP_OK;
}

// Forward multislice; snapshots of the wave entering slice s go to
// snap + (s / snap_every) * plane when s % snap_every == 0 (snap_first = 0:
// checkpoints), or the wave after every slice to stack (snap_first = 1).
int fresnel_forward(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw, const float* psi0,
                    int n_probes, int psi0_per_probe, const int32_t* positions, const float* H, const float* H_lo,
                    double dz,
                    double energy, float* exit, float* dp, float* stack, float* ckpt, int ckpt_every,
                    cudaStream_t st) {
  int rc = check_common(p, V, n_slices, n_draws, psi0, n_probes, exit);
  if (rc) return rc;
  if (!H) return fail(WAP_ERR_ARG, "H must be a non-NULL device pointer");
  if (p->op != WAP_OP_FRESNEL_AS) return fail(WAP_ERR_ARG, "plan was not created for the Fresnel/AS path");
  if (p->generic) {
    if (ckpt)
      return fail(WAP_ERR_UNSUPPORTED, "checkpointed forwards (gradients) need power-of-two grids, got %d x %d", p->ny,
                  p->nx);
    return generic_fresnel_forward(p, V, n_slices, n_draws, draw, psi0, n_probes, psi0_per_probe, positions, H, H_lo,
                                   dz, energy, exit, dp, stack, st);
  }
  const Physics ph = physics(energy, dz);
  const long long plane = (long long)p->ny * p->nx;
  const int nck = ckpt ? (n_slices + ckpt_every - 1) / ckpt_every : 0;

  RowArgs r = base_row_args(p, ph, V, n_slices, draw);
  r.psi = reinterpret_cast<float2*>(exit);
  r.psi_bstride = plane;
  r.src = reinterpret_cast<const float2*>(psi0);
  r.src_bstride = psi0_per_probe ? plane : 0;
  r.shifts = positions;
  ColArgs c = base_col_args(p, H, H_lo);
  c.psi = r.psi;
  c.psi_bstride = plane;
  c.dp = dp;
  p->chain_ran = 0;
  // exp(i phi(V)) tabulated once per (draw, slice) (use_trans_table), else
  // evaluated inline by the row pass.  (The single-probe kernels below take
  // the table too: evaluated inline on the 16 SMs of a cluster it costs more
  // than the table launch on all SMs - 128^2 x 20 slices on B200: 117 us
  // inline against 83 + 9 us.)
  int trans_flag = ROW_TRANS;
  if (use_trans_table(p, n_probes, n_slices, n_draws) && build_trans_table(p, V, n_slices, n_draws, r, st) == WAP_OK) {
    r.ttab = p->ttab;
    trans_flag = ROW_TRANS_TAB;
  } else {
    clear_error();
  }
  // few probes: every slice in one launch when the grid qualifies - the wave
  // held in a thread-block cluster (wap_cluster.cu), else a cooperative grid
  // (wap_chain.cu) - else one launch per pass below
  if (!ckpt) {
    int rc2 = cluster_forward(p, r, c, n_probes, n_slices, reinterpret_cast<float2*>(stack), st);
    if (rc2 != -1) return rc2;
    rc2 = chain_forward(p, r, c, n_probes, n_slices, reinterpret_cast<float2*>(stack), st);
    if (rc2 != -1) return rc2;
  }

  for (int s = 0; s <= n_slices; ++s) {
    r.slice = s;
    r.flags = (s == 0 ? ROW_LOAD_SRC : ROW_IFFT) | (s < n_slices ? (trans_flag | ROW_FFT) : 0);
    r.snap = nullptr;
    if (stack && s >= 1) {
      r.snap = reinterpret_cast<float2*>(stack) + (long long)(s - 1) * plane;
      r.snap_bstride = (long long)n_slices * plane;
    } else if (ckpt && s < n_slices && s % ckpt_every == 0) {
      r.snap = reinterpret_cast<float2*>(ckpt) + (long long)(s / ckpt_every) * plane;
      r.snap_bstride = (long long)nck * plane;
    }
    cudaError_t e = row_chunks(p, r, n_probes, st);
    if (e != cudaSuccess) return cuda_fail(e, "row pass");
    if (s == n_slices) break;
    c.flags = (s == n_slices - 1 && dp) ? COL_DP : 0;
    e = col_chunks(p, c, n_probes, st);
    if (e != cudaSuccess) return cuda_fail(e, "column pass");
  }
  return WAP_OK;
}

}  // namespace wap

extern "C" {

int wap_spectrum_propagate(wap_plan* p, const float* X, int n, const float* H, const float* H_lo, float* out,
                           void* stream) {
  clear_error();
  if (!p || !X || !H || !out) return fail(WAP_ERR_ARG, "NULL argument");
  if (n < 1 || n > p->max_batch) return fail(WAP_ERR_ARG, "n=%d outside 1..%d (plan batch)", n, p->max_batch);
  if (p->generic) return fail(WAP_ERR_UNSUPPORTED, "spectrum propagation needs a power-of-two grid");
  cudaStream_t st = (cudaStream_t)stream;
  const long long plane = (long long)p->ny * p->nx;
  cudaError_t e;
  if (out != X && (e = cudaMemcpyAsync(out, X, (size_t)n * plane * sizeof(float2), cudaMemcpyDeviceToDevice, st)) !=
                      cudaSuccess)
    return cuda_fail(e, "spectrum copy");
  // columns: * H (hi + lo), inverse column FFT (no forward one)
  ColArgs c = base_col_args(p, H, H_lo);
  c.psi = reinterpret_cast<float2*>(out);
  c.psi_bstride = plane;
  c.flags = COL_NO_FFT;
  if ((e = col_chunks(p, c, n, st)) != cudaSuccess) return cuda_fail(e, "spectrum column pass");
  // rows: inverse row FFT and the 1/(ny nx) of ifft2
  RowArgs r{};
  r.psi = reinterpret_cast<float2*>(out);
  r.psi_bstride = plane;
  r.tw = p->tw_row;
  r.ny = p->ny;
  r.nx = p->nx;
  r.flags = ROW_IFFT;
  r.scale = (float)(1.0 / (double)plane);
  r.tw_ready = 1;
  if ((e = row_chunks(p, r, n, st)) != cudaSuccess) return cuda_fail(e, "spectrum row pass");
  return WAP_OK;
}

int wap_multislice_fwd(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw, const float* psi0,
                       int n_probes, int psi0_per_probe, const int32_t* positions, const float* H, const float* H_lo,
                       double dz, double energy, float* exit, float* dp, float* stack, void* stream) {
  clear_error();
  return fresnel_forward(p, V, n_slices, n_draws, draw, psi0, n_probes, psi0_per_probe, positions, H, H_lo, dz, energy,
                         exit, dp, stack, nullptr, 1, (cudaStream_t)stream);
}

int wap_multislice_fwd_ckpt(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw,
                            const float* psi0, int n_probes, int psi0_per_probe, const int32_t* positions,
                            const float* H, const float* H_lo, double dz, double energy, float* exit, float* dp,
                            float* ckpt, int ckpt_every, void* stream) {
  clear_error();
  if (!ckpt) return fail(WAP_ERR_ARG, "ckpt must be a non-NULL device pointer");
  if (ckpt_every < 1) return fail(WAP_ERR_ARG, "ckpt_every must be >= 1");
  return fresnel_forward(p, V, n_slices, n_draws, draw, psi0, n_probes, psi0_per_probe, positions, H, H_lo, dz, energy,
                         exit, dp, nullptr, ckpt, ckpt_every, (cudaStream_t)stream);
}

// ----------------------------------------------------------------------------
// adjoint (gradient w.r.t. V)
// ----------------------------------------------------------------------------
int wap_multislice_bwd(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw, int n_probes,
                       const float* H, const float* H_lo, double dz, double energy, const float* exit, const float* ckpt,
                       int ckpt_every,
                       const float* grad_dp, const float* grad_exit, float* grad_V, float* work, void* stream) {
  clear_error();
  int rc = check_common(p, V, n_slices, n_draws, exit, n_probes, const_cast<float*>(exit));
  if (rc) return rc;
  if (!H || !ckpt || !grad_V || !work) return fail(WAP_ERR_ARG, "H, ckpt, grad_V and work must be non-NULL");
  if (!grad_dp && !grad_exit) return fail(WAP_ERR_ARG, "need grad_dp or grad_exit");
  if (ckpt_every < 1) return fail(WAP_ERR_ARG, "ckpt_every must be >= 1");
  if (p->op != WAP_OP_FRESNEL_AS) return fail(WAP_ERR_ARG, "plan was not created for the Fresnel/AS path");
  if (p->generic) return fail(WAP_ERR_UNSUPPORTED, "gradients need power-of-two grids, got %d x %d", p->ny, p->nx);
  cudaStream_t st = (cudaStream_t)stream;
  const Physics ph = physics(energy, dz);
  const long long plane = (long long)p->ny * p->nx;
  const int k = ckpt_every;
  const int nck = (n_slices + k - 1) / k;
  const long long wstride = (long long)(k + 2) * plane;
  float2* w = reinterpret_cast<float2*>(work);
  float2* lam = w;                 // slot 0: adjoint state
  float2* buf = w + plane;         // slot 1: recompute / seed buffer
  float2* seg = w + 2 * plane;     // slots 2..k+1: psi_s of the segment
  const float2* ck = reinterpret_cast<const float2*>(ckpt);
  cudaError_t e;

  // seed: lambda_psi_N = grad_exit / 2 + F^H (g Z), Z = fft2(exit);
  // lambda_a_{N-1} = ifft2(conj(H) fft2(lambda_psi_N))
  RowArgs r = base_row_args(p, ph, V, n_slices, draw);
  // transmission shared by the probes of a draw, for the recompute and the
  // adjoint passes
  const float2* ttab = nullptr;
  if (use_trans_table(p, n_probes, n_slices, n_draws) && build_trans_table(p, V, n_slices, n_draws, r, st) == WAP_OK)
    ttab = p->ttab;
  else clear_error();
  r.psi = lam;
  r.psi_bstride = wstride;
  r.src = reinterpret_cast<const float2*>(exit);
  r.src_bstride = plane;
  r.flags = ROW_LOAD_SRC | ROW_FFT;
  if ((e = row_chunks(p, r, n_probes, st)) != cudaSuccess) return cuda_fail(e, "seed row pass");
  if (grad_exit) {
    r.psi = buf;
    r.src = reinterpret_cast<const float2*>(grad_exit);
    r.flags = ROW_LOAD_SRC | ROW_FFT | ROW_SCALE_SRC;
    r.src_scale = 0.5f;
    if ((e = row_chunks(p, r, n_probes, st)) != cudaSuccess) return cuda_fail(e, "seed row pass");
    r.src_scale = 1.0f;
  }
  ColArgs c = base_col_args(p, H, H_lo);
  c.psi = lam;
  c.psi_bstride = wstride;
  c.flags = COL_SEED | COL_CONJ_H;
  c.g = grad_dp;
  c.seed2 = grad_exit ? buf : nullptr;
  c.seed2_bstride = wstride;
  if ((e = col_chunks(p, c, n_probes, st)) != cudaSuccess) return cuda_fail(e, "seed column pass");

  for (int j = nck - 1; j >= 0; --j) {
    const int s0 = j * k, s1 = std::min(s0 + k, n_slices);
    // recompute psi_{s0+1} .. psi_{s1-1} from the checkpoint psi_{s0}
    for (int s = s0; s < s1 - 1; ++s) {
      RowArgs q = base_row_args(p, ph, V, n_slices, draw);
      q.psi = buf;
      q.psi_bstride = wstride;
      q.slice = s;
      q.ttab = ttab;
      const int tf = ttab ? ROW_TRANS_TAB : ROW_TRANS;
      if (s == s0) {
        q.src = ck + (long long)j * plane;
        q.src_bstride = (long long)nck * plane;
        q.flags = ROW_LOAD_SRC | tf | ROW_FFT;
      } else {
        q.flags = ROW_IFFT | tf | ROW_FFT;
        q.snap = seg + (long long)(s - s0) * plane;
        q.snap_bstride = wstride;
      }
      if ((e = row_chunks(p, q, n_probes, st)) != cudaSuccess) return cuda_fail(e, "recompute row pass");
      ColArgs cc = base_col_args(p, H, H_lo);
      cc.psi = buf;
      cc.psi_bstride = wstride;
      if ((e = col_chunks(p, cc, n_probes, st)) != cudaSuccess) return cuda_fail(e, "recompute column pass");
    }
    if (s1 - 1 > s0) {
      RowArgs q = base_row_args(p, ph, V, n_slices, draw);
      q.psi = buf;
      q.psi_bstride = wstride;
      q.slice = s1 - 1;
      q.flags = ROW_IFFT;
      q.snap = seg + (long long)(s1 - 1 - s0) * plane;
      q.snap_bstride = wstride;
      if ((e = row_chunks(p, q, n_probes, st)) != cudaSuccess) return cuda_fail(e, "recompute row pass");
    }
    // adjoint sweep s1-1 .. s0
    for (int s = s1 - 1; s >= s0; --s) {
      RowArgs a = base_row_args(p, ph, V, n_slices, draw);
      a.psi = lam;
      a.psi_bstride = wstride;
      a.slice = s;
      a.flags = ROW_IFFT | ROW_ADJOINT | (s > 0 ? ROW_FFT : 0);
      if (s == s0) {
        a.aux = ck + (long long)j * plane;
        a.aux_bstride = (long long)nck * plane;
      } else {
        a.aux = seg + (long long)(s - s0) * plane;
        a.aux_bstride = wstride;
      }
      a.grad = grad_V;
      a.ttab = ttab;
      if ((e = row_chunks(p, a, n_probes, st)) != cudaSuccess) return cuda_fail(e, "adjoint row pass");
      if (s == 0) break;
      ColArgs ca = base_col_args(p, H, H_lo);
      ca.psi = lam;
      ca.psi_bstride = wstride;
      ca.flags = COL_CONJ_H;
      if ((e = col_chunks(p, ca, n_probes, st)) != cudaSuccess) return cuda_fail(e, "adjoint column pass");
    }
  }
  return WAP_OK;
}

}  // extern "C"
