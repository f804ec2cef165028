// Internal declarations shared by the libwap.so translation units.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "../../include/wap.h"

namespace wap {
// Detector window of a diffraction pattern: rows y0 .. y0+ny-1 and columns
// x0 .. x0+nx-1 of the fftshifted |fft2(psi)|^2 - the centre crop of
// downsample_to_max_angle (propagation.py:424-439).  A plan keeps ny == 0 for
// "the whole grid"; kernels always receive a resolved window.
struct Detector {
  int y0 = 0, x0 = 0, ny = 0, nx = 0;
  __host__ __device__ Detector resolved(int gy, int gx) const { return ny == 0 ? Detector{0, 0, gy, gx} : *this; }
  // pixels of one probe's pattern
  __host__ __device__ long long plane() const { return (long long)ny * nx; }
};

// One axis of a grid that is not a power of two (wap_generic.cu): a length-n
// DFT as Bluestein's chirp convolution through an m-point FFT (m the power of
// two >= 2n - 1), or, for a power-of-two axis of such a grid, the plain
// n-point FFT (m = n, blue = 0).  Device pointers; tables of float64 values
// stored as float hi + lo parts.
struct GenAxis {
  int n = 0, m = 0, e = 16, blue = 0;
  const float4* tw = nullptr;       // twiddles of the m-point FFT
  const float4* chirp = nullptr;    // (n) w_p = exp(-i pi p^2 / n)
  const float4* bhat_f = nullptr;   // (m) fft_m(b) / m, b_q = conj(w_q) on the circular index range
  const float4* bhat_i = nullptr;   // (m) fft_m(conj(b)) / m
};
}  // namespace wap

struct wap_plan {
  int device = 0;
  int ny = 0, nx = 0, max_batch = 0, op = 0, n_bins = 0;
  int row_e = 16, col_e = 16, col_w = 16;   // FFT launch shape (autotuned)
  float4* tw_row = nullptr;                 // twiddles for nx / row_e (hi, lo)
  float4* tw_col = nullptr;                 // twiddles for ny / col_e (hi, lo)
  // WPM workspace
  float2* fields = nullptr;                 // (max_batch, n_bins, ny, nx)
  float2* dpbuf = nullptr;                  // (max_batch, ny, nx)
  float2* blend = nullptr;                  // (max_batch, ny, nx) WPM bin-split blend
  float2* hvac = nullptr;                   // (ny, nx) hi part
  float2* hvac_lo = nullptr;                // (ny, nx) lo part
  float* ky2 = nullptr;
  float* kx2 = nullptr;
  double hvac_key[4] = {0, 0, 0, 0};        // (dy, dx, dz, energy) of hvac
  float* refs = nullptr;                    // (draws, n_slices, n_bins)
  size_t refs_cap = 0;
  float2* ttab = nullptr;                   // transmission table (draws, n_slices, ny, nx)
  size_t ttab_cap = 0;
  wap::Detector det;                        // diffraction-pattern window (wap_plan_set_detector)
  unsigned long long* counter = nullptr;    // probe builder: aperture pixel count (allocated on first use)
  // a grid with an axis that is not a power of two: Bluestein transforms
  bool generic = false;
  wap::GenAxis gen_x, gen_y;                // along x (rows) and y (columns)
  // one-launch chain of a single probe (wap_chain.cu): its twiddle table,
  // grid-barrier counter and status word (allocated on first use)
  float4* chain_tw = nullptr;
  int chain_e = 0;
  unsigned* chain_count = nullptr;
  int* chain_status = nullptr;
  int chain_ran = 0;                 // the last forward on this plan ran the chain kernel
  // cluster kernel (wap_cluster.cu): its (n, E) twiddle table, and whether the
  // device co-schedules a cluster of it (-1 not asked yet)
  float4* cl_tw = nullptr;
  int cl_e = 0;
  int cl_fits = -1;
};

namespace wap {

struct Physics {
  double e0, lambda, ri_a, ri_inv_den, kphase, k0, e_plus_e0;
};

Physics physics(double energy, double dz);
std::vector<float4> twiddle_table(int n, int e);

int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);
void clear_error();
const char* last_error();

int check_common(const wap_plan* p, const float* V, int n_slices, int n_draws, const float* psi0, int n_probes,
                 float* exit);
int rows_per_cta(int nx, int e, int ny);
bool size_supported(int n);

struct RowArgs;
struct ColArgs;
struct WpmColArgs;
struct WpmRowArgs;
cudaError_t launch_row(int n, int e, const RowArgs& a, int nb, int k, cudaStream_t st);
cudaError_t launch_col(int n, int e, const ColArgs& a, int nb, int k, cudaStream_t st);
cudaError_t launch_wpm_col(int n, int e, const WpmColArgs& a, int nb, int k, cudaStream_t st);
cudaError_t launch_wpm_row(int n, int e, const WpmRowArgs& a, int nb, int k, cudaStream_t st);
// resident CTAs per SM of the WPM column (k = columns per CTA) and row (k = rows per CTA) kernels
int wpm_col_occupancy(int n, int e, int k, int K);
int wpm_row_occupancy(int n, int e, int k, int K);
cudaError_t row_chunks(const wap_plan* p, RowArgs r, int n_probes, cudaStream_t st);
cudaError_t col_chunks(const wap_plan* p, ColArgs c, int n_probes, cudaStream_t st);

// scheduler / chain overrides (wap_scan_debug_override), -1: default
int knob_value(int which);
// one-launch chain of a single probe (wap_chain.cu); returns -1 when the
// plan or the call does not qualify (the caller then launches per pass)
int chain_forward(wap_plan* p, const RowArgs& r, const ColArgs& c, int n_probes, int n_slices, float2* stack,
                  cudaStream_t st);
int cluster_forward(wap_plan* p, const RowArgs& r, const ColArgs& c, int n_probes, int n_slices, float2* stack,
                    cudaStream_t st);

// grids that are not powers of two (wap_generic.cu)
bool generic_size_supported(int n);
int generic_axis_create(GenAxis* ax, int n);
void generic_axis_free(GenAxis* ax);
int generic_fresnel_forward(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw,
                            const float* psi0, int n_probes, int psi0_per_probe, const int32_t* positions,
                            const float* H, const float* H_lo, double dz, double energy, float* exit, float* dp,
                            float* stack, cudaStream_t st);
int generic_wpm_forward(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw,
                        const float* psi0, int n_probes, int psi0_per_probe, const int32_t* positions, double dz,
                        double energy, double sampling_y, double sampling_x, double power_spacing, float* exit,
                        float* dp, float* stack, cudaStream_t st);
ColArgs base_col_args(const wap_plan* p, const float* H, const float* H_lo);
RowArgs base_row_args(const wap_plan* p, const Physics& ph, const float* V, int n_slices, const int32_t* draw);
int build_trans_table(wap_plan* p, const float* V, int n_slices, int n_draws, const RowArgs& r, cudaStream_t st);

// kernel-level tracing (wap_prof.cu)
struct ProfToken {
  bool active;
  int kind;
  cudaEvent_t a, b;
};
ProfToken prof_begin(int kind, cudaStream_t st);
void count_launch();  // every kernel launch of the library bumps wap_launch_count()
void prof_end(const ProfToken& t, cudaStream_t st, double bytes);

}  // namespace wap
