// WPM adaptive-binning forward (propagation.py:215-256, :358-387).
//
// Launch sequence for N slices, all in place on the caller's exit buffer:
//   wpm_bins_kernel            reference deltas of every slice (one launch)
//   row pass  (load, FFT)      psi0 -> row spectrum
//   for s in 0..N-1:
//     wpm_col_kernel  s        column FFT, K x (propagate, column IFFT) -> fields
//     wpm_row_kernel  s        K x row IFFT, smoothstep blend -> wave after slice s,
//                              then its row FFT (input of slice s+1)
//   wpm_col_kernel (dp mode)   |fftshift(fft2(exit))|^2
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "wap_internal.h"
#include "wap_passes.cuh"

namespace wap {

// WPM vacuum propagator exp(i dz sqrt_c(k0^2 - k_perp^2)) in float64 on the
// 'xy' meshgrid of propagation.py:224-228 (rows: ky = 2 pi fftfreq(ny, dy)),
// rounded once to complex64, plus the float32 tables (2 pi f)^2 per axis.
struct HvacArgs {
  int ny, nx;
  double dy, dx, dz, k0;
  float2* hvac;
  float2* hvac_lo;
  float* ky2;
  float* kx2;
};

__global__ void wpm_vacuum_kernel(const HvacArgs a) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)a.ny * a.nx) return;
  const int iy = (int)(idx / a.nx), ix = (int)(idx % a.nx);
  const double ky = 2.0 * M_PI * fftfreq_d(iy, a.ny, a.dy);
  const double kx = 2.0 * M_PI * fftfreq_d(ix, a.nx, a.dx);
  const double q = a.k0 * a.k0 - (kx * kx + ky * ky);
  double re, im;
  if (q >= 0.0) {
    sincos(a.dz * sqrt(q), &im, &re);
  } else {
    re = exp(-a.dz * sqrt(-q));
    im = 0.0;
  }
  const float rh = (float)re, ih = (float)im;
  a.hvac[idx] = make_float2(rh, ih);
  a.hvac_lo[idx] = make_float2((float)(re - (double)rh), (float)(im - (double)ih));
  if (ix == 0) a.ky2[iy] = (float)(ky * ky);
  if (iy == 0) a.kx2[ix] = (float)(kx * kx);
}

}  // namespace wap

using namespace wap;

extern "C" int wap_wpm_fwd(wap_plan* p, const float* V, int n_slices, int n_draws, const int32_t* draw,
                           const float* psi0, int n_probes, int psi0_per_probe, const int32_t* positions, double dz,
                           double energy, double sampling_y, double sampling_x, double power_spacing, float* exit,
                           float* dp, float* stack, void* stream) {
  clear_error();
  int rc = check_common(p, V, n_slices, n_draws, psi0, n_probes, exit);
  if (rc) return rc;
  if (p->op != WAP_OP_WPM) return fail(WAP_ERR_ARG, "plan was not created for the WPM path");
  if (!(sampling_y > 0) || !(sampling_x > 0)) return fail(WAP_ERR_ARG, "sampling must be positive");
  if (!(power_spacing > 0)) return fail(WAP_ERR_ARG, "power_spacing must be positive");
  cudaStream_t st = (cudaStream_t)stream;
  const Physics ph = physics(energy, dz);
  const int K = p->n_bins;
  const long long plane = (long long)p->ny * p->nx;
  cudaError_t e;

  const size_t need = (size_t)n_draws * n_slices * K;
  if (need > p->refs_cap) {
    cudaFree(p->refs);
    p->refs = nullptr;
    p->refs_cap = 0;
    if ((e = cudaMalloc(&p->refs, need * sizeof(float))) != cudaSuccess) return cuda_fail(e, "cudaMalloc(refs)");
    p->refs_cap = need;
  }
  const double key[4] = {sampling_y, sampling_x, dz, energy};
  if (!std::equal(key, key + 4, p->hvac_key)) {
    HvacArgs h{p->ny, p->nx, sampling_y, sampling_x, dz, ph.k0, p->hvac, p->hvac_lo, p->ky2, p->kx2};
    count_launch();
    wpm_vacuum_kernel<<<(unsigned)((plane + 255) / 256), 256, 0, st>>>(h);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "wpm_vacuum_kernel");
    std::copy(key, key + 4, p->hvac_key);
  }
  if (p->generic)
    return generic_wpm_forward(p, V, n_slices, n_draws, draw, psi0, n_probes, psi0_per_probe, positions, dz, energy,
                               sampling_y, sampling_x, power_spacing, exit, dp, stack, st);

  WpmBinsArgs bargs{V, p->refs, (int)plane, n_slices, K, (float)ph.ri_a, (float)ph.ri_inv_den, power_spacing};
  {
    const ProfToken tok = prof_begin(WAP_KIND_WPM_BINS, st);
    count_launch();
    wpm_bins_kernel<<<dim3(n_slices, n_draws), 1024, 0, st>>>(bargs);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "wpm_bins_kernel");
    prof_end(tok, st, 4.0 * plane * n_slices * n_draws);
  }

  // psi0 -> row spectrum
  RowArgs r = base_row_args(p, ph, V, n_slices, draw);
  r.psi = reinterpret_cast<float2*>(exit);
  r.psi_bstride = plane;
  r.src = reinterpret_cast<const float2*>(psi0);
  r.src_bstride = psi0_per_probe ? plane : 0;
  r.shifts = positions;
  r.flags = ROW_LOAD_SRC | ROW_FFT;
  if ((e = row_chunks(p, r, n_probes, st)) != cudaSuccess) return cuda_fail(e, "row pass");

  WpmColArgs c{};
  c.psi = reinterpret_cast<const float2*>(exit);
  c.fields = p->fields;
  c.hvac = p->hvac;
  c.hvac_lo = p->hvac_lo;
  c.ky2 = p->ky2;
  c.kx2 = p->kx2;
  c.refs = p->refs;
  c.draw = draw;
  c.tw = p->tw_col;
  c.ny = p->ny;
  c.nx = p->nx;
  c.K = K;
  c.n_slices = n_slices;
  c.k02 = (float)(ph.k0 * ph.k0);
  c.dz = (float)dz;
  c.det = p->det.resolved(p->ny, p->nx);

  WpmRowArgs w{};
  w.psi = reinterpret_cast<float2*>(exit);
  w.fields = p->fields;
  w.dpbuf = p->dpbuf;
  w.dpbuf_bstride = plane;
  w.V = V;
  w.draw = draw;
  w.v_draw_stride = (long long)n_slices * plane;
  w.refs = p->refs;
  w.tw = p->tw_row;
  w.ny = p->ny;
  w.nx = p->nx;
  w.K = K;
  w.n_slices = n_slices;
  w.scale = (float)(1.0 / (double)plane);
  w.ri_a = (float)ph.ri_a;
  w.ri_inv_den = (float)ph.ri_inv_den;
  w.snap_bstride = (long long)n_slices * plane;
  const int rows = rows_per_cta(p->nx, p->row_e, p->ny);

  // Few probes leave most SMs idle (a 512^2 probe is 128 column and 128 row
  // CTAs): then the K bins are split across CTA groups - each column CTA
  // redoes the column FFT for its share of the bins, each row CTA blends the
  // pixels whose left bin is in its share, and a row pass applies the row FFT.
  // The group count minimises (waves of resident CTAs) x (transforms per CTA).
  int sms = 0;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
  const int col_slots = std::max(1, wpm_col_occupancy(p->ny, p->col_e, p->col_w, K)) * sms;
  const int row_slots = std::max(1, wpm_row_occupancy(p->nx, p->row_e, rows, K)) * sms;
  // Bins per group (the launched group count is ceil(units / per)).  Column
  // CTA: 1 + per transforms; row CTA: K transforms unsplit, else per + 1 and
  // the row pass that follows (counted as one more).
  auto best_per = [&](long long ctas0, int slots, int units, bool col) {
    int best = units;
    double best_cost = 1e300;
    for (int per = units; per >= 1; --per) {
      const long long g = (units + per - 1) / per;
      const double waves = std::ceil((double)(ctas0 * g) / slots);
      const double work = col ? 1.0 + per : (g == 1 ? (double)K : per + 2.0);
      if (waves * work < best_cost) {
        best_cost = waves * work;
        best = per;
      }
    }
    return best;
  };

  for (int b0 = 0; b0 < n_probes; b0 += 65535) {
    const int nb = std::min(65535, n_probes - b0);
    c.probe0 = b0;
    w.probe0 = b0;
    c.kpg = best_per((long long)(p->nx / p->col_w) * nb, col_slots, K, true);
    w.kpg = best_per((long long)(p->ny / rows) * nb, row_slots, K - 1, false);
    const int gr = (K - 1 + w.kpg - 1) / w.kpg;
    w.blend = gr > 1 ? p->blend : nullptr;
    RowArgs fin = base_row_args(p, ph, V, n_slices, draw);   // the row FFT after a bin-split blend
    fin.src = p->blend;
    fin.src_bstride = plane;
    fin.shifts = nullptr;
    fin.flags = ROW_LOAD_SRC | ROW_FFT;
    for (int s = 0; s < n_slices; ++s) {
      c.slice = s;
      c.dp_mode = 0;
      ProfToken tok = prof_begin(WAP_KIND_WPM_COL, st);
      if ((e = launch_wpm_col(p->ny, p->col_e, c, nb, p->col_w, st)) != cudaSuccess) return cuda_fail(e, "wpm column pass");
      // wave in, K fields out, vacuum propagator once
      prof_end(tok, st, (8.0 + 8.0 * K) * plane * nb + 8.0 * plane);
      w.slice = s;
      w.last = (s == n_slices - 1);
      w.snap = stack ? reinterpret_cast<float2*>(stack) + (long long)s * plane : nullptr;
      tok = prof_begin(WAP_KIND_WPM_ROW, st);
      if ((e = launch_wpm_row(p->nx, p->row_e, w, nb, rows, st)) != cudaSuccess) return cuda_fail(e, "wpm row pass");
      // K fields in, potential, wave out (+ dp buffer on the last slice, + snapshot)
      prof_end(tok, st, (8.0 * K + 4.0 + 8.0 + (w.last ? 8.0 : 0.0) + (w.snap ? 8.0 : 0.0)) * plane * nb);
      if (w.blend) {
        // row FFT of the blended wave; the spatial wave is this slice's snapshot
        // (at the last slice: the exit wave, the transform going to the dp buffer)
        fin.probe0 = b0;
        fin.psi = w.last ? p->dpbuf : reinterpret_cast<float2*>(exit);
        fin.psi_bstride = plane;
        fin.snap = w.last ? reinterpret_cast<float2*>(exit) : w.snap;
        fin.snap_bstride = w.last ? plane : (long long)n_slices * plane;
        if ((e = launch_row(p->nx, p->row_e, fin, nb, rows, st)) != cudaSuccess) return cuda_fail(e, "wpm row FFT");
        if (w.last && w.snap &&
            (e = cudaMemcpy2DAsync(w.snap + (long long)b0 * n_slices * plane, (size_t)n_slices * plane * sizeof(float2),
                                   reinterpret_cast<float2*>(exit) + (long long)b0 * plane, plane * sizeof(float2),
                                   plane * sizeof(float2), nb, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
          return cuda_fail(e, "wpm last snapshot");
      }
    }
    if (dp) {
      WpmColArgs d = c;
      d.psi = p->dpbuf;
      d.dp = dp;
      d.dp_mode = 1;
      const ProfToken tok = prof_begin(WAP_KIND_WPM_COL, st);
      if ((e = launch_wpm_col(p->ny, p->col_e, d, nb, p->col_w, st)) != cudaSuccess) return cuda_fail(e, "wpm dp pass");
      prof_end(tok, st, 12.0 * plane * nb);
    }
  }
  return WAP_OK;
}
