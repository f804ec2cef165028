/*
 * wap.h - C ABI of the B200 multislice library (libwap.so).
 *
 * Replaces the device work of the reference's Python multislice path
 * (wide_angle_propagation/propagation.py).  Plain pointers and sizes only:
 * every array argument is a CUDA device pointer unless stated otherwise,
 * complex arrays are interleaved (re, im) float32 ("complex64") or float64
 * ("complex128") in C order, and `stream` is a cudaStream_t passed as void*.
 * All calls are stream-ordered and return 0 on success or a negative
 * WAP_ERR_* code; wap_last_error() gives the message of the calling thread's
 * last failure.  Nothing allocated by the caller is freed by the library and
 * vice versa.  A plan is not thread-safe: use one plan per host thread.
 */
#ifndef WAP_H_
#define WAP_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define WAP_OK 0
#define WAP_ERR_ARG (-1)          /* bad argument (null pointer, size, ...) */
#define WAP_ERR_UNSUPPORTED (-2)  /* grid size the kernels do not implement */
#define WAP_ERR_CUDA (-3)         /* CUDA runtime error */
#define WAP_ERR_TIMEOUT (-4)      /* device-side bounded wait expired */

#define WAP_OP_FRESNEL_AS 0       /* simulate_fresnel_as path */
#define WAP_OP_WPM 1              /* simulate_wpm path */

#define WAP_TF_FRESNEL 0          /* fresnel_propagation_kernel */
#define WAP_TF_ANGULAR 1          /* angular_spectrum_propagation_kernel */

typedef struct wap_plan wap_plan;

/* Version / build information string. */
const char* wap_version(void);

/* Message of the calling thread's last failed call ("" if none). */
const char* wap_last_error(void);

/* Create a plan for ny x nx grids and up to max_batch probes per call.  Sides
 * that are powers of two in [32, 2048] take the fast kernels; a grid with
 * another side (any n in [17, 1024]) runs Bluestein transforms through the
 * same FFT core (wap_multislice_fwd and wap_wpm_fwd only; the checkpointed
 * forward, the adjoint, wap_spectrum_propagate and wap_aperture_probe return
 * WAP_ERR_UNSUPPORTED for such plans).  op is WAP_OP_*; n_bins is the WPM bin count
 * (ignored for WAP_OP_FRESNEL_AS).  Allocates twiddle tables and, for WPM,
 * the per-probe reference-field workspace on the current device.
 * Replaces the per-call setup implicit in propagation.py:305 / :358. */
int wap_plan_create(wap_plan** plan, int ny, int nx, int max_batch, int op, int n_bins);

/* Release a plan and everything it allocated. */
int wap_plan_destroy(wap_plan* plan);

/* Status of the plan's last one-launch chain (single-probe forwards run all
 * slices in one cooperative kernel whose grid-wide waits are bounded): a copy
 * of the status word (0 or WAP_ERR_TIMEOUT) into host_status, pinned host
 * memory, enqueued on `stream`; valid once the stream reaches it.  No
 * counterpart in the reference. */
int wap_plan_status_async(wap_plan* plan, int* host_status, void* stream);
/* *pending = 1 when the last wap_multislice_fwd on this plan ran the one-launch
 * chain (so wap_plan_status_async has a status to report), else 0 (the
 * cluster kernel and the per-pass launches have no device-side waits).  Host
 * only.  No counterpart in the reference. */
int wap_plan_status_pending(wap_plan* plan, int* pending);

/* FFT launch shape of the row pass (elements per thread) and column pass
 * (elements per thread, columns per CTA); set by the autotuner.  Elements
 * per thread: 8 or 16, and 4 for Fresnel/AS plans on grids up to 1024;
 * WAP_ERR_ARG for a shape the kernels cannot launch. */
int wap_plan_set_config(wap_plan* plan, int row_e, int col_e, int col_w);
int wap_plan_get_config(const wap_plan* plan, int* row_e, int* col_e, int* col_w);

/* Detector window of the diffraction pattern for the plan's later calls:
 * the last column pass stores only rows y0 .. y0+ny-1 and columns
 * x0 .. x0+nx-1 of the fftshifted |fft2(exit)|^2, so dp (and grad_dp of
 * wap_multislice_bwd) is (n_probes, ny, nx).  The centre crop of
 * downsample_to_max_angle / max_angle_gpts (propagation.py:394-439) fused
 * into the diffraction epilogue.  ny = nx = 0: the whole grid (default). */
int wap_plan_set_detector(wap_plan* plan, int y0, int x0, int ny, int nx);

/* Transfer function on the device, evaluated in float64.
 *   WAP_TF_FRESNEL: propagation.py:139-145
 *       H[i,j] = exp(i 2 pi z/lam) exp(-i pi lam z (fx_i^2 + fy_j^2))
 *   WAP_TF_ANGULAR: propagation.py:148-156
 *       H[i,j] = exp(i 2 pi z sqrt_c(1/lam^2 - fx_i^2 - fy_j^2))
 * with fx = fftfreq(n, ps0), fy = fftfreq(m, ps1) (meshgrid 'ij', shape n x m).
 * out is complex128 when out_c128 != 0, else complex64; for complex64, out_lo
 * (nullable) receives the rounding remainder value - (complex64)value, the
 * H_lo argument of the multislice calls. */
int wap_transfer_function(int kind, int n, int m, double ps0, double ps1, double z,
                          double energy, void* out, int out_c128, void* out_lo, void* stream);

/* Fresnel / angular-spectrum multislice forward, propagation.py:305-352.
 *   V        (n_draws, n_slices, ny, nx) float32 mean potential per slice [V]
 *   draw     (n_probes) int32 potential draw of each probe, or NULL (all 0)
 *   psi0     complex64 initial wave: (n_probes, ny, nx) if psi0_per_probe,
 *            else one (ny, nx) probe shared by all
 *   positions(n_probes, 2) int32 probe centres (row, col) applied like
 *            move_probe (propagation.py:263-276), or NULL (no shift)
 *   H        (ny, nx) complex64 transfer function
 *   H_lo     (ny, nx) complex64 remainder H - (complex64)H of a float64
 *            transfer function, or NULL.  The same rounding of H is applied
 *            at every slice, so its error grows linearly with the slice count;
 *            with H_lo the product is formed as X H + X H_lo.
 *   exit     (n_probes, ny, nx) complex64 out (also the working buffer)
 *   dp       (n_probes, ny, nx) float32 |fftshift(fft2(exit))|^2, or NULL
 *   stack    (n_probes, n_slices, ny, nx) complex64 wave after every slice,
 *            or NULL (the reference always stacks; NULL skips those writes)
 */
int wap_multislice_fwd(wap_plan* plan, const float* V, int n_slices, int n_draws,
                       const int32_t* draw, const float* psi0, int n_probes,
                       int psi0_per_probe, const int32_t* positions, const float* H,
                       const float* H_lo, double dz, double energy, float* exit, float* dp,
                       float* stack, void* stream);

/* out[b] = ifft2(H X[b]) for n spectra X (complex64, (n, ny, nx)), H the plan
 * grid's complex64 hi part and H_lo its remainder (or NULL): the inverse
 * transform of wpm_propagation_kernel (propagation.py:159-167), whose H is
 * exp(i dz sqrt(n^2 k0^2 - k_perp^2)) (build it with wap_line_transfer over the
 * flattened k_perp^2).  out may equal X. */
int wap_spectrum_propagate(wap_plan* plan, const float* X, int n, const float* H, const float* H_lo, float* out,
                           void* stream);

/* 1D helpers (propagation.py:609-652) and the naive per-pixel WPM step.
 *
 * wap_line_transfer: out (n) complex128 =
 *   WAP_TF_FRESNEL  exp(-i kx_sq dy / (2 k0))            fresnel_kernel_1d (:617-619)
 *   WAP_TF_ANGULAR  exp(i dy sqrt(k0^2 - kx_sq)), the principal complex root
 *                                                        angular_spectrum_kernel_1d (:622-626)
 *   evaluated in float64; kx_sq is (n) float64.
 * wap_line_propagate: out[l] = ifft(fft(psi[l]) H) for n_lines complex64 lines of
 *   n points (a power of two in [32, 2048]): propagate_1d (:629-633).  H is
 *   (n) complex64 shared by every line, or (n_lines, n) with h_per_line; H_lo
 *   its float64 remainder or NULL.
 * wap_line_wpm: out[k] = ifft(psi_k exp(i dy sqrt((n_vals[k] k0)^2 - kx_sq)))
 *   for n_refs indices: wpm_kernel_1d / wpm_kernel_1d_vmap (:636-652); psi_k is
 *   one (n) complex64 spectral line, the transfer function is evaluated in
 *   float64 and applied as hi + lo parts.
 * wap_wpm_naive_step: wpm_step (:184-212): out[p] = pixel p of
 *   ifft2(fft2(wave) exp(i dz sqrt((n_map[p] k0)^2 - k_perp^2))) with k_perp
 *   from get_frequencies(ny, nx, (ps0, ps1)), evaluated as direct float64 sums
 *   (any ny x nx up to 65536 pixels; O(P^2) work).  wave and out are (ny, nx)
 *   complex128, n_map (ny, nx) float64, work 2 ny nx complex128. */
int wap_line_transfer(int kind, int n, const double* kx_sq, double k0, double dy, double* out, void* stream);
int wap_line_propagate(int n, int n_lines, const float* psi, const float* H, const float* H_lo, int h_per_line,
                       float* out, void* stream);
int wap_line_wpm(int n, int n_refs, const float* psi_k, const double* n_vals, double k0, const double* kx_sq,
                 double dy, float* out, void* stream);
int wap_wpm_naive_step(int ny, int nx, const double* wave, const double* n_map, double dz, double energy,
                       double ps0, double ps1, double* out, double* work, void* stream);

/* Projected potential of Gaussian atoms, built on the device:
 *   V[s, y, x] = scale * sum_{a in slice s} amp_a exp(-(dy^2 + dx^2) / (2 sigma^2))
 * with dy, dx the periodic distances ((p - c + L/2) mod L) - L/2 of pixel
 * (y ps_y, x ps_x) to atom a on the (ny ps_y) x (nx ps_x) box.
 *   atoms        (n_atoms, 3) float64: y, x (A), amplitude (V A), grouped by slice
 *   slice_start  (n_slices + 1) int32 offsets: slice s holds atoms
 *                slice_start[s] .. slice_start[s+1]-1
 *   scale        e.g. 1/dz to pass the potential in volts
 *   V            (n_slices, ny, nx) float32 out
 * Atoms farther than 7 sigma from a pixel are skipped (< 2.3e-11 of a peak).
 * Replaces the host-side potential construction that precedes the multislice
 * (get_abtem_transmit, propagation.py:286-299, builds abTEM potentials on the
 * host; the benchmark configurations use this Gaussian-atom model). */
int wap_gaussian_potential(int n_slices, int ny, int nx, double ps_y, double ps_x, const double* atoms,
                           const int32_t* slice_start, double sigma, double scale, float* V, void* stream);

/* Convergent probe on the device, into out ((ny, nx) complex64 of the plan's
 * grid): a hard aperture |f| lambda < alpha_mrad / 1000 with the defocus phase
 * exp(-i pi lambda defocus |f|^2) inside it (f from fftfreq(ny, ps_y) x
 * fftfreq(nx, ps_x), float64), inverse-transformed, normalised to
 * sum |psi|^2 = ny nx and, with centred != 0, rolled to the grid centre
 * (ny/2, nx/2) - the position move_probe (propagation.py:263-276) measures
 * shifts from.  Replaces the host-side probe construction that precedes the
 * multislice (the reference's notebooks build probes with abTEM on the host,
 * e.g. wpm/cbed.ipynb; the benchmark configurations use this probe model).
 * The plan keeps one 8-byte counter, allocated on the first call. */
int wap_aperture_probe(wap_plan* plan, double ps_y, double ps_x, double energy, double alpha_mrad, double defocus,
                       int centred, float* out, void* stream);

/* Sum diffraction patterns per output pattern, in a fixed order (no atomics):
 *   out[p] = sum_{j = start[p]}^{start[p+1]-1} dp[probes[j]]
 * dp is (n_probes, plane) float32, out (n_patterns, plane), start
 * (n_patterns + 1) and probes int32, all device pointers.  With several
 * frozen-phonon draws per scan position (probes of one position sharing a
 * pattern) this is the per-position accumulation of the incoherent average
 * the reference's callers form by summing simulate_fresnel_as patterns over
 * configurations.  Indices outside [0, n_probes) are skipped and set *bad = 1
 * (bad: device int, nullable). */
int wap_pattern_accumulate(const float* dp, int n_probes, long long plane, const int32_t* start,
                           const int32_t* probes, int n_patterns, float* out, int* bad, void* stream);

/* WPM adaptive-binning multislice forward, propagation.py:358-387 with the
 * step of propagation.py:215-256 (n_bins reference indices spaced
 * n_min + (n_max - n_min) t^power_spacing per slice, smoothstep blend of the
 * two bracketing fields).  sampling = (dy, dx) as the reference's `ps`.
 * Arguments otherwise as wap_multislice_fwd; n_bins must equal the plan's. */
int wap_wpm_fwd(wap_plan* plan, const float* V, int n_slices, int n_draws,
                const int32_t* draw, const float* psi0, int n_probes, int psi0_per_probe,
                const int32_t* positions, double dz, double energy, double sampling_y,
                double sampling_x, double power_spacing, float* exit, float* dp,
                float* stack, void* stream);

/* Gradient of a loss of the Fresnel/AS multislice w.r.t. the potential.
 * No counterpart function in the reference, whose paper claims autodiff
 * through JAX (Paper/main.tex:271-274); this is the hand-written adjoint.
 *   exit       (n_probes, ny, nx) forward exit waves (from wap_multislice_fwd)
 *   ckpt       (n_probes, ceil(n_slices/ckpt_every), ny, nx) complex64 waves
 *              entering slices 0, k, 2k, ... (from wap_multislice_fwd_ckpt)
 *   grad_dp    (n_probes, ny, nx) float32 dL/d(dp), or NULL
 *   grad_exit  (n_probes, ny, nx) complex64 torch-convention gradient of the
 *              exit wave (dL/dRe + i dL/dIm), or NULL
 *   grad_V     (n_draws, n_slices, ny, nx) float32 out, accumulated (+=)
 *   work       complex64 workspace of (n_probes, ckpt_every + 2, ny, nx)
 */
int wap_multislice_fwd_ckpt(wap_plan* plan, const float* V, int n_slices, int n_draws,
                            const int32_t* draw, const float* psi0, int n_probes,
                            int psi0_per_probe, const int32_t* positions, const float* H,
                            const float* H_lo, double dz, double energy, float* exit, float* dp,
                            float* ckpt, int ckpt_every, void* stream);

int wap_multislice_bwd(wap_plan* plan, const float* V, int n_slices, int n_draws,
                       const int32_t* draw, int n_probes, const float* H, const float* H_lo,
                       double dz, double energy, const float* exit, const float* ckpt, int ckpt_every,
                       const float* grad_dp, const float* grad_exit, float* grad_V,
                       float* work, void* stream);

/* Fresnel / angular-spectrum forward that allocates no device memory.  No
 * counterpart in the reference: it exists for callers that cannot allocate
 * when they run (recording a CUDA graph under a framework that forbids
 * allocation during capture, fixed-pool hosts, plugin hosts that only pass
 * in/out buffers).  Same arguments and results as wap_multislice_fwd without
 * the plan (ny x nx given explicitly, one potential draw, default launch
 * shape, transmission evaluated per probe).  The FFT twiddle tables live in a
 * fixed 128 KiB array inside the library (held by every GPU that loads it
 * until exit) and are rewritten by each call; calls that overlap on the GPU
 * share that array and race.  The first call on a device looks up the array's
 * device address: make it before any stream capture.  Grids whose tables do
 * not fit are rejected with WAP_ERR_UNSUPPORTED. */
int wap_multislice_fwd_noalloc(const float* V, int n_slices, int ny, int nx, const float* psi0,
                               int n_probes, int psi0_per_probe, const int32_t* positions,
                               const float* H, const float* H_lo, double dz, double energy,
                               float* exit, float* dp, float* stack, void* stream);

/* Batched scan: one grid class of probes (square n x n grid, n in
 * {128, 256, 512, 1024}) with its own potential draws, probe and propagator.
 * All pointers are device pointers; the probe is shared and rolled to each
 * position like move_probe (propagation.py:263-276). */
typedef struct wap_scan_class {
  int n, n_slices, n_draws, n_probes;
  const float* V;            /* (n_draws, n_slices, n, n) float32 volts */
  const int32_t* draw;       /* (n_probes) or NULL */
  const float* psi0;         /* (n, n) complex64 probe */
  const int32_t* positions;  /* (n_probes, 2) probe centres or NULL */
  const float* H;            /* (n, n) complex64 transfer function */
  const float* H_lo;         /* (n, n) complex64 remainder or NULL */
  double dz, energy;
  float* exit;               /* (n_probes, n, n) complex64: working buffer, exit waves */
  float* dp;                 /* (n_probes, n, n) float32, or (n_probes, det_ny, det_nx), or NULL */
  int group;                 /* probes advanced together, used as given (0: automatic:
                                about 4 x the resident CTAs in tiles, then evened out
                                over n_probes) */
  int det_y0, det_x0;        /* detector window of dp (see wap_plan_set_detector); */
  int det_ny, det_nx;        /*   det_ny = det_nx = 0: the whole grid */
} wap_scan_class;

typedef struct wap_scan wap_scan;

/* Persistent batched scheduler for simulate_fresnel_as over many probes
 * (the caller loop of propagation.py:305-352 over move_probe positions).
 * wap_scan_create lays out the device work queue (groups of probes x passes
 * x tiles), tensor maps and transmission tables for up to 4 classes;
 * wap_scan_run issues, on `stream`, the counter resets, one transmission
 * table kernel per class and ONE persistent kernel that runs every tile of
 * every class (capturable in a CUDA graph).  Every device-side wait is
 * bounded; wap_scan_status (synchronising) returns WAP_ERR_TIMEOUT if one
 * expired. */
int wap_scan_create(wap_scan** scan, int n_classes, const wap_scan_class* classes);
int wap_scan_run(wap_scan* scan, void* stream);
/* Gradient scan (one class): the forward of wap_scan_run that also keeps
 * the waves entering every ckpt_every-th slice and the whole last segment,
 * and a backward that recomputes each earlier segment from its checkpoint and
 * sweeps the adjoint in reverse slice order, all in the persistent
 * scheduler.  dp must be non-NULL.  wap_scan_grad_backward accumulates
 * dL/dV (+=, laid out like V) for a loss whose gradient w.r.t. the
 * diffraction pattern is grad_dp (n_probes, n, n), or (n_probes, det_ny,
 * det_nx) with a detector window.  No counterpart function in
 * the reference (its paper claims autodiff through JAX, Paper/main.tex:271-274). */
int wap_scan_grad_create(wap_scan** scan, const wap_scan_class* cls, int ckpt_every);
int wap_scan_grad_backward(wap_scan* scan, const float* grad_dp, float* grad_V, void* stream);
/* The same for a loss on the diffraction pattern and/or on the exit wave:
 * grad_exit (n_probes, n, n) complex64 in the torch convention (dL/dRe +
 * i dL/dIm), either pointer may be NULL (not both).  The exit-wave term enters
 * the seed as fft2(grad_exit / 2), formed with the pass kernels first. */
int wap_scan_grad_backward_ex(wap_scan* scan, const float* grad_dp, const float* grad_exit, float* grad_V,
                              void* stream);
/* Re-point a scan at other buffers of the same shapes (the column-tile tensor
 * maps are re-encoded on the host; a class's detector window may change - the
 * first window set on a class allocates its full-grid pattern scratch, nothing
 * else is allocated). */
int wap_scan_bind(wap_scan* scan, int n_classes, const wap_scan_class* classes);
int wap_scan_status(wap_scan* scan, int* status);
/* Non-blocking form: enqueue on `stream` a copy of the scan's status word (0
 * or WAP_ERR_TIMEOUT, as left by the last run issued before it on that
 * stream) into host_status, a host int the GPU can write (pinned memory).
 * The value is valid once the stream has reached the copy.  The Python layer
 * turns a non-zero status into WapError. */
int wap_scan_status_async(wap_scan* scan, int* host_status, void* stream);
/* Work-queue tickets, launched CTAs and the probe-group size class 0 runs with. */
int wap_scan_info(const wap_scan* scan, long long* tickets, int* grid, int* group0);
int wap_scan_destroy(wap_scan* scan);
/* Failure injection for tests (no counterpart in the reference): tiles of
 * pass `pass` get a dependency nothing satisfies, so their bounded waits
 * expire after `spin_limit` polls and the run reports WAP_ERR_TIMEOUT; pass
 * -1 restores normal operation.  No device fault is involved. */
int wap_scan_debug_stall(wap_scan* scan, int pass, long long spin_limit);
/* Debug validation and counters (no counterpart in the reference): with
 * on & 1 every task is range-checked before use and a bad one is skipped;
 * with on & 2 the producers count the tickets whose inputs were not complete
 * when claimed and the polls spent waiting for them.  record (8 ints,
 * nullable) receives [where, class, pass, probe, tile, valid] of the first
 * violation (where = 0: none), then the two counters (cumulative since the
 * scan was created; the second as an unsigned count). */
int wap_scan_debug_checks(wap_scan* scan, int on, int* record);
/* Scheduler overrides for A/B timing and tests (no counterpart in the
 * reference), process-wide, read by every later wap_scan_create /
 * wap_scan_grad_create; value -1 restores the library's own choice.  Nothing
 * else (no environment variable) changes these choices.
 *   WAP_KNOB_ELEMS     elements per thread of forward scans: 16 or 8
 *   WAP_KNOB_TWIDDLES  stage-twiddle table: WAP_TW_FULL (hi + lo) or WAP_TW_HI
 *                      (hi only; by default scans of at most 160 slices)
 *   WAP_KNOB_TW_SMEM   reserved (the twiddle image is always in shared memory)
 *   WAP_KNOB_PSI       how adjoint rows read psi_s: 0 global, 1 second stage,
 *                      2 the one stage refilled (default)
 *   WAP_KNOB_GROUP     probe-group size of classes that ask for automatic
 *   WAP_KNOB_CHAIN     0: single-probe forwards as one launch per pass instead
 *                      of the one-launch chain kernel (default 1)
 *   WAP_KNOB_SUSPEND   suspend-time hint (ns) of the scheduler's mbarrier
 *                      waits, 0: none (the default)
 *   WAP_KNOB_H_HI      reserved
 *   WAP_KNOB_CLUSTER   0: single-probe forwards without the cluster kernel
 *                      (wave in distributed shared memory); 1: its launch
 *                      counts as refused by the device without being issued
 *                      (the plan falls back to the chain kernel for good);
 *                      4 / 8 / 16 that many elements per thread */
#define WAP_KNOB_ELEMS 0
#define WAP_KNOB_TWIDDLES 1
#define WAP_KNOB_TW_SMEM 2
#define WAP_KNOB_PSI 3
#define WAP_KNOB_GROUP 4
#define WAP_KNOB_CHAIN 5
#define WAP_KNOB_SUSPEND 6
#define WAP_KNOB_H_HI 7
#define WAP_KNOB_CLUSTER 8
#define WAP_KNOB_COUNT 9
#define WAP_TW_FULL 1
#define WAP_TW_HI 2
int wap_scan_debug_override(int which, int value);

/* Kernel-level tracing (no counterpart in the reference, which has none).
 * While enabled, each pass launch is bracketed by CUDA events on its stream
 * and tagged with its kind and algorithmic bytes (wave in/out, potential,
 * snapshots).  wap_profile_read waits for the recorded events and returns the
 * launch count, summed device milliseconds and summed bytes of one kind. */
#define WAP_KIND_ROW 0        /* row pass (transmission + row FFTs) */
#define WAP_KIND_COL 1        /* column pass (column FFTs + propagator) */
#define WAP_KIND_WPM_COL 2    /* WPM column pass (K reference fields) */
#define WAP_KIND_WPM_ROW 3    /* WPM row pass (K row IFFTs + blend) */
#define WAP_KIND_WPM_BINS 4   /* WPM per-slice bin edges */
#define WAP_KIND_SCHED 5      /* persistent batched scheduler */
#define WAP_KIND_TRANS 6      /* transmission table exp(i phi(V)) */
/* Number of kernels this library has launched in this process (all kinds). */
long long wap_launch_count(void);
int wap_profile_enable(int on);
int wap_profile_reset(void);
int wap_profile_read(int kind, long long* launches, double* total_ms, double* total_bytes);

/* FP32 peak probe for the roofline (no counterpart in the reference):
 * `blocks` CTAs of 256 threads, each thread `iters` x 8 independent FMAs
 * (2 flops each), one float per thread written to `out` (blocks x 256).
 * The caller times the launch on `stream`. */
int wap_fp32_probe(int blocks, int iters, float* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* WAP_H_ */
