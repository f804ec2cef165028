"""CPU oracle: a NumPy/SciPy restatement of the reference multislice path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this module;
only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline /
reference arm use it, and only as the checker or the timed CPU baseline.

What it restates (reference file ``wide_angle_propagation/propagation.py``):

* physics constants and conversions ............ :14-50, :66-81
* frequency grids / smoothstep / poly bins ..... :102-127
* Fresnel and angular-spectrum transfer funcs .. :139-156
* WPM single-index propagator (+vmap) .......... :159-171
* ``Propagator`` (fft2 . H . ifft2) .............. :178-181
* naive ``wpm_step`` (one propagate per pixel) .. :184-212
* ``wpm_step_adaptive`` .......................... :215-256
* ``move_probe`` ................................. :263-276
* ``simulate_fresnel_as`` ........................ :305-352
* ``simulate_wpm`` ............................... :358-387
* detector crop ``max_angle_gpts`` /
  ``downsample_to_max_angle`` .................... :394-439
* Lippmann-Schwinger 2D (kernel, convolution,
  GMRES solve) ................................... :446-602
* 1D helpers ``get_kx_1d`` .. ``wpm_kernel_1d_vmap`` :609-652

Parity pin: the reference module cannot be imported with its real
dependencies here (jax, jaxlib, abtem and ase are not installed).  The
fixtures in ``tests/golden/`` were produced by executing the reference's own
``propagation.py`` with NumPy standing in for ``jax.numpy`` (script:
``tests/golden/make_golden.py``); ``tests/test_oracle_golden.py`` checks this
restatement against those fixtures to ~1e-12.  What stays unpinned: XLA's FFT
rounding (vs pocketfft here, differences at the 1e-15 level) and the ASE
constants, which are hard-coded below as ASE's default CODATA-2014 set.

Three numeric modes:

``"fp64"``        the reference algorithm in float64/complex128 (the FP64
                  oracle, i.e. the reference as its notebooks run it, with
                  ``jax_enable_x64``).
``"fp32"``        the reference formulas evaluated naively in float32 /
                  complex64 (what the reference computes when fed FP32
                  arrays).  Informational: its own error vs FP64 is larger
                  than 1e-5 for long stacks because ``sqrt(ratio) - 1``
                  cancels (propagation.py:78-81).
``"fp32_stable"`` the same algorithm in float32 with the cancellation-free
                  forms the CUDA kernels use (informational).
"""
from __future__ import annotations

import math
import os

import numpy as np
import scipy.fft as sfft

# ---------------------------------------------------------------------------
# Constants: ASE default (CODATA 2014) values used through ``ase.units`` in
# propagation.py:6, :18-21, :44-50.
# ---------------------------------------------------------------------------
HPLANCK = 6.626070040e-34   # J s
C_LIGHT = 299792458.0       # m / s
M_E = 9.10938356e-31        # kg
Q_E = 1.6021766208e-19      # C

_WORKERS = max(1, os.cpu_count() or 1)


def set_workers(n: int) -> None:
    """Thread count handed to scipy.fft (the CPU baseline uses all cores)."""
    global _WORKERS
    _WORKERS = max(1, int(n))


def _dtypes(mode: str):
    if mode == "fp64":
        return np.float64, np.complex128
    if mode in ("fp32", "fp32_stable"):
        return np.float32, np.complex64
    raise ValueError(f"unknown oracle mode {mode!r}")


def _fft2(a):
    return sfft.fft2(a, axes=(-2, -1), workers=_WORKERS)


def _ifft2(a):
    return sfft.ifft2(a, axes=(-2, -1), workers=_WORKERS)


# ---------------------------------------------------------------------------
# propagation.py:14-50
# ---------------------------------------------------------------------------
def electron_rest_energy() -> float:
    """E0 = m_e c^2 / e in eV (propagation.py:14-21)."""
    return M_E * C_LIGHT ** 2 / Q_E


def relativistic_mass_correction(energy: float) -> float:
    """propagation.py:24-26."""
    return 1 + Q_E * energy / (M_E * C_LIGHT ** 2)


def energy2mass(energy: float) -> float:
    """propagation.py:29-35."""
    return relativistic_mass_correction(energy) * M_E


def energy2wavelength(energy: float) -> float:
    """Relativistic de Broglie wavelength in Angstrom (propagation.py:38-50)."""
    return (HPLANCK * C_LIGHT
            / math.sqrt(energy * (2 * M_E * C_LIGHT ** 2 / Q_E + energy))
            / Q_E * 1.0e10)


# ---------------------------------------------------------------------------
# propagation.py:66-81  (and the cancellation-free form used by the kernels)
# ---------------------------------------------------------------------------
def electron_refractive_index(potential, energy, mode: str = "fp64"):
    """n(V) exactly as propagation.py:66-81 (V in volts, E in eV)."""
    fdt, _ = _dtypes(mode)
    potential = np.asarray(potential, dtype=fdt)
    E0 = electron_rest_energy()
    E = energy
    V = -potential                      # :75
    EminusV = E - V                     # :76
    numerator = 2 * EminusV * E0 + EminusV ** 2      # :78
    denominator = 2 * E * E0 + E ** 2                # :79
    return np.sqrt(numerator / denominator)          # :81


def refractive_index_minus_one(potential, energy, mode: str = "fp64"):
    """n - 1 for the same n(V) as propagation.py:66-81.

    ``fp64``/``fp32``: the reference's literal ``sqrt(ratio) - 1``.
    ``fp32_stable``: r/(sqrt(1+r)+1) with r = V(2E0+2E+V)/(E(2E0+E)), the
    algebraically identical cancellation-free form.
    """
    fdt, _ = _dtypes(mode)
    if mode != "fp32_stable":
        return electron_refractive_index(potential, energy, mode) - fdt(1)
    p = np.asarray(potential, dtype=np.float32)
    E0 = electron_rest_energy()
    inv_den = np.float32(1.0 / (energy * (2 * E0 + energy)))
    a = np.float32(2 * E0 + 2 * energy)
    r = p * (a + p) * inv_den
    return (r / (np.sqrt(np.float32(1) + r) + np.float32(1))).astype(np.float32)


# ---------------------------------------------------------------------------
# propagation.py:102-127
# ---------------------------------------------------------------------------
def get_frequencies(n, m, ps):
    """fftfreq grids, meshgrid indexing='ij' (propagation.py:102-107)."""
    fx = np.fft.fftfreq(n, ps[0])
    fy = np.fft.fftfreq(m, ps[1])
    Fx, Fy = np.meshgrid(fx, fy, indexing="ij")
    return Fx, Fy


def smoothstep(x):
    """3x^2 - 2x^3 on clip(x, 0, 1) (propagation.py:110-116)."""
    x = np.clip(x, 0.0, 1.0)
    return 3 * x ** 2 - 2 * x ** 3


def get_polynomial_bins(n_min, n_max, n_bins, power=2.0):
    """n_min + (n_max - n_min) * linspace(0,1,K)**power (propagation.py:119-127)."""
    t = np.linspace(0, 1, n_bins)
    t_warped = t ** power
    return n_min + (n_max - n_min) * t_warped


# ---------------------------------------------------------------------------
# propagation.py:139-171
# ---------------------------------------------------------------------------
def fresnel_propagation_kernel(n, m, ps, z, energy):
    """H = exp(i 2pi z/lam) exp(-i pi lam z (Fx^2+Fy^2)) (propagation.py:139-145)."""
    wavelength = energy2wavelength(energy)
    Fx, Fy = get_frequencies(n, m, ps)
    return (np.exp(1j * (2 * np.pi / wavelength) * z)
            * np.exp(-1j * np.pi * wavelength * z * (Fx ** 2 + Fy ** 2)))


def angular_spectrum_propagation_kernel(n, m, ps, z, energy):
    """H = exp(i 2pi z sqrt(1/lam^2 - f^2)), complex sqrt (propagation.py:148-156)."""
    wavelength = energy2wavelength(energy)
    Fx, Fy = get_frequencies(n, m, ps)
    kz = np.sqrt(np.asarray((1 / wavelength) ** 2 - Fx ** 2 - Fy ** 2,
                            dtype=np.complex128))
    return np.exp(1j * 2 * np.pi * z * kz)


def wpm_propagation_kernel(Ek, n_val, k0, k_perp2, dz):
    """ifft2(exp(i dz sqrt(n^2 k0^2 - k_perp^2)) Ek) (propagation.py:159-167)."""
    kz = np.sqrt(np.asarray(n_val ** 2 * k0 ** 2 - k_perp2, dtype=np.complex128))
    H = np.exp(1j * dz * kz)
    return _ifft2(H * Ek)


# ---------------------------------------------------------------------------
# propagation.py:178-181
# ---------------------------------------------------------------------------
def Propagator(u, H):
    """ifft2(H * fft2(u)) (propagation.py:178-181)."""
    return _ifft2(H * _fft2(u))


# ---------------------------------------------------------------------------
# propagation.py:184-212
# ---------------------------------------------------------------------------
def wpm_step(wave, n_map, dz, energy, ps):
    """Naive WPM step (propagation.py:184-212): pixel p of the new wave is
    pixel p of ifft2(fft2(wave) exp(i dz sqrt((n_p k0)^2 - k_perp^2))), one
    full propagate per pixel.  k_perp^2 from get_frequencies(ny, nx, ps)
    (axis 0: fftfreq(ny, ps[0]), axis 1: fftfreq(nx, ps[1]))."""
    wave = np.asarray(wave, dtype=np.complex128)
    ny, nx = wave.shape
    k0 = 2 * np.pi / energy2wavelength(energy)
    Fy, Fx = get_frequencies(ny, nx, ps)
    k_perp2 = (2 * np.pi * Fx) ** 2 + (2 * np.pi * Fy) ** 2
    Ek = _fft2(wave)
    n_flat = np.asarray(n_map, dtype=np.float64).reshape(-1)
    out = np.empty(ny * nx, np.complex128)
    for p in range(n_flat.size):
        out[p] = wpm_propagation_kernel(Ek, n_flat[p], k0, k_perp2, dz).reshape(-1)[p]
    return out.reshape(ny, nx)


# ---------------------------------------------------------------------------
# propagation.py:215-256
# ---------------------------------------------------------------------------
def _wpm_kperp2(ny, nx, ps):
    """k_perp^2 on the 'xy' meshgrid of propagation.py:224-228."""
    dy, dx = ps
    ky = 2 * np.pi * np.fft.fftfreq(ny, d=dy)
    kx = 2 * np.pi * np.fft.fftfreq(nx, d=dx)
    Fx, Fy = np.meshgrid(kx, ky)
    return Fx ** 2 + Fy ** 2


def wpm_step_adaptive(wave, n_map, dz, energy, ps, n_bins=256, power_spacing=2.0):
    """Adaptive-binning WPM step in complex128 (propagation.py:215-256).

    Returns (new_wave, w, idx_L, n_refs) like the reference.
    """
    ny, nx = wave.shape
    wavelength = energy2wavelength(energy)
    k0 = 2 * np.pi / wavelength
    k_perp2 = _wpm_kperp2(ny, nx, ps)
    Ek = _fft2(wave)
    n_min, n_max = n_map.min(), n_map.max()                       # :232
    n_refs = get_polynomial_bins(n_min, n_max, n_bins, power=power_spacing)
    ref_fields = np.stack([wpm_propagation_kernel(Ek, nk, k0, k_perp2, dz)
                           for nk in n_refs])                     # :236
    idx_R = np.searchsorted(n_refs, n_map)                        # :239 side='left'
    idx_R = np.clip(idx_R, 1, n_bins - 1)                         # :240
    idx_L = idx_R - 1
    n_L = n_refs[idx_L]
    n_R = n_refs[idx_R]
    denom = n_R - n_L
    w_raw = (n_map - n_L) / np.where(denom == 0, 1.0, denom)      # :248
    w = smoothstep(w_raw)
    field_L = np.take_along_axis(ref_fields, idx_L[None, ...], axis=0)[0]
    field_R = np.take_along_axis(ref_fields, idx_R[None, ...], axis=0)[0]
    new_wave = (1 - w) * field_L + w * field_R                    # :254
    return new_wave, w, idx_L, n_refs


def _wpm_step_fp32_stable(wave, dn, dz, energy, ps, n_bins, power_spacing, hvac64):
    """FP32 emulation of the kernels' WPM step (informational).

    Works in delta = n - 1 (same bins: n_refs - 1 = delta_min + (delta_max -
    delta_min) t^p) and splits each bin's propagator into the FP64-tabulated
    vacuum part times a small FP32 phase
    dz (n^2-1) k0^2 / (kz_n + kz_vac).
    """
    ny, nx = wave.shape
    wavelength = energy2wavelength(energy)
    k0 = 2 * np.pi / wavelength
    kp2 = _wpm_kperp2(ny, nx, ps).astype(np.float32)
    Ek = sfft.fft2(wave.astype(np.complex64), workers=_WORKERS)
    d_min, d_max = np.float64(dn.min()), np.float64(dn.max())
    d_refs = get_polynomial_bins(d_min, d_max, n_bins, power=power_spacing).astype(np.float32)
    k0f = np.float32(k0)
    k02 = np.float32(k0 * k0)
    kzv = np.sqrt(np.maximum(k02 - kp2, 0)).astype(np.float32)
    fields = np.empty((n_bins, ny, nx), np.complex64)
    for k, d in enumerate(d_refs):
        a = np.float32(d) * (np.float32(2) + np.float32(d)) * k02
        kzn = np.sqrt(np.maximum(k02 + a - kp2, 0)).astype(np.float32)
        ph = np.float32(dz) * a / (kzn + kzv)
        fields[k] = sfft.ifft2(hvac64 * Ek * np.exp(1j * ph).astype(np.complex64), workers=_WORKERS)
    idx_R = np.clip(np.searchsorted(d_refs, dn), 1, n_bins - 1)
    idx_L = idx_R - 1
    dL, dR = d_refs[idx_L], d_refs[idx_R]
    den = dR - dL
    w = smoothstep((dn - dL) / np.where(den == 0, np.float32(1), den)).astype(np.float32)
    fl = np.take_along_axis(fields, idx_L[None], 0)[0]
    fr = np.take_along_axis(fields, idx_R[None], 0)[0]
    return ((1 - w) * fl + w * fr).astype(np.complex64)


# ---------------------------------------------------------------------------
# propagation.py:263-276
# ---------------------------------------------------------------------------
def move_probe(probe, new_pos):
    """Roll the probe so its centre (ny//2, nx//2) lands on new_pos (propagation.py:263-276)."""
    shift_row = new_pos[0] - probe.shape[0] // 2
    shift_col = new_pos[1] - probe.shape[1] // 2
    return np.roll(probe, (shift_row, shift_col), axis=(0, 1))


# ---------------------------------------------------------------------------
# propagation.py:305-352
# ---------------------------------------------------------------------------
def _diffraction(exit_wave):
    """|fftshift(fft2(exit))|^2 (propagation.py:346-350)."""
    d = np.fft.fftshift(_fft2(exit_wave), axes=(-2, -1))
    return np.square(d.real) + np.square(d.imag)


def simulate_fresnel_as(potential, probe, prop_kernel, slice_thickness, energy,
                        mode: str = "fp64", return_wavefronts: bool = True):
    """Fresnel / angular-spectrum multislice (propagation.py:305-352).

    ``potential`` (N, ny, nx) in volts; ``probe`` (ny, nx) or (B, ny, nx);
    ``prop_kernel`` (ny, nx).  Returns (exit_wave, diffraction_pattern,
    stacked wavefronts or None).
    """
    fdt, cdt = _dtypes(mode)
    wavelength = energy2wavelength(energy)
    V = np.asarray(potential, dtype=fdt)
    wave = np.asarray(probe).astype(cdt)
    H = np.asarray(prop_kernel).astype(cdt)
    waves = []
    for i in range(V.shape[0]):
        if mode == "fp32_stable":
            dn = refractive_index_minus_one(V[i], energy, mode)
            ph = (np.float32(2 * np.pi * slice_thickness / wavelength) * dn)
            t = (np.cos(ph) + 1j * np.sin(ph)).astype(cdt)
        else:
            n = electron_refractive_index(V[i], energy, mode)       # :333
            t = np.exp(1j * 2 * np.pi * (n - 1) * slice_thickness / wavelength).astype(cdt)  # :336
        wave = (wave * t).astype(cdt)                              # :337
        wave = Propagator(wave, H).astype(cdt)                     # :340
        if return_wavefronts:
            waves.append(wave)
    dp = _diffraction(wave).astype(fdt)
    stack = np.stack(waves, axis=-3) if return_wavefronts else None
    return wave, dp, stack


# ---------------------------------------------------------------------------
# propagation.py:358-387
# ---------------------------------------------------------------------------
def simulate_wpm(potential, probe, slice_thickness, energy, sampling,
                 n_bins=128, power_spacing=2.0, mode: str = "fp64",
                 return_wavefronts: bool = True):
    """WPM adaptive-binning multislice (propagation.py:358-387)."""
    fdt, cdt = _dtypes(mode)
    V = np.asarray(potential, dtype=fdt)
    wave = np.asarray(probe).astype(cdt)
    batched = wave.ndim == 3
    waves_in = wave if batched else wave[None]
    outs, dps, stacks = [], [], []
    if mode == "fp32_stable":
        ny, nx = waves_in.shape[-2:]
        k0 = 2 * np.pi / energy2wavelength(energy)
        kp2 = _wpm_kperp2(ny, nx, sampling)
        hvac64 = np.exp(1j * slice_thickness * np.sqrt((k0 * k0 - kp2).astype(np.complex128))).astype(np.complex64)
    for w in waves_in:
        ws = []
        for i in range(V.shape[0]):
            if mode == "fp32_stable":
                dn = refractive_index_minus_one(V[i], energy, mode)
                w = _wpm_step_fp32_stable(w, dn, slice_thickness, energy, sampling,
                                          n_bins, power_spacing, hvac64)
            else:
                n = electron_refractive_index(V[i], energy, mode)   # :369
                w, _, _, _ = wpm_step_adaptive(w, n, slice_thickness, energy,
                                               sampling, n_bins=n_bins,
                                               power_spacing=power_spacing)
                w = w.astype(cdt)
            if return_wavefronts:
                ws.append(w)
        outs.append(w)
        dps.append(_diffraction(w).astype(fdt))
        stacks.append(np.stack(ws) if return_wavefronts else None)
    if batched:
        return (np.stack(outs), np.stack(dps),
                np.stack(stacks) if return_wavefronts else None)
    return outs[0], dps[0], stacks[0]


# ---------------------------------------------------------------------------
# propagation.py:394-439 (detector crop; post-processing after the path)
# ---------------------------------------------------------------------------
def max_angle_gpts(shape, sampling, wavelength, max_angle_mrad, parity="odd"):
    """propagation.py:394-421."""
    ny, nx = shape
    dx, dy = float(sampling[0]), float(sampling[1])
    max_freq = float(max_angle_mrad) / (float(wavelength) * 1000.0)
    dfx = 1.0 / (nx * dx)
    dfy = 1.0 / (ny * dy)
    half_x = int(np.floor(max_freq / dfx))
    half_y = int(np.floor(max_freq / dfy))
    half_x = max(0, min(half_x, nx // 2))
    half_y = max(0, min(half_y, ny // 2))
    if parity == "even":
        new_nx, new_ny = 2 * half_x, 2 * half_y
    else:
        new_nx, new_ny = 2 * half_x + 1, 2 * half_y + 1
    new_nx = max(1, min(new_nx, nx))
    new_ny = max(1, min(new_ny, ny))
    return new_ny, new_nx


def downsample_to_max_angle(pattern, sampling, wavelength, max_angle_mrad, parity="odd"):
    """propagation.py:424-439."""
    arr = np.asarray(pattern)
    ny, nx = arr.shape[-2:]
    new_ny, new_nx = max_angle_gpts((ny, nx), sampling, wavelength, max_angle_mrad, parity=parity)
    if (new_ny, new_nx) == (ny, nx):
        return arr
    cy, cx = ny // 2, nx // 2
    y0 = cy - new_ny // 2
    x0 = cx - new_nx // 2
    return arr[..., y0:y0 + new_ny, x0:x0 + new_nx]


# ---------------------------------------------------------------------------
# propagation.py:446-602 (Lippmann-Schwinger 2D)
# ---------------------------------------------------------------------------
def _greens_2d_hankel(k0, r):
    """(i/4) H0^(1)(k0 r) (propagation.py:448-451)."""
    from scipy.special import hankel1
    return 0.25j * hankel1(0, k0 * r)


def _self_weight_cell_average(k0, hx, hy, oversamp=32):
    """Cell average of the Green's function over the singular cell (:454-461)."""
    xs = (np.arange(oversamp) + 0.5) / oversamp * hx - 0.5 * hx
    ys = (np.arange(oversamp) + 0.5) / oversamp * hy - 0.5 * hy
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    return _greens_2d_hankel(k0, np.sqrt(X ** 2 + Y ** 2)).mean() * (hx * hy)


def build_lippmann_schwinger_kernel_2d(k0, hx, hy, Nx, Ny, pad_to_double=True, oversamp_self=32):
    """FFT of the embedded Green's function kernel and the embedding shape (:464-501)."""
    Ex, Ey = (2 * Nx, 2 * Ny) if pad_to_double else (Nx, Ny)
    x = (np.arange(Nx) - Nx // 2) * hx
    y = (np.arange(Ny) - Ny // 2) * hy
    X, Y = np.meshgrid(x, y, indexing="ij")
    K = (hx * hy) * _greens_2d_hankel(k0, np.sqrt(X ** 2 + Y ** 2))
    K[Nx // 2, Ny // 2] = _self_weight_cell_average(k0, hx, hy, oversamp=oversamp_self)
    Kemb = np.zeros((Ex, Ey), dtype=np.complex128)
    sx, sy = (Ex - Nx) // 2, (Ey - Ny) // 2
    Kemb[sx:sx + Nx, sy:sy + Ny] = K
    return np.fft.fftn(np.fft.ifftshift(Kemb)), (Ex, Ey)


def apply_convolution(source, Khat, embed_shape, roi_shape):
    """Centre-embedded FFT convolution with the kernel, cropped back (:504-514)."""
    Ex, Ey = embed_shape
    Nx, Ny = roi_shape
    sx, sy = (Ex - Nx) // 2, (Ey - Ny) // 2
    src = np.zeros((Ex, Ey), dtype=np.complex128)
    src[sx:sx + Nx, sy:sy + Ny] = source
    return np.fft.ifftn(Khat * np.fft.fftn(src))[sx:sx + Nx, sy:sy + Ny]


def solve_scattering_2d_lippmann_schwinger(potential_grid, energy_ev, pixel_size_A, pad_factor=2,
                                           absorb_frac=0.15, absorb_strength=4.0, gmres_tol=1e-4,
                                           gmres_restart=70):
    """(I - G V_scale V) psi = psi_inc by restarted GMRES on the padded grid
    (:517-602); psi_inc = exp(i k0 y) along axis 1; returns the unpadded psi."""
    import scipy.sparse.linalg as sla
    m0, hc = 510998.95000, 12398.4193
    hbar = HPLANCK / (2 * np.pi)
    gamma = 1.0 + energy_ev / (M_E * C_LIGHT ** 2 / Q_E)
    V_scale = -(2.0 * gamma * M_E * Q_E / hbar ** 2) * 1e-20
    k0 = 2 * np.pi / (hc / np.sqrt(energy_ev * (energy_ev + 2 * m0)))
    orig = np.shape(potential_grid)
    padded = [s * pad_factor for s in orig]
    pad = [((p - o) // 2, (p - o) - (p - o) // 2) for p, o in zip(padded, orig)]
    Vp = np.pad(np.asarray(potential_grid, dtype=np.float64), pad, mode="constant")
    Khat, emb = build_lippmann_schwinger_kernel_2d(float(k0), float(pixel_size_A), float(pixel_size_A),
                                                   padded[0], padded[1])

    def matvec(v):
        psi = v.reshape(padded)
        return (psi - apply_convolution(V_scale * Vp * psi, Khat, emb, padded)).ravel()

    y = np.arange(padded[1]) * pixel_size_A
    y = y - y.mean()
    b = np.broadcast_to(np.exp(1j * k0 * y), padded).ravel()
    n = b.size
    op = sla.LinearOperator((n, n), matvec=matvec, dtype=np.complex128)
    x, _ = sla.gmres(op, b, rtol=gmres_tol, atol=0.0, restart=gmres_restart)
    x = x.reshape(padded)
    return x[pad[0][0]:pad[0][0] + orig[0], pad[1][0]:pad[1][0] + orig[1]]


# ---------------------------------------------------------------------------
# propagation.py:609-652 (1D helpers)
# ---------------------------------------------------------------------------
def get_kx_1d(n, dx):
    """2 pi fftfreq(n, dx) (propagation.py:609-614)."""
    return 2 * np.pi * np.fft.fftfreq(n, d=dx)


def fresnel_kernel_1d(kx_sq, k0, dy):
    """exp(-i kx^2 dy / (2 k0)) (propagation.py:617-619)."""
    return np.exp(-1j * np.asarray(kx_sq) * dy / (2 * k0))


def angular_spectrum_kernel_1d(kx_sq, k0, dy):
    """exp(i dy sqrt(k0^2 - kx^2)), complex sqrt (propagation.py:622-626)."""
    kz = np.sqrt(np.asarray(k0 ** 2 - np.asarray(kx_sq), dtype=np.complex128))
    return np.exp(1j * dy * kz)


def propagate_1d(psi, H):
    """ifft(fft(psi) H) along the last axis (propagation.py:629-633)."""
    return np.fft.ifft(np.fft.fft(np.asarray(psi, dtype=np.complex128), axis=-1) * H, axis=-1)


def wpm_kernel_1d(psi_k, n_val, k0, kx_sq, dy):
    """ifft(psi_k exp(i dy sqrt((n k0)^2 - kx^2))) (propagation.py:636-649)."""
    kz = np.sqrt(np.asarray((n_val * k0) ** 2 - np.asarray(kx_sq), dtype=np.complex128))
    return np.fft.ifft(np.asarray(psi_k) * np.exp(1j * dy * kz))


def wpm_kernel_1d_vmap(psi_k, n_vals, k0, kx_sq, dy):
    """wpm_kernel_1d over an array of refractive indices (propagation.py:652)."""
    return np.stack([wpm_kernel_1d(psi_k, n, k0, kx_sq, dy) for n in np.asarray(n_vals)])


def rel_l2(a, b) -> float:
    """||a - b||_2 / ||b||_2 in float64."""
    a = np.asarray(a).astype(np.complex128)
    b = np.asarray(b).astype(np.complex128)
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))
