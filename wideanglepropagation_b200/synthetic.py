"""Seeded synthetic inputs with the shapes of the five benchmark workloads.

The reference builds its potentials and probes with abTEM/ASE in notebooks
(e.g. ``wpm/cbed.ipynb``); neither library is available, so these generators
stand in for them: sums of isotropic Gaussians (projected potential in V*A,
divided by the slice thickness to give the per-slice mean potential in volts
that ``simulate_fresnel_as`` / ``simulate_wpm`` expect), and aperture probes.

Gaussian sums are evaluated separably: sum_a amp g_a(y) g_a(x) is the matrix
product (amp * Gy)^T @ Gx, with minimum-image periodic wrap.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .physics import energy2wavelength


def _gauss_1d(coords, centres, L, sigma):
    d = (coords[None, :] - centres[:, None] + L / 2) % L - L / 2
    return np.exp(-d * d / (2 * sigma * sigma))


def gaussian_slice(ny, nx, ps, centres_yx, amp, sigma):
    """Projected potential (V*A) of Gaussians at ``centres_yx`` (A), periodic."""
    centres_yx = np.asarray(centres_yx, dtype=np.float64).reshape(-1, 2)
    if centres_yx.shape[0] == 0:
        return np.zeros((ny, nx))
    Ly, Lx = ny * ps, nx * ps
    gy = _gauss_1d(np.arange(ny) * ps, centres_yx[:, 0], Ly, sigma)
    gx = _gauss_1d(np.arange(nx) * ps, centres_yx[:, 1], Lx, sigma)
    return (amp * gy).T @ gx


def random_gaussian_atoms(rng, n_slices, ny, nx, ps, n_atoms=30):
    """Atom list of ``random_gaussian_stack``: (positions (M, 2) in A, slice of each atom)."""
    L = np.array([ny * ps, nx * ps])
    pos = np.concatenate([rng.uniform(0, 1, (n_atoms, 2)) * L for _ in range(n_slices)])
    return pos, np.repeat(np.arange(n_slices), n_atoms)


def random_gaussian_stack(rng, n_slices, ny, nx, ps, n_atoms=30, amp=20.0, sigma=0.3):
    """Each slice: ``n_atoms`` Gaussians at seed-uniform centres (V*A)."""
    pos, sl = random_gaussian_atoms(rng, n_slices, ny, nx, ps, n_atoms)
    out = np.empty((n_slices, ny, nx), np.float64)
    for s in range(n_slices):
        out[s] = gaussian_slice(ny, nx, ps, pos[sl == s], amp, sigma)
    return out


# fractional in-plane positions of the atomic layers met along [100]; one
# entry per slice of thickness a/4 (diamond) or a/2 (FCC), cycling with depth
DIAMOND_LAYERS = [[(0, 0), (0.5, 0.5)], [(0.25, 0.25), (0.75, 0.75)],
                  [(0.5, 0), (0, 0.5)], [(0.75, 0.25), (0.25, 0.75)]]
FCC_LAYERS = [[(0, 0), (0.5, 0.5)], [(0.5, 0), (0, 0.5)]]


def lattice_atoms(rng, n_slices, ny, nx, ps, a, layers, jitter):
    """Atom list of ``lattice_stack``: (positions (M, 2) in A, slice of each atom).

    Slice s holds the atomic layer ``layers[s % len(layers)]``; every atom
    gets an independent N(0, jitter) in-plane displacement (frozen phonon).
    """
    Ly, Lx = ny * ps, nx * ps
    ncy, ncx = int(math.ceil(Ly / a)), int(math.ceil(Lx / a))
    all_pos, all_sl = [], []
    for s in range(n_slices):
        frac = np.asarray(layers[s % len(layers)], dtype=np.float64)
        iy, ix = np.meshgrid(np.arange(ncy), np.arange(ncx), indexing="ij")
        cells = np.stack([iy.ravel(), ix.ravel()], 1).astype(np.float64)
        pos = (cells[:, None, :] + frac[None, :, :]).reshape(-1, 2) * a
        pos = pos[(pos[:, 0] < Ly) & (pos[:, 1] < Lx)]
        pos = pos + rng.normal(0, jitter, pos.shape)
        all_pos.append(pos)
        all_sl.append(np.full(pos.shape[0], s))
    return np.concatenate(all_pos), np.concatenate(all_sl)


def lattice_stack(rng, n_slices, ny, nx, ps, a, layers, amp, sigma, jitter):
    """Per-slice projected potential of a cubic lattice seen along [100]
    (the atoms of ``lattice_atoms``, Gaussians of ``amp`` V*A and ``sigma`` A)."""
    pos, sl = lattice_atoms(rng, n_slices, ny, nx, ps, a, layers, jitter)
    out = np.empty((n_slices, ny, nx), np.float64)
    for s in range(n_slices):
        out[s] = gaussian_slice(ny, nx, ps, pos[sl == s], amp, sigma)
    return out


def aperture_probe(ny, nx, ps, energy, alpha_mrad, defocus=0.0, centred=True,
                   dtype=np.complex128):
    """Convergent probe: hard aperture |f| lam < alpha with defocus phase.

    The defocus enters as exp(-i pi lam df |f|^2) inside the aperture.  The
    probe is normalised to sum |psi|^2 = ny*nx and, if ``centred``, rolled to
    the grid centre (ny//2, nx//2), the position move_probe measures from.
    """
    lam = energy2wavelength(energy)
    fy = np.fft.fftfreq(ny, ps)
    fx = np.fft.fftfreq(nx, ps)
    f2 = fy[:, None] ** 2 + fx[None, :] ** 2
    ap = (np.sqrt(f2) * lam < alpha_mrad * 1e-3).astype(np.complex128)
    ap *= np.exp(-1j * np.pi * lam * defocus * f2)
    p = np.fft.ifft2(ap)
    if centred:
        p = np.fft.fftshift(p)
    p *= math.sqrt(ny * nx) / np.linalg.norm(p)
    return p.astype(dtype)


def raster_positions(ny, nx, n_per_side_y, n_per_side_x):
    """Integer probe centres on a uniform raster over the window."""
    ys = (np.arange(n_per_side_y) * ny) // n_per_side_y
    xs = (np.arange(n_per_side_x) * nx) // n_per_side_x
    yy, xx = np.meshgrid(ys, xs, indexing="ij")
    return np.stack([yy.ravel(), xx.ravel()], 1).astype(np.int32)


@dataclass
class Workload:
    name: str
    ny: int
    nx: int
    ps: float
    n_slices: int
    dz: float
    energy: float
    potential: np.ndarray               # (draws, N, ny, nx) float32 volts
    probe: np.ndarray                   # (ny, nx) complex
    positions: Optional[np.ndarray] = None   # (B, 2) int32 probe centres
    draw_of_probe: Optional[np.ndarray] = None  # (B,) int32 potential index
    method: str = "fresnel"             # fresnel | as | wpm
    n_bins: int = 0
    power_spacing: float = 1.0
    extra: dict = field(default_factory=dict)

    @property
    def n_probes(self) -> int:
        return 1 if self.positions is None else int(self.positions.shape[0])

    @property
    def slice_steps(self) -> int:
        return self.n_probes * self.n_slices


def plain_fresnel(seed=0, n_slices=20):
    """256^2, 0.1 A, 20 x 2 A slices, 200 keV, 30 Gaussians/slice (20 V*A, 0.3 A),
    20 mrad centred probe, Fresnel propagator."""
    rng = np.random.default_rng(seed)
    ny = nx = 256
    ps, dz, E = 0.1, 2.0, 200e3
    V = random_gaussian_stack(rng, n_slices, ny, nx, ps, 30, 20.0, 0.3) / dz
    probe = aperture_probe(ny, nx, ps, E, 20.0, 0.0, dtype=np.complex64)
    return Workload("fresnel_256_N20", ny, nx, ps, n_slices, dz, E,
                    V[None].astype(np.float32), probe, method="fresnel")


def angular_spectrum_diamond(seed=0, n_slices=100, n=1024):
    """1024^2, 0.05 A, 100 x 1.3575 A slices, 300 keV, plane wave, diamond
    [100] (a = 5.43 A), Gaussian atoms 25 V*A / 0.25 A, 0.08 A jitter."""
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.05, 1.3575, 300e3
    V = lattice_stack(rng, n_slices, n, n, ps, 5.43, DIAMOND_LAYERS, 25.0, 0.25, 0.08) / dz
    probe = np.ones((n, n), np.complex64)
    return Workload(f"as_diamond_{n}_N{n_slices}", n, n, ps, n_slices, dz, E,
                    V[None].astype(np.float32), probe, method="as")


def wpm_fcc(seed=0, n_slices=200, n=512, n_bins=16, power_spacing=1.0):
    """512^2, 0.05 A, 200 x 2.04 A slices, 300 keV, plane wave, FCC [100]
    (a = 4.08 A), Gaussian atoms 80 V*A / 0.2 A, 0.07 A jitter, K = 16 bins."""
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.05, 2.04, 300e3
    V = lattice_stack(rng, n_slices, n, n, ps, 4.08, FCC_LAYERS, 80.0, 0.2, 0.07) / dz
    probe = np.ones((n, n), np.complex64)
    return Workload(f"wpm_fcc_{n}_N{n_slices}_K{n_bins}", n, n, ps, n_slices, dz, E,
                    V[None].astype(np.float32), probe, method="wpm",
                    n_bins=n_bins, power_spacing=power_spacing)


def batched_scan_class(seed, n, n_slices, n_side, n_draws):
    """One grid class of the batched 4D-STEM scan: diamond [100] lattice at
    0.05 A, 300 keV, 25 mrad / -50 A defocus probe, an n_side x n_side raster
    of integer probe positions, repeated over ``n_draws`` frozen-phonon
    draws of the potential."""
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.05, 1.3575, 300e3
    V = np.stack([lattice_stack(rng, n_slices, n, n, ps, 5.43, DIAMOND_LAYERS, 25.0, 0.25, 0.08) / dz
                  for _ in range(n_draws)]).astype(np.float32)
    probe = aperture_probe(n, n, ps, E, 25.0, -50.0, dtype=np.complex64)
    pos = raster_positions(n, n, n_side, n_side)
    positions = np.concatenate([pos] * n_draws)
    draws = np.repeat(np.arange(n_draws, dtype=np.int32), pos.shape[0])
    return Workload(f"scan_{n}_N{n_slices}_B{positions.shape[0]}", n, n, ps, n_slices, dz, E,
                    V, probe, positions=positions.astype(np.int32),
                    draw_of_probe=draws, method="as")


def batched_scan_class_atoms(seed, n, n_slices, n_side, n_draws):
    """Atom lists behind ``batched_scan_class`` (same seed, same draws):
    positions (M, 2) in A and the row of each atom in the (n_draws * n_slices)
    stack of slices; the potential is these atoms as 25 V*A / 0.25 A Gaussians
    divided by the slice thickness 1.3575 A."""
    rng = np.random.default_rng(seed)
    pos, rows = [], []
    for d in range(n_draws):
        p, s = lattice_atoms(rng, n_slices, n, n, 0.05, 5.43, DIAMOND_LAYERS, 0.08)
        pos.append(p)
        rows.append(s + d * n_slices)
    return np.concatenate(pos), np.concatenate(rows)


def batched_scan(seed=0, small=False):
    """The uneven batch: 1024 probes on 256^2 (16x16 raster x 4 phonon draws,
    80 slices) + 64 probes on 512^2 (8x8 raster, 150 slices).  ``small``
    shrinks counts for tests."""
    if small:
        return [batched_scan_class(seed, 64, 6, 4, 2), batched_scan_class(seed + 1, 128, 5, 2, 1)]
    return [batched_scan_class(seed, 256, 80, 16, 4), batched_scan_class(seed + 1, 512, 150, 8, 1)]


def inverse_problem(seed=0, n=512, n_slices=64, n_side=8):
    """Gradient workload: 512^2, 64 x 2 A slices, 300 keV, 8x8 probe raster;
    the target potential is a seed-drawn 30-Gaussians/slice stack (20 V*A,
    0.3 A) and the unknown starts at zero."""
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.05, 2.0, 300e3
    Vt = random_gaussian_stack(rng, n_slices, n, n, ps, 30, 20.0, 0.3) / dz
    probe = aperture_probe(n, n, ps, E, 25.0, -50.0, dtype=np.complex64)
    pos = raster_positions(n, n, n_side, n_side)
    return Workload(f"inverse_{n}_N{n_slices}_B{pos.shape[0]}", n, n, ps, n_slices, dz, E,
                    Vt[None].astype(np.float32), probe, positions=pos,
                    draw_of_probe=np.zeros(pos.shape[0], np.int32), method="fresnel")
