"""Lippmann-Schwinger 2D solver (propagation.py:446-602) on the device.

The scattering problem (I - G V_scale V) psi = psi_inc is solved by restarted
GMRES whose operator applications - the FFT convolutions with the Green's
function, the part that repeats - run in libwap.so's 2D transform kernels:
``apply_convolution`` embeds the source, applies ifft2(K_hat fft2(.)) through
the one-slice propagator with K_hat as its transfer function (complex64 hi +
lo parts of the complex128 K_hat), and crops.  The Green's function kernel is
built once per solve on the host in float64 (scipy's Hankel function and a
NumPy FFT), as the reference builds it (propagation.py:464-501).  The Krylov
basis and the small Hessenberg problem are kept in complex128.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .propagation import _device, _ptr, _to, get_plan, split_transfer

__all__ = ["build_lippmann_schwinger_kernel_2d", "apply_convolution", "solve_scattering_2d_lippmann_schwinger"]

# CODATA-2014 constants of ase.units used by the reference solver (propagation.py:540-547)
_HPLANCK = 6.626070040e-34
_ME = 9.10938356e-31
_C = 299792458.0
_QE = 1.6021766208e-19


def _greens_2d_hankel(k0, r):
    from scipy.special import hankel1
    return 0.25j * hankel1(0, k0 * r)


def build_lippmann_schwinger_kernel_2d(k0, hx, hy, Nx, Ny, pad_to_double=True, oversamp_self=32):
    """FFT of the centre-embedded Green's function kernel (i/4) H0(k0 r) hx hy,
    the singular cell replaced by its cell average (propagation.py:454-501).

    Returns (K_hat on the device, complex128, (Ex, Ey))."""
    Ex, Ey = (2 * Nx, 2 * Ny) if pad_to_double else (Nx, Ny)
    x = (np.arange(Nx) - Nx // 2) * hx
    y = (np.arange(Ny) - Ny // 2) * hy
    X, Y = np.meshgrid(x, y, indexing="ij")
    K = (hx * hy) * _greens_2d_hankel(k0, np.sqrt(X ** 2 + Y ** 2))
    s = (np.arange(oversamp_self) + 0.5) / oversamp_self
    SX, SY = np.meshgrid(s * hx - 0.5 * hx, s * hy - 0.5 * hy, indexing="ij")
    K[Nx // 2, Ny // 2] = _greens_2d_hankel(k0, np.sqrt(SX ** 2 + SY ** 2)).mean() * (hx * hy)
    Kemb = np.zeros((Ex, Ey), dtype=np.complex128)
    sx, sy = (Ex - Nx) // 2, (Ey - Ny) // 2
    Kemb[sx:sx + Nx, sy:sy + Ny] = K
    Khat = np.fft.fftn(np.fft.ifftshift(Kemb))
    return torch.as_tensor(Khat).to(_device()), (Ex, Ey)


class _Convolution:
    """ifft2(K_hat fft2(embed(source)))[roi] with the device transform kernels."""

    def __init__(self, Khat, embed_shape, roi_shape):
        dev = _device()
        self.Ex, self.Ey = embed_shape
        self.Nx, self.Ny = roi_shape
        self.sx, self.sy = (self.Ex - self.Nx) // 2, (self.Ey - self.Ny) // 2
        self.Kh, self.Kl = split_transfer(Khat, dev)
        if tuple(self.Kh.shape) != (self.Ex, self.Ey):
            raise ValueError(f"K_hat shape {tuple(self.Kh.shape)} does not match the embedding {embed_shape}")
        self.V0 = torch.zeros((1, self.Ex, self.Ey), dtype=torch.float32, device=dev)   # transmission exactly 1
        self.src = torch.zeros((self.Ex, self.Ey), dtype=torch.complex64, device=dev)
        self.out = torch.empty((self.Ex, self.Ey), dtype=torch.complex64, device=dev)

    def __call__(self, source: torch.Tensor) -> torch.Tensor:
        plan = get_plan(self.Ex, self.Ey, 1, _lib.WAP_OP_FRESNEL_AS)
        self.src.zero_()
        self.src[self.sx:self.sx + self.Nx, self.sy:self.sy + self.Ny] = source
        cur = plan.begin()
        _lib.check(_lib.lib().wap_multislice_fwd(
            plan.handle, _ptr(self.V0), 1, 1, None, _ptr(self.src), 1, 0, None, _ptr(self.Kh), _ptr(self.Kl),
            1.0, 1.0e5, _ptr(self.out), None, None, ctypes.c_void_p(cur.cuda_stream)))
        plan.end(cur)
        return self.out[self.sx:self.sx + self.Nx, self.sy:self.sy + self.Ny]


def apply_convolution(source, Khat, embed_shape, roi_shape):
    """FFT convolution of ``source`` with the kernel (propagation.py:504-514);
    complex64 result on the device."""
    src = _to(source, torch.complex64, _device())
    return _Convolution(Khat, embed_shape, roi_shape)(src).clone()


def _gmres(A, b, tol, restart, maxiter):
    """Restarted GMRES(restart): stops when ||b - A x|| <= tol ||b|| (the
    criterion of jax.scipy.sparse.linalg.gmres / scipy's rtol).  Two-pass
    classical Gram-Schmidt on the device, complex Givens rotations on the host.
    Returns (x, info) with info = 0 on convergence."""
    n = b.numel()
    x = torch.zeros_like(b)
    atol = tol * float(torch.linalg.vector_norm(b))
    for _ in range(maxiter):
        r = b - A(x)
        beta = float(torch.linalg.vector_norm(r))
        if beta <= atol:
            return x, 0
        m = min(restart, n)
        Q = torch.empty((m + 1, n), dtype=b.dtype, device=b.device)
        Q[0] = r / beta
        R = np.zeros((m + 1, m), dtype=np.complex128)
        cs = np.zeros(m)
        sn = np.zeros(m, dtype=np.complex128)
        g = np.zeros(m + 1, dtype=np.complex128)
        g[0] = beta
        k = 0
        for j in range(m):
            w = A(Q[j])
            h = Q[:j + 1].conj() @ w
            w = w - Q[:j + 1].T @ h
            h2 = Q[:j + 1].conj() @ w
            w = w - Q[:j + 1].T @ h2
            hn = float(torch.linalg.vector_norm(w))
            col = np.zeros(m + 1, dtype=np.complex128)
            col[:j + 1] = (h + h2).cpu().numpy()
            col[j + 1] = hn
            for i in range(j):   # earlier rotations
                a, c = col[i], col[i + 1]
                col[i] = cs[i] * a + sn[i] * c
                col[i + 1] = -np.conj(sn[i]) * a + cs[i] * c
            a, c = col[j], col[j + 1]
            rho = math.hypot(abs(a), abs(c))
            if rho == 0.0:
                cs[j], sn[j] = 1.0, 0.0
            elif abs(a) == 0.0:
                cs[j], sn[j] = 0.0, 1.0
            else:
                cs[j], sn[j] = abs(a) / rho, (a / abs(a)) * np.conj(c) / rho
            col[j] = cs[j] * a + sn[j] * c
            col[j + 1] = 0.0
            g[j + 1] = -np.conj(sn[j]) * g[j]
            g[j] = cs[j] * g[j]
            R[:, j] = col
            k = j + 1
            if hn > 0.0:
                Q[j + 1] = w / hn
            if abs(g[j + 1]) <= atol or hn == 0.0:
                break
        y = np.linalg.solve(np.triu(R[:k, :k]), g[:k])
        x = x + Q[:k].T @ torch.as_tensor(y, device=b.device)
    r = b - A(x)
    return x, 0 if float(torch.linalg.vector_norm(r)) <= atol else 1


def solve_scattering_2d_lippmann_schwinger(potential_grid, energy_ev, pixel_size_A, pad_factor=2, absorb_frac=0.15,
                                           absorb_strength=4.0, gmres_tol=1e-4, gmres_restart=70,
                                           gmres_maxiter=200):
    """Total wave of the 2D scalar Helmholtz problem for a pixelised potential
    (volts, shape (Nx, Ny)) and a plane wave exp(i k0 y) along axis 1, by the
    Lippmann-Schwinger equation on a ``pad_factor``-padded grid
    (propagation.py:517-602).  ``absorb_frac`` / ``absorb_strength`` are
    accepted and unused, as in the reference.  The padded grid times two (the
    convolution grid) must be a power of two in [32, 2048] or any size in
    [17, 1024] per axis (Bluestein transforms).  Returns complex128 (Nx, Ny)."""
    dev = _device()
    hbar = _HPLANCK / (2 * np.pi)
    gamma = 1.0 + energy_ev / (_ME * _C ** 2 / _QE)
    V_scale = -(2.0 * gamma * _ME * _QE / hbar ** 2) * 1e-20
    m0, hc = 510998.95000, 12398.4193
    k0 = 2 * np.pi / (hc / np.sqrt(energy_ev * (energy_ev + 2 * m0)))
    V = _to(potential_grid, torch.float64, dev)
    orig = tuple(V.shape)
    padded = tuple(s * pad_factor for s in orig)
    pad = [((p - o) // 2, (p - o) - (p - o) // 2) for p, o in zip(padded, orig)]
    Vp = torch.zeros(padded, dtype=torch.float64, device=dev)
    Vp[pad[0][0]:pad[0][0] + orig[0], pad[1][0]:pad[1][0] + orig[1]] = V
    Khat, emb = build_lippmann_schwinger_kernel_2d(float(k0), float(pixel_size_A), float(pixel_size_A),
                                                   padded[0], padded[1])
    conv = _Convolution(Khat, emb, padded)
    coupling = (V_scale * Vp).to(torch.complex128)

    def A(v):
        psi = v.reshape(padded)
        scattered = conv((coupling * psi).to(torch.complex64)).to(torch.complex128)
        return (psi - scattered).reshape(-1)

    y = torch.arange(padded[1], dtype=torch.float64, device=dev) * pixel_size_A
    y = y - y.mean()
    b = torch.exp(1j * k0 * y).expand(padded).reshape(-1).contiguous()
    x, info = _gmres(A, b, float(gmres_tol), int(gmres_restart), int(gmres_maxiter))
    if info != 0:
        print(f"  Warning: GMRES did not converge (info={info})")
    x = x.reshape(padded)
    return x[pad[0][0]:pad[0][0] + orig[0], pad[1][0]:pad[1][0] + orig[1]]
