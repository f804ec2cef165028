"""1D line helpers (propagation.py:609-652) and the naive WPM step (:184-212).

Same names and argument meaning as the reference; the work runs in
``csrc/wap_lines.cu``:

* ``fresnel_kernel_1d`` / ``angular_spectrum_kernel_1d`` - float64 transfer
  functions on the device (complex128 results, as the reference's);
* ``propagate_1d`` - ifft(fft(psi) H) per line on the radix-16 FFT core
  (complex64 lines, H applied as complex64 hi + lo parts of a complex128 H);
* ``wpm_kernel_1d`` / ``wpm_kernel_1d_vmap`` - one line per refractive index,
  the transfer function evaluated in float64 inside the kernel;
* ``wpm_step`` - the per-pixel WPM step as direct float64 sums: an exactness
  check for the binned WPM on small grids (any shape up to 65536 pixels).

Line lengths for the FFT helpers are powers of two in [32, 2048]
(``ValueError`` otherwise); the reference accepts any length.
"""
from __future__ import annotations

import math

import torch

from . import _lib
from .propagation import _device, _fftfreq, _pair, _ptr, _stream, _to, split_transfer

__all__ = ["get_kx_1d", "fresnel_kernel_1d", "angular_spectrum_kernel_1d", "propagate_1d", "wpm_kernel_1d",
           "wpm_kernel_1d_vmap", "wpm_step"]


def get_kx_1d(n: int, dx: float) -> torch.Tensor:
    """Angular spatial frequencies 2 pi fftfreq(n, dx) (propagation.py:609-614), float64."""
    return 2 * math.pi * _fftfreq(int(n), float(dx), _device())


def _line_transfer(kind: int, kx_sq, k0: float, dy: float) -> torch.Tensor:
    dev = _device()
    kx = _to(kx_sq, torch.float64, dev)
    kx2 = kx.reshape(-1)
    out = torch.empty(kx2.shape[0], dtype=torch.complex128, device=dev)
    _lib.check(_lib.lib().wap_line_transfer(kind, kx2.shape[0], _ptr(kx2), float(k0), float(dy), _ptr(out),
                                            _stream()))
    return out.reshape(kx.shape)


def fresnel_kernel_1d(kx_sq, k0, dy) -> torch.Tensor:
    """exp(-i kx^2 dy / (2 k0)) (propagation.py:617-619), complex128."""
    return _line_transfer(_lib.WAP_TF_FRESNEL, kx_sq, k0, dy)


def angular_spectrum_kernel_1d(kx_sq, k0, dy) -> torch.Tensor:
    """exp(i dy sqrt(k0^2 - kx^2)) with the complex square root (propagation.py:622-626)."""
    return _line_transfer(_lib.WAP_TF_ANGULAR, kx_sq, k0, dy)


def propagate_1d(psi, H) -> torch.Tensor:
    """ifft(fft(psi) * H) along the last axis (propagation.py:629-633).

    ``psi`` (..., n); ``H`` (n,) shared by every line, or the same shape as
    ``psi``.  Returns complex64 of ``psi``'s shape.
    """
    dev = _device()
    x = _to(psi, torch.complex64, dev)
    n = x.shape[-1]
    lines = x.reshape(-1, n)
    Hh, Hl = split_transfer(H, dev)
    if Hh.shape[-1] != n:
        raise ValueError(f"H has {Hh.shape[-1]} points, psi lines have {n}")
    per_line = Hh.numel() != n
    if per_line and Hh.numel() != lines.numel():
        raise ValueError("H must be (n,) or the shape of psi")
    out = torch.empty_like(lines)
    _lib.check(_lib.lib().wap_line_propagate(n, lines.shape[0], _ptr(lines), _ptr(Hh), _ptr(Hl), 1 if per_line else 0,
                                             _ptr(out), _stream()))
    return out.reshape(x.shape)


def wpm_kernel_1d_vmap(psi_k, n_vals, k0, kx_sq, dy) -> torch.Tensor:
    """ifft(psi_k exp(i dy sqrt((n k0)^2 - kx^2))) for every n in ``n_vals``
    (propagation.py:636-652); returns (len(n_vals), n) complex64."""
    dev = _device()
    pk = _to(psi_k, torch.complex64, dev).reshape(-1)
    nv = _to(n_vals, torch.float64, dev).reshape(-1)
    kx2 = _to(kx_sq, torch.float64, dev).reshape(-1)
    n = pk.shape[0]
    if kx2.shape[0] != n:
        raise ValueError("kx_sq and psi_k differ in length")
    out = torch.empty((nv.shape[0], n), dtype=torch.complex64, device=dev)
    _lib.check(_lib.lib().wap_line_wpm(n, nv.shape[0], _ptr(pk), _ptr(nv), float(k0), _ptr(kx2), float(dy), _ptr(out),
                                       _stream()))
    return out


def wpm_kernel_1d(psi_k, n_val, k0, kx_sq, dy) -> torch.Tensor:
    """WPM 1D kernel for one refractive index (propagation.py:636-649)."""
    return wpm_kernel_1d_vmap(psi_k, [float(n_val)], k0, kx_sq, dy)[0]


def wpm_step(wave, n_map, dz, energy, ps) -> torch.Tensor:
    """Naive WPM step (propagation.py:184-212): every pixel takes its own full
    propagate with its own refractive index.  Returns (ny, nx) complex128."""
    dev = _device()
    w = _to(wave, torch.complex128, dev)
    nm = _to(n_map, torch.float64, dev)
    if w.ndim != 2 or nm.shape != w.shape:
        raise ValueError("wave and n_map must be (ny, nx) of the same shape")
    ny, nx = w.shape
    p0, p1 = _pair(ps)
    out = torch.empty_like(w)
    work = torch.empty(2 * ny * nx, dtype=torch.complex128, device=dev)
    _lib.check(_lib.lib().wap_wpm_naive_step(ny, nx, _ptr(w), _ptr(nm), float(dz), float(energy), p0, p1, _ptr(out),
                                             _ptr(work), _stream()))
    return out
