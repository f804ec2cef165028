"""Device-side potential builders.

``gaussian_potential`` builds the per-slice projected potential of Gaussian
atoms on the device (``wap_gaussian_potential``), so a multislice call can
start from an atom list of a few kilobytes instead of a host-built potential
of hundreds of megabytes and its host->device copy.  The reference builds its
potentials on the host through abTEM (``get_abtem_transmit``,
propagation.py:286-299); this package's workloads use the Gaussian-atom model
of its benchmark configurations, which this builder evaluates.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib
from .propagation import _device, _pair, _ptr, _stream


def gaussian_potential(n_slices: int, ny: int, nx: int, ps, positions, slices, amp, sigma: float,
                       scale: float = 1.0) -> torch.Tensor:
    """(n_slices, ny, nx) float32 on the device:
    ``scale * sum_a amp_a exp(-(dy^2 + dx^2) / (2 sigma^2))`` per slice, periodic.

    positions  (M, 2) atom centres (y, x) in A
    slices     (M,) slice index of each atom
    amp        scalar or (M,) amplitudes (V*A)
    scale      e.g. ``1 / slice_thickness`` for a potential in volts
    """
    dev = _device()
    ps_y, ps_x = _pair(ps)
    pos = np.asarray(positions, dtype=np.float64).reshape(-1, 2)
    sl = np.asarray(slices, dtype=np.int64).reshape(-1)
    if sl.shape[0] != pos.shape[0]:
        raise ValueError("one slice index per atom")
    if sl.size and (sl.min() < 0 or sl.max() >= n_slices):
        raise ValueError("slice index out of range")
    a = np.broadcast_to(np.asarray(amp, dtype=np.float64), (pos.shape[0],))
    order = np.argsort(sl, kind="stable")
    atoms = np.concatenate([pos[order], a[order][:, None]], axis=1)
    start = np.concatenate([[0], np.cumsum(np.bincount(sl, minlength=n_slices))]).astype(np.int32)
    if not atoms.size:
        atoms = np.zeros((1, 3))   # no atoms at all: every slice_start is 0, the row is never read
    d_atoms = torch.as_tensor(np.ascontiguousarray(atoms)).to(dev)
    d_start = torch.as_tensor(start).to(dev)
    V = torch.empty((n_slices, ny, nx), dtype=torch.float32, device=dev)
    _lib.check(_lib.lib().wap_gaussian_potential(n_slices, ny, nx, ps_y, ps_x, _ptr(d_atoms), _ptr(d_start),
                                                 float(sigma), float(scale), _ptr(V), _stream()))
    return V
