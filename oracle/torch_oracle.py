"""Gradient oracle: the reference Fresnel/AS multislice restated in torch
complex128 on the CPU, differentiated by torch autograd.

TEST INFRASTRUCTURE ONLY (stand-in for ``jax.grad`` of the reference, which
cannot run here: jax is not installed).  Restates
``wide_angle_propagation/propagation.py``:66-81 (n(V)), :178-181
(Propagator), :263-276 (move_probe), :305-352 (simulate_fresnel_as).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .propagation_oracle import electron_rest_energy, energy2wavelength


def simulate(V, probe, H, dz, energy, positions=None, device=None):
    """V: (N, ny, nx) float64 tensor (may require grad); probe (ny, nx) complex;
    returns (exit (B, ny, nx), dp (B, ny, nx)).  Runs on V's device (or
    ``device`` when V is not a tensor); float64 / complex128 throughout."""
    lam = energy2wavelength(energy)
    E0 = electron_rest_energy()
    if not isinstance(V, torch.Tensor):
        V = torch.as_tensor(np.asarray(V, dtype=np.float64), device=device)
    dev = V.device
    H = torch.as_tensor(H).to(dev, torch.complex128)
    p = torch.as_tensor(probe).to(dev, torch.complex128)
    ny, nx = p.shape[-2:]
    if positions is None:
        waves = p[None] if p.ndim == 2 else p
    else:
        waves = torch.stack([torch.roll(p, (int(r) - ny // 2, int(c) - nx // 2), (0, 1)) for r, c in positions])
    for s in range(V.shape[0]):
        EmV = energy + V[s]
        n = torch.sqrt((2 * EmV * E0 + EmV ** 2) / (2 * energy * E0 + energy ** 2))     # :66-81
        t = torch.exp(1j * 2 * math.pi * (n - 1) * dz / lam)                              # :336
        waves = torch.fft.ifft2(H * torch.fft.fft2(waves * t))                            # :178-181
    Z = torch.fft.fftshift(torch.fft.fft2(waves), dim=(-2, -1))
    dp = Z.real ** 2 + Z.imag ** 2
    return waves, dp


def loss_and_grad(V, probe, H, dz, energy, target, positions=None):
    """L = sum (dp - target)^2 and dL/dV (float64 numpy)."""
    Vt = torch.tensor(np.asarray(V, dtype=np.float64), requires_grad=True)
    _, dp = simulate(Vt, probe, H, dz, energy, positions)
    L = ((dp - torch.as_tensor(target, dtype=torch.float64)) ** 2).sum()
    L.backward()
    return float(L), Vt.grad.numpy()
