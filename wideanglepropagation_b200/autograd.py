"""Differentiable Fresnel/AS multislice w.r.t. the potential.

``MultisliceFunction`` wraps the forward kernels (which also save the wave
entering every ``ckpt_every``-th slice) and the hand-written adjoint
(``wap_multislice_bwd``): it walks the checkpoint segments backwards,
recomputes the waves inside each segment, and sweeps the conjugate
propagator ifft2(conj(H) fft2(.)) in reverse slice order while accumulating

    dL/dV_s = sum_probes 2 Re(conj(lambda_s) i t_s psi_s) dphi/dV,
    phi = 2 pi (n(V) - 1) dz / lambda,
    dphi/dV = (2 pi dz / lambda) (E + E0 + V) / (n (2 E E0 + E^2)).

The reference has no gradient code of its own; its paper claims autodiff
through JAX (Paper/main.tex:271-274, :325-327).  The convention for complex
outputs is torch's (grad = dL/dRe + i dL/dIm).
"""
from __future__ import annotations

import math

import torch

from . import _lib
from .propagation import _device, _prepare, _ptr, _stream, get_plan, split_transfer


class MultisliceFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, V, probe, H, dz, energy, positions, draw, ckpt_every):
        dev = V.device
        Vc, psi, per_probe, pos, dr, B, N, ny, nx, batched = _prepare(V.detach(), probe, positions, draw, dev)
        Hc, Hl = split_transfer(H, dev)
        plan = get_plan(ny, nx, B, _lib.WAP_OP_FRESNEL_AS)
        k = max(1, int(ckpt_every))
        nck = (N + k - 1) // k
        exit_wave = torch.empty((B, ny, nx), dtype=torch.complex64, device=dev)
        dp = torch.empty((B, ny, nx), dtype=torch.float32, device=dev)
        ckpt = torch.empty((B, nck, ny, nx), dtype=torch.complex64, device=dev)
        _lib.check(_lib.lib().wap_multislice_fwd_ckpt(
            plan.handle, _ptr(Vc), N, Vc.shape[0], _ptr(dr), _ptr(psi), B, 1 if per_probe else 0,
            _ptr(pos), _ptr(Hc), _ptr(Hl), float(dz), float(energy), _ptr(exit_wave), _ptr(dp), _ptr(ckpt), k,
            _stream()))
        empty = torch.empty(0, device=dev)
        ctx.save_for_backward(Vc, Hc, Hl if Hl is not None else empty, exit_wave, ckpt,
                              dr if dr is not None else empty)
        ctx.meta = (B, N, ny, nx, float(dz), float(energy), k, dr is not None, V.shape, batched)
        if not batched:
            return exit_wave[0], dp[0]
        return exit_wave, dp

    @staticmethod
    def backward(ctx, g_exit, g_dp):
        Vc, Hc, Hl, exit_wave, ckpt, dr = ctx.saved_tensors
        B, N, ny, nx, dz, energy, k, has_draw, vshape, batched = ctx.meta
        dev = Vc.device
        plan = get_plan(ny, nx, B, _lib.WAP_OP_FRESNEL_AS)
        if g_exit is not None:
            g_exit = g_exit.to(torch.complex64).reshape(B, ny, nx).contiguous()
        if g_dp is not None:
            g_dp = g_dp.to(torch.float32).reshape(B, ny, nx).contiguous()
        grad_V = torch.zeros(Vc.shape, dtype=torch.float32, device=dev)
        work = torch.empty((B, k + 2, ny, nx), dtype=torch.complex64, device=dev)
        _lib.check(_lib.lib().wap_multislice_bwd(
            plan.handle, _ptr(Vc), N, Vc.shape[0], _ptr(dr) if has_draw else None, B, _ptr(Hc),
            _ptr(Hl) if Hl.numel() else None, dz, energy,
            _ptr(exit_wave), _ptr(ckpt), k, _ptr(g_dp), _ptr(g_exit), _ptr(grad_V), _ptr(work), _stream()))
        return grad_V.reshape(vshape), None, None, None, None, None, None, None


def simulate_fresnel_as_differentiable(potential: torch.Tensor, probe, prop_kernel, slice_thickness, energy, *,
                                       positions=None, draw=None, ckpt_every: int | None = None):
    """(exit_wave, diffraction_pattern) with gradients flowing to ``potential``.

    ``ckpt_every`` defaults to round(sqrt(N)) slices between saved waves.
    """
    _device()
    if not isinstance(potential, torch.Tensor):
        raise TypeError("potential must be a torch tensor to differentiate")
    N = potential.shape[-3]
    if ckpt_every is None:
        ckpt_every = max(1, int(round(math.sqrt(N))))
    return MultisliceFunction.apply(potential, probe, prop_kernel, slice_thickness, energy, positions, draw,
                                    ckpt_every)
