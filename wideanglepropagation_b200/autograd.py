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

import ctypes
import threading

from . import _lib
from .propagation import (SCAN_MIN_PROBES, SCAN_SIZES, StreamOrder, _detector, _device, _dp_shape, _prepare, _ptr,
                          get_plan, scan_class, split_transfer)

# gradient scans (persistent scheduler) by shape, each with the StreamOrder of
# its workspace; a scan is held from the forward until its backward has run,
# so several pending graphs get their own
_pool: dict = {}
_pool_lock = threading.Lock()


def _acquire(key, cls, k):
    arr = (_lib.ScanClass * 1)(cls)
    ptr = ctypes.cast(arr, ctypes.c_void_p)
    L = _lib.lib()
    with _pool_lock:
        free = _pool.setdefault(key, [])
        if free:
            h, order = free.pop()
            _lib.check(L.wap_scan_bind(h, 1, ptr))
            return h, order
    h = ctypes.c_void_p()
    _lib.check(L.wap_scan_grad_create(ctypes.byref(h), ptr, int(k)))
    return h, StreamOrder()


_POOL_IDLE_MAX = 2   # idle gradient scans kept per shape (each holds its checkpoints and segment waves)


def _release(key, h, order):
    with _pool_lock:
        free = _pool.setdefault(key, [])
        if len(free) < _POOL_IDLE_MAX:
            free.append((h, order))
            return
    _lib.lib().wap_scan_destroy(h)


def release_pool() -> None:
    """Destroy every idle pooled gradient scan (scans held by pending graphs stay)."""
    with _pool_lock:
        handles = [h for free in _pool.values() for h, _ in free]
        _pool.clear()
    if handles:
        torch.cuda.synchronize()
        for h in handles:
            _lib.lib().wap_scan_destroy(h)


class _Lease:
    """A pooled gradient scan held by one forward: returned to the pool by
    its backward, or when the graph is freed without a backward."""

    def __init__(self, key, h, order):
        self.key, self.h, self.order, self.done = key, h, order, False

    def release(self):
        if not self.done:
            self.done = True
            _release(self.key, self.h, self.order)

    def __del__(self):
        self.release()


class MultisliceFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, V, probe, H, dz, energy, positions, draw, ckpt_every, det, check=True):
        dev = V.device
        ctx.set_materialize_grads(False)
        Vc, psi, per_probe, pos, dr, B, N, ny, nx, batched = _prepare(V.detach(), probe, positions, draw, dev)
        Hc, Hl = split_transfer(H, dev)
        ctx.scan = None
        if ctx.needs_input_grad[0] and ny == nx and ny in SCAN_SIZES and B >= SCAN_MIN_PROBES and not per_probe:
            # persistent scheduler: forward with checkpoints now, adjoint later
            exit_wave = torch.empty((B, ny, nx), dtype=torch.complex64, device=dev)
            dp = torch.empty(_dp_shape(B, ny, nx, det), dtype=torch.float32, device=dev)
            k = max(1, min(int(ckpt_every), N))
            key = (torch.cuda.current_device(), ny, N, Vc.shape[0], B, k)
            h, order = _acquire(key, scan_class(Vc, psi, pos, dr, Hc, Hl, dz, energy, exit_wave, dp, det), k)
            ctx.scan = _Lease(key, h, order)
            cur = order.begin(torch.cuda.current_stream(dev))
            _lib.check(_lib.lib().wap_scan_run(h, ctypes.c_void_p(cur.cuda_stream)))
            ctx.check = check
            token = _lib.scan_status_begin(h, f"gradient scan forward of {B} probes on {ny}x{nx}, {N} slices",
                                           stream=cur)
            order.end(cur)
            if check:
                _lib.scan_status_end(token)
            else:
                _lib.defer_status(token)
            # everything the scan reads in the backward must outlive it.  The
            # exit wave is an output: it goes through save_for_backward (a
            # plain attribute would tie output -> graph -> ctx -> output in a
            # cycle that only the garbage collector frees)
            ctx.keep = (psi, pos, dr, Hc, Hl)
            ctx.save_for_backward(Vc, exit_wave)
            ctx.meta = (B, N, ny, nx, float(dz), float(energy), k, dr is not None, V.shape, batched, det)
            if not batched:
                return exit_wave[0], dp[0]
            return exit_wave, dp
        plan = get_plan(ny, nx, B, _lib.WAP_OP_FRESNEL_AS)
        plan.set_detector(det)
        k = max(1, int(ckpt_every))
        nck = (N + k - 1) // k
        exit_wave = torch.empty((B, ny, nx), dtype=torch.complex64, device=dev)
        dp = torch.empty(_dp_shape(B, ny, nx, det), dtype=torch.float32, device=dev)
        ckpt = torch.empty((B, nck, ny, nx), dtype=torch.complex64, device=dev)
        cur = plan.begin()
        _lib.check(_lib.lib().wap_multislice_fwd_ckpt(
            plan.handle, _ptr(Vc), N, Vc.shape[0], _ptr(dr), _ptr(psi), B, 1 if per_probe else 0,
            _ptr(pos), _ptr(Hc), _ptr(Hl), float(dz), float(energy), _ptr(exit_wave), _ptr(dp), _ptr(ckpt), k,
            ctypes.c_void_p(cur.cuda_stream)))
        plan.end(cur)
        empty = torch.empty(0, device=dev)
        ctx.save_for_backward(Vc, Hc, Hl if Hl is not None else empty, exit_wave, ckpt,
                              dr if dr is not None else empty)
        ctx.meta = (B, N, ny, nx, float(dz), float(energy), k, dr is not None, V.shape, batched, det)
        if not batched:
            return exit_wave[0], dp[0]
        return exit_wave, dp

    @staticmethod
    def backward(ctx, g_exit, g_dp):
        if ctx.scan is not None:
            lease = ctx.scan
            Vc, _ = ctx.saved_tensors
            B, N, ny, nx, dz, energy, k, has_draw, vshape, batched, det = ctx.meta
            try:
                grad_V = torch.zeros(Vc.shape, dtype=torch.float32, device=Vc.device)
                if g_exit is None and g_dp is None:
                    return grad_V.reshape(vshape), None, None, None, None, None, None, None, None, None
                g = None if g_dp is None else g_dp.to(torch.float32).reshape(_dp_shape(B, ny, nx, det)).contiguous()
                ge = None if g_exit is None else g_exit.to(torch.complex64).reshape(B, ny, nx).contiguous()
                cur = lease.order.begin(torch.cuda.current_stream(Vc.device))
                _lib.check(_lib.lib().wap_scan_grad_backward_ex(lease.h, _ptr(g), _ptr(ge), _ptr(grad_V),
                                                                ctypes.c_void_p(cur.cuda_stream)))
                token = _lib.scan_status_begin(lease.h, f"gradient scan backward of {B} probes on {ny}x{nx}, "
                                                        f"{N} slices", stream=cur)
                lease.order.end(cur)
                if ctx.check:
                    _lib.scan_status_end(token)
                else:
                    _lib.defer_status(token)
                return grad_V.reshape(vshape), None, None, None, None, None, None, None, None, None
            finally:
                lease.release()
        Vc, Hc, Hl, exit_wave, ckpt, dr = ctx.saved_tensors
        B, N, ny, nx, dz, energy, k, has_draw, vshape, batched, det = ctx.meta
        dev = Vc.device
        plan = get_plan(ny, nx, B, _lib.WAP_OP_FRESNEL_AS)
        plan.set_detector(det)
        if g_exit is not None:
            g_exit = g_exit.to(torch.complex64).reshape(B, ny, nx).contiguous()
        if g_dp is not None:
            g_dp = g_dp.to(torch.float32).reshape(_dp_shape(B, ny, nx, det)).contiguous()
        grad_V = torch.zeros(Vc.shape, dtype=torch.float32, device=dev)
        work = torch.empty((B, k + 2, ny, nx), dtype=torch.complex64, device=dev)
        cur = plan.begin()
        _lib.check(_lib.lib().wap_multislice_bwd(
            plan.handle, _ptr(Vc), N, Vc.shape[0], _ptr(dr) if has_draw else None, B, _ptr(Hc),
            _ptr(Hl) if Hl.numel() else None, dz, energy,
            _ptr(exit_wave), _ptr(ckpt), k, _ptr(g_dp), _ptr(g_exit), _ptr(grad_V), _ptr(work),
            ctypes.c_void_p(cur.cuda_stream)))
        plan.end(cur)
        return grad_V.reshape(vshape), None, None, None, None, None, None, None, None, None


def simulate_fresnel_as_differentiable(potential: torch.Tensor, probe, prop_kernel, slice_thickness, energy, *,
                                       positions=None, draw=None, ckpt_every: int | None = None,
                                       max_angle=None, sampling=None, parity="odd", check: bool = True):
    """(exit_wave, diffraction_pattern) with gradients flowing to ``potential``.

    ``ckpt_every`` defaults to round(sqrt(N)) slices between saved waves.
    ``max_angle`` / ``sampling`` / ``parity``: the pattern is cropped to the
    detector window as in ``simulate_fresnel_as`` (the loss sees only it).
    On the persistent scheduler the forward and the backward raise WapError
    if a bounded device-side wait expired; ``check=False`` defers that to
    ``check_errors()`` (or the next call) instead of waiting for the GPU.
    """
    _device()
    _lib.poll_errors()
    if not isinstance(potential, torch.Tensor):
        raise TypeError("potential must be a torch tensor to differentiate")
    N = potential.shape[-3]
    if ckpt_every is None:
        ckpt_every = max(1, int(round(math.sqrt(N))))
    det = _detector(tuple(potential.shape[-2:]), sampling, energy, max_angle, parity)
    return MultisliceFunction.apply(potential, probe, prop_kernel, slice_thickness, energy, positions, draw,
                                    ckpt_every, det, check)
