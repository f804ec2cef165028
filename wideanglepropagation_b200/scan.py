"""Batched multislice scans: many probes, uneven grids, one submission.

A scan is a list of grid classes (e.g. 1024 probes on 256^2 windows plus 64
probes on 512^2 windows); each class has its own potential draws, probe,
positions and transfer function.  The reference runs such a scan as a caller
loop of ``simulate_fresnel_as(V, move_probe(probe, pos), H, dz, E)``
(propagation.py:263-276, :305-352); here every probe of every class is
advanced in the same kernels.  Three execution modes are offered:

``plain``       one probe per launch sequence (the reference's loop, on the GPU)
``batched``     per class, every pass covers all probes of the class
``graph``       ``batched`` captured once into a CUDA graph and replayed
``persistent``  every class in ONE persistent kernel (``wap_scan_run``: device
                ticket queue, L2-resident probe groups, TMA tile loads),
                captured once into a CUDA graph and replayed
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import torch

from . import _lib
from .propagation import _ptr, _stream, get_plan, transfer_pair


@dataclass
class DeviceClass:
    ny: int
    nx: int
    n_slices: int
    n_draws: int
    n_probes: int
    dz: float
    energy: float
    V: torch.Tensor           # (D, N, ny, nx) float32
    probe: torch.Tensor       # (ny, nx) complex64
    positions: torch.Tensor   # (B, 2) int32
    draw: torch.Tensor        # (B,) int32
    H: torch.Tensor           # (ny, nx) complex64 (hi part)
    H_lo: torch.Tensor        # (ny, nx) complex64 rounding remainder
    exit: torch.Tensor        # (B, ny, nx) complex64 (working buffer)
    dp: torch.Tensor          # (B, ny, nx) float32

    @property
    def slice_steps(self) -> int:
        return self.n_probes * self.n_slices

    @property
    def pixel_slice_steps(self) -> int:
        return self.slice_steps * self.ny * self.nx


def to_device_class(w, device=None) -> DeviceClass:
    """Upload a synthetic ``Workload`` and build its transfer function on the device."""
    dev = device or torch.device("cuda", torch.cuda.current_device())
    V = torch.as_tensor(w.potential, dtype=torch.float32).to(dev).contiguous()
    probe = torch.as_tensor(w.probe).to(dev, torch.complex64).contiguous()
    B = w.n_probes
    pos = torch.as_tensor(w.positions if w.positions is not None else np.array([[w.ny // 2, w.nx // 2]]),
                          dtype=torch.int32).to(dev).contiguous()
    draw = torch.as_tensor(w.draw_of_probe if w.draw_of_probe is not None else np.zeros(B, np.int32),
                           dtype=torch.int32).to(dev).contiguous()
    H, H_lo = transfer_pair(w.method, w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    return DeviceClass(w.ny, w.nx, w.n_slices, V.shape[0], B, w.dz, w.energy, V, probe, pos, draw, H, H_lo,
                       torch.empty((B, w.ny, w.nx), dtype=torch.complex64, device=dev),
                       torch.empty((B, w.ny, w.nx), dtype=torch.float32, device=dev))


def _fwd(c: DeviceClass, b0: int, nb: int) -> None:
    plan = get_plan(c.ny, c.nx, nb, _lib.WAP_OP_FRESNEL_AS)
    plane = c.ny * c.nx
    ex = ctypes.c_void_p(c.exit.data_ptr() + b0 * plane * 8)
    dp = ctypes.c_void_p(c.dp.data_ptr() + b0 * plane * 4)
    pos = ctypes.c_void_p(c.positions.data_ptr() + b0 * 8)
    dr = ctypes.c_void_p(c.draw.data_ptr() + b0 * 4)
    cur = plan.begin()
    _lib.check(_lib.lib().wap_multislice_fwd(
        plan.handle, _ptr(c.V), c.n_slices, c.n_draws, dr, _ptr(c.probe), nb, 0, pos, _ptr(c.H), _ptr(c.H_lo),
        c.dz, c.energy, ex, dp, None, ctypes.c_void_p(cur.cuda_stream)))
    plan.end(cur)


def launches_per_step(classes: List[DeviceClass], mode: str) -> int:
    """Kernel launches one step issues (two passes per slice plus the final row pass)."""
    per = [2 * c.n_slices + 1 for c in classes]
    if mode == "plain":
        return sum(p * c.n_probes for p, c in zip(per, classes))
    return sum(p * ((c.n_probes + 65534) // 65535) for p, c in zip(per, classes))


class PersistentScan:
    """Owns a ``wap_scan`` (device work queue over all classes)."""

    def __init__(self, classes: List[DeviceClass], groups: Optional[List[int]] = None):
        from . import autotune
        if groups is None:   # autotuned probe-group sizes (0: the scheduler's own)
            groups = [autotune.balanced_group(autotune.lookup_scan(c.ny), c.n_probes) if c.ny == c.nx else 0
                      for c in classes]
        arr = (_lib.ScanClass * len(classes))()
        for i, c in enumerate(classes):
            if c.ny != c.nx:
                raise ValueError("the persistent scheduler takes square grids")
            arr[i] = _lib.ScanClass(c.ny, c.n_slices, c.n_draws, c.n_probes, c.V.data_ptr(), c.draw.data_ptr(),
                                    c.probe.data_ptr(), c.positions.data_ptr(), c.H.data_ptr(),
                                    c.H_lo.data_ptr() if c.H_lo is not None else None, c.dz, c.energy,
                                    c.exit.data_ptr(), c.dp.data_ptr(), groups[i])
        h = ctypes.c_void_p()
        _lib.check(_lib.lib().wap_scan_create(ctypes.byref(h), len(classes), ctypes.cast(arr, ctypes.c_void_p)))
        self.handle = h
        self.classes = classes   # keeps the buffers alive

    def run(self) -> None:
        _lib.check(_lib.lib().wap_scan_run(self.handle, _stream()))

    def status(self) -> int:
        st = ctypes.c_int()
        rc = _lib.lib().wap_scan_status(self.handle, ctypes.byref(st))
        if rc not in (0, _lib.WAP_ERR_TIMEOUT):
            _lib.check(rc)
        return st.value

    def info(self) -> dict:
        t, g, g0 = ctypes.c_longlong(), ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().wap_scan_info(self.handle, ctypes.byref(t), ctypes.byref(g), ctypes.byref(g0)))
        return {"tickets": t.value, "grid": g.value, "group0": g0.value}

    def debug_stall(self, pass_index: int, spin_limit: int = 0) -> None:
        _lib.check(_lib.lib().wap_scan_debug_stall(self.handle, int(pass_index), int(spin_limit)))

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            _lib.lib().wap_scan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchedScan:
    """Runs a list of ``DeviceClass`` scans in one of the four modes."""

    def __init__(self, classes: List[DeviceClass], mode: str = "batched", plain_subset: Optional[int] = None,
                 groups: Optional[List[int]] = None):
        if mode not in ("plain", "batched", "graph", "persistent"):
            raise ValueError(f"unknown mode {mode!r}")
        self.classes = classes
        self.mode = mode
        self.plain_subset = plain_subset
        self.graph = None
        self.sched = PersistentScan(classes, groups) if mode == "persistent" else None
        for c in classes:   # create plans outside any capture
            get_plan(c.ny, c.nx, c.n_probes, _lib.WAP_OP_FRESNEL_AS)

    def _eager(self):
        if self.sched is not None:
            self.sched.run()
            return
        for c in self.classes:
            if self.mode == "plain":
                n = c.n_probes if self.plain_subset is None else min(self.plain_subset, c.n_probes)
                for b in range(n):
                    _fwd(c, b, 1)
            else:
                _fwd(c, 0, c.n_probes)

    def capture(self) -> None:
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self._eager()   # warm: attribute setup, plan tables
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self._eager()

    def step(self) -> None:
        if self.mode in ("graph", "persistent"):
            if self.graph is None:
                self.capture()
            self.graph.replay()
        else:
            self._eager()

    def slice_steps(self) -> int:
        if self.mode == "plain" and self.plain_subset is not None:
            return sum(min(self.plain_subset, c.n_probes) * c.n_slices for c in self.classes)
        return sum(c.slice_steps for c in self.classes)

    def launches(self) -> int:
        if self.mode == "persistent":
            return 2 * len(self.classes) + 1
        if self.mode == "plain" and self.plain_subset is not None:
            return sum((2 * c.n_slices + 1) * min(self.plain_subset, c.n_probes) for c in self.classes)
        return launches_per_step(self.classes, "plain" if self.mode == "plain" else "batched")
