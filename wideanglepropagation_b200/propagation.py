"""Drop-in replacements for the reference multislice API.

Same names, argument meaning and return structure as
``wide_angle_propagation/propagation.py``; arrays may be NumPy arrays or torch
tensors (any device) and results are torch tensors on the current CUDA
device.  The wave is carried in complex64 and every slice step runs in the
hand-written sm_100a kernels of libwap.so; there is no CPU path.

Extensions over the reference signatures (keyword-only, defaults keep the
reference behaviour):

* ``return_wavefronts`` - the reference always returns the stacked
  wavefronts (propagation.py:352); ``False`` returns ``None`` instead and skips
  those writes.
* ``positions`` - (B, 2) probe centres; the initial wave of probe b is
  ``move_probe(probe, positions[b])`` (propagation.py:263-276), so a whole
  scan is one call.
* a (B, ny, nx) probe runs B independent probes; a (D, N, ny, nx) potential
  holds D frozen-phonon draws selected per probe by ``draw``.
* ``max_angle`` (mrad) with ``sampling`` and ``parity`` - the diffraction
  pattern comes back already cropped to the detector window that
  ``downsample_to_max_angle`` (propagation.py:424-439) would keep; the crop is
  fused into the last column pass, which stores only that window.
"""
from __future__ import annotations

import ctypes
import math
import threading
from typing import Optional

import numpy as np
import torch

from . import _lib
from .physics import (electron_rest_energy, energy2mass, energy2sigma,  # noqa: F401
                      energy2wavelength, refractive_index_coefficients,
                      relativistic_mass_correction)

__all__ = [
    "electron_rest_energy", "relativistic_mass_correction", "energy2mass",
    "energy2wavelength", "energy2sigma", "electron_refractive_index",
    "electron_refractive_index_taylor", "get_frequencies", "smoothstep",
    "get_polynomial_bins", "shift_kernel", "fresnel_propagation_kernel",
    "angular_spectrum_propagation_kernel", "Propagator", "wpm_step_adaptive",
    "move_probe", "transmission_function", "simulate_fresnel_as",
    "simulate_fresnel_as_jit", "simulate_fresnel", "simulate_wpm",
    "simulate_wpm_jit", "max_angle_gpts", "downsample_to_max_angle", "detector_window",
    "wpm_propagation_kernel", "wpm_propagation_kernel_vmap", "get_abtem_transmit", "release_caches",
    "check_errors", "accumulate_patterns", "aperture_probe",
]


# ---------------------------------------------------------------------------
# device / tensor plumbing
# ---------------------------------------------------------------------------
def _device() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("wideanglepropagation_b200 runs on a CUDA device (sm_100a); "
                           "no CUDA device is visible and there is no CPU path")
    return torch.device("cuda", torch.cuda.current_device())


_copy_streams: dict = {}


def _copy_stream(device) -> torch.cuda.Stream:
    key = torch.device(device).index
    s = _copy_streams.get(key)
    if s is None:
        s = _copy_streams[key] = torch.cuda.Stream(device=device)
    return s


def _to(x, dtype, device) -> torch.Tensor:
    if not isinstance(x, torch.Tensor):
        x = torch.as_tensor(np.asarray(x))
    if x.is_complex() and not dtype.is_complex:
        raise ValueError("expected a real array, got a complex one")
    if (x.device.type == "cpu" and x.dtype == dtype and x.is_contiguous() and x.numel() > 0
            and torch.device(device).type == "cuda" and x.is_pinned()):
        # Pinned host input: copy on a side stream so the upload overlaps the
        # kernels already queued on the caller's stream; the caller's stream
        # waits for the copy before it uses the data.  (As with any
        # non-blocking copy, the host buffer must not change until then.)
        cur = torch.cuda.current_stream(device)
        cs = _copy_stream(device)
        with torch.cuda.stream(cs):
            y = torch.empty(x.shape, dtype=dtype, device=device)
            y.copy_(x, non_blocking=True)
        cur.wait_stream(cs)
        y.record_stream(cur)
        return y
    return x.to(device=device, dtype=dtype).contiguous()


# Recent splits of complex128 device tensors: (source tensor, its version,
# device, hi, lo, event recorded after the split on the stream that made it,
# that stream's handle).
# An entry keeps its source alive, so no other tensor can take its memory
# while cached, and an in-place change of the source bumps its version and
# misses.  Inference tensors carry no version counter and are never cached.
_SPLIT_CACHE_MAX = 4
_split_cache: list = []
_split_lock = threading.Lock()


def _version_of(t: torch.Tensor):
    """The tensor's version counter, or None where it has none (inference tensors)."""
    if t.is_inference():
        return None
    try:
        return t._version
    except RuntimeError:
        return None


def split_transfer(H, device, cache: bool = True):
    """complex64 hi part and remainder of a transfer function.

    A complex128 H is split into H_hi = (complex64)H and H_lo = H - H_hi; the
    kernels apply X*H_hi + X*H_lo, which removes the rounding of H that would
    otherwise repeat identically at every slice.  A complex64 H has no lo part.
    A complex128 tensor already on the device is split once and reused while
    it is unchanged (a transfer function normally serves many calls); a caller
    on another stream than the one that made the split waits for it first.
    ``cache=False`` (internal scratch that the kernels rewrite) always splits,
    and so does a call inside a CUDA graph capture (the split becomes part of
    the graph: the cache's events cannot cross the capture boundary).
    """
    t = H if isinstance(H, torch.Tensor) else torch.as_tensor(np.asarray(H))
    if t.dtype == torch.complex128:
        dev = torch.device(device)
        ver = _version_of(t) if cache else None
        cacheable = (ver is not None and t.device.type == "cuda" and t.device == dev
                     and not torch.cuda.is_current_stream_capturing())
        if cacheable:
            with _split_lock:
                for i, (src, sver, d, hi, lo, ev, sid) in enumerate(_split_cache):
                    if src is t and sver == ver and d == dev:
                        _split_cache.append(_split_cache.pop(i))
                        cur = torch.cuda.current_stream(dev)
                        if cur.cuda_stream != sid:
                            # made on another stream: wait for it, and keep the
                            # halves' memory until this stream is done with it
                            cur.wait_event(ev)
                            hi.record_stream(cur)
                            lo.record_stream(cur)
                        return hi, lo
        t = t.to(device)
        hi = t.to(torch.complex64).contiguous()
        lo = (t - hi.to(torch.complex128)).to(torch.complex64).contiguous()
        if cacheable:
            cur = torch.cuda.current_stream(dev)
            ev = torch.cuda.Event()
            ev.record(cur)
            with _split_lock:
                _split_cache.append((H, ver, dev, hi, lo, ev, cur.cuda_stream))
                del _split_cache[:-_SPLIT_CACHE_MAX]
        return hi, lo
    return _to(t, torch.complex64, device), None


def _ptr(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _pair(ps) -> tuple:
    if isinstance(ps, (int, float)):
        return float(ps), float(ps)
    ps = tuple(float(v) for v in ps)
    if len(ps) != 2:
        raise ValueError("sampling must be a scalar or a pair")
    return ps


class StreamOrder:
    """Stream order of one cached native object (a plan or a scan: device
    workspace that every call reuses).  It remembers the stream of the last
    use; a use from another stream first waits for everything issued on that
    stream so far (an event recorded there at the switch), so that calls on
    different CUDA streams never run on the same workspace at once.  Uses on
    one stream are ordered by the stream itself and cost nothing here.  A use
    inside a CUDA graph capture does not wait (a dependency on work outside
    the capture is not allowed there): a captured graph is ordered by the
    stream it is replayed on, like any graph.  If the last stream can no
    longer take an event (a caller's external stream, destroyed since), the
    switch waits for the whole device instead."""

    __slots__ = ("last",)

    def __init__(self):
        self.last = None

    def begin(self, cur):
        last = self.last
        if last is not None and last.cuda_stream != cur.cuda_stream \
                and not torch.cuda.is_current_stream_capturing():
            try:
                ev = torch.cuda.Event()
                ev.record(last)
                cur.wait_event(ev)
            except RuntimeError:
                torch.cuda.synchronize(cur.device)
        return cur

    def end(self, cur) -> None:
        self.last = cur


class Plan:
    """Owns one ``wap_plan`` (twiddle tables, WPM workspace) on one device;
    ``order`` keeps its uses from different streams apart."""

    def __init__(self, ny: int, nx: int, max_batch: int, op: int, n_bins: int = 0):
        L = _lib.lib()
        h = ctypes.c_void_p()
        _lib.check(L.wap_plan_create(ctypes.byref(h), ny, nx, max_batch, op, n_bins))
        self.handle = h
        self.ny, self.nx, self.max_batch, self.op, self.n_bins = ny, nx, max_batch, op, n_bins
        self.device = torch.cuda.current_device()
        self.det = None
        self.order = StreamOrder()

    def begin(self):
        """The current stream, after the plan's last use on another stream."""
        return self.order.begin(torch.cuda.current_stream(self.device))

    def end(self, cur) -> None:
        self.order.end(cur)

    def set_config(self, row_e: int, col_e: int, col_w: int) -> None:
        _lib.check(_lib.lib().wap_plan_set_config(self.handle, row_e, col_e, col_w))

    def set_detector(self, det) -> None:
        """Diffraction-pattern window (y0, x0, ny, nx) of later calls; None: whole grid."""
        if det != self.det:
            y0, x0, dny, dnx = det if det is not None else (0, 0, 0, 0)
            _lib.check(_lib.lib().wap_plan_set_detector(self.handle, y0, x0, dny, dnx))
            self.det = det

    def config(self) -> tuple:
        a, b, c = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        _lib.check(_lib.lib().wap_plan_get_config(self.handle, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c)))
        return a.value, b.value, c.value

    def close(self) -> None:
        if getattr(self, "handle", None) is not None and self.handle.value:
            try:
                torch.cuda.synchronize(self.device)
            except Exception:
                pass
            _lib.lib().wap_plan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_plans: dict = {}
_plans_lock = threading.Lock()


def get_plan(ny: int, nx: int, batch: int, op: int, n_bins: int = 0) -> Plan:
    """Cached plan for (device, grid, op, bins, batch class) holding at least
    ``batch`` probes; one- and two-probe calls get their own plan with the
    launch shapes tuned for them."""
    from . import autotune
    dev = torch.cuda.current_device()
    cls = autotune.batch_class(batch)
    key = (dev, ny, nx, op, n_bins, cls)
    with _plans_lock:
        p = _plans.get(key)
        if p is None or p.max_batch < batch:
            if p is not None:
                p.close()
            cap = batch if (op == _lib.WAP_OP_WPM or cls == "single") else max(batch, 64)
            p = Plan(ny, nx, cap, op, n_bins)
            cfg = autotune.lookup(ny, nx, op, n_bins, cls)
            if cfg is not None:
                p.set_config(*cfg)
            _plans[key] = p
        p.set_detector(None)   # cached plans are shared: whole-grid patterns unless a caller sets a window
        return p


# ---------------------------------------------------------------------------
# physics helpers (propagation.py:66-127)
# ---------------------------------------------------------------------------
def electron_refractive_index(potential, energy):
    """n(V) = sqrt((2(E+V)E0 + (E+V)^2) / (2EE0 + E^2)) (propagation.py:66-81),
    float64 on the device."""
    dev = _device()
    V = _to(potential, torch.float64, dev)
    E0 = electron_rest_energy()
    EmV = energy + V
    return torch.sqrt((2 * EmV * E0 + EmV ** 2) / (2 * energy * E0 + energy ** 2))


def electron_refractive_index_taylor(potential, energy):
    """1 + (E + E0)/(E (E + 2E0)) V (propagation.py:84-95)."""
    dev = _device()
    V = _to(potential, torch.float64, dev)
    E0 = electron_rest_energy()
    return 1.0 + (energy + E0) / (energy * (energy + 2 * E0)) * V


def _fftfreq(n: int, d: float, device) -> torch.Tensor:
    return torch.fft.fftfreq(n, d=d, dtype=torch.float64, device=device)


def get_frequencies(n, m, ps):
    """fftfreq grids with meshgrid indexing='ij' (propagation.py:102-107)."""
    dev = _device()
    p0, p1 = _pair(ps)
    return torch.meshgrid(_fftfreq(n, p0, dev), _fftfreq(m, p1, dev), indexing="ij")


def smoothstep(x):
    """3x^2 - 2x^3 on clip(x, 0, 1) (propagation.py:110-116)."""
    x = torch.clamp(torch.as_tensor(x), 0.0, 1.0)
    return 3 * x ** 2 - 2 * x ** 3


def get_polynomial_bins(n_min, n_max, n_bins, power=2.0):
    """n_min + (n_max - n_min) linspace(0, 1, K)^power (propagation.py:119-127)."""
    t = torch.from_numpy(np.linspace(0, 1, n_bins))
    n_min = torch.as_tensor(n_min, dtype=torch.float64)
    n_max = torch.as_tensor(n_max, dtype=torch.float64)
    t = t.to(n_min.device)
    return n_min + (n_max - n_min) * t ** power


def shift_kernel(x0, y0, Fx, Fy):
    """exp(-2 pi i (Fx x0 + Fy y0)) (propagation.py:134-136)."""
    return torch.exp(-1j * 2 * math.pi * (Fx * x0 + Fy * y0))


# ---------------------------------------------------------------------------
# transfer functions (propagation.py:139-156), float64 on the device
# ---------------------------------------------------------------------------
def _transfer(kind: int, n: int, m: int, ps, z: float, energy: float,
              dtype=torch.complex128, with_lo: bool = False):
    dev = _device()
    p0, p1 = _pair(ps)
    out = torch.empty((int(n), int(m)), dtype=dtype, device=dev)
    lo = torch.empty((int(n), int(m)), dtype=torch.complex64, device=dev) if with_lo else None
    if with_lo and dtype != torch.complex64:
        raise ValueError("with_lo needs dtype=torch.complex64")
    _lib.check(_lib.lib().wap_transfer_function(kind, int(n), int(m), p0, p1, float(z), float(energy),
                                                _ptr(out), 1 if dtype == torch.complex128 else 0, _ptr(lo),
                                                _stream()))
    return (out, lo) if with_lo else out


def transfer_pair(method: str, n: int, m: int, ps, z: float, energy: float):
    """(H_hi, H_lo) complex64 pair of the Fresnel ('fresnel') or angular-spectrum
    ('as') transfer function, evaluated in float64 on the device."""
    kind = _lib.WAP_TF_ANGULAR if method == "as" else _lib.WAP_TF_FRESNEL
    return _transfer(kind, n, m, ps, z, energy, torch.complex64, with_lo=True)


def fresnel_propagation_kernel(n: int, m: int, ps, z: float, energy: float, *, dtype=torch.complex128):
    """H = exp(i 2 pi z/lam) exp(-i pi lam z (Fx^2 + Fy^2)) (propagation.py:139-145)."""
    return _transfer(_lib.WAP_TF_FRESNEL, n, m, ps, z, energy, dtype)


def angular_spectrum_propagation_kernel(n: int, m: int, ps, z: float, energy: float, *, dtype=torch.complex128):
    """H = exp(i 2 pi z sqrt(1/lam^2 - Fx^2 - Fy^2)), complex sqrt (propagation.py:148-156)."""
    return _transfer(_lib.WAP_TF_ANGULAR, n, m, ps, z, energy, dtype)


# ---------------------------------------------------------------------------
# probe tools (propagation.py:263-283)
# ---------------------------------------------------------------------------
def move_probe(probe, new_pos):
    """Roll the probe so its centre (ny//2, nx//2) moves to new_pos (propagation.py:263-276)."""
    p = probe if isinstance(probe, torch.Tensor) else torch.as_tensor(np.asarray(probe))
    sr = int(new_pos[0]) - p.shape[-2] // 2
    sc = int(new_pos[1]) - p.shape[-1] // 2
    return torch.roll(p, shifts=(sr, sc), dims=(-2, -1))


def transmission_function(potential, energy):
    """exp(i sigma V) (propagation.py:279-283); not used by the simulators."""
    dev = _device()
    V = _to(potential, torch.float64, dev)
    return torch.exp(1j * energy2sigma(energy) * V)


# ---------------------------------------------------------------------------
# simulators (propagation.py:305-391)
# ---------------------------------------------------------------------------
def _prepare(potential, probe, positions, draw, dev):
    V = _to(potential, torch.float32, dev)
    if V.ndim == 3:
        V = V.unsqueeze(0)
    if V.ndim != 4:
        raise ValueError(f"potential must be (N, ny, nx) or (draws, N, ny, nx), got {tuple(V.shape)}")
    n_draws, n_slices, ny, nx = V.shape
    psi = _to(probe, torch.complex64, dev)
    if psi.shape[-2:] != (ny, nx):
        raise ValueError(f"probe grid {tuple(psi.shape[-2:])} does not match potential grid {(ny, nx)}")
    per_probe = psi.ndim == 3
    if psi.ndim not in (2, 3):
        raise ValueError("probe must be (ny, nx) or (B, ny, nx)")
    pos = None
    if positions is not None:
        pos = _to(positions, torch.int32, dev).reshape(-1, 2)
    B = psi.shape[0] if per_probe else (pos.shape[0] if pos is not None else 1)
    if pos is not None and pos.shape[0] != B:
        raise ValueError("positions and batched probe disagree on the batch size")
    dr = None
    if draw is not None:
        # host arrays are range-checked before the upload (no device sync);
        # a device tensor is checked on the device
        on_host = not isinstance(draw, torch.Tensor) or draw.device.type == "cpu"
        if on_host:
            d = draw.reshape(-1) if isinstance(draw, torch.Tensor) else np.asarray(draw).reshape(-1)
            if d.shape[0] == B and d.shape[0] > 0 and (int(d.min()) < 0 or int(d.max()) >= n_draws):
                raise ValueError("draw index out of range")
        dr = _to(draw, torch.int32, dev).reshape(-1)
        if dr.shape[0] != B:
            raise ValueError("draw must have one entry per probe")
        if not on_host and (int(dr.min()) < 0 or int(dr.max()) >= n_draws):
            raise ValueError("draw index out of range")
    elif n_draws > 1:
        raise ValueError("a potential with several draws needs `draw`")
    batched = per_probe or pos is not None
    return V, psi, per_probe, pos, dr, B, n_slices, ny, nx, batched


SCAN_SIZES = (128, 256, 512, 1024)
SCAN_MIN_PROBES = 8
# forwards of at most this many probes on these square grids run as one launch (a
# cooperative grid, or a thread-block cluster per probe at 128)
CHAIN_SIZES = (128, 256)
CHAIN_MAX_PROBES = 2
_scans: dict = {}          # key -> (scan handle, StreamOrder)
_scans_lock = threading.Lock()


def detector_window(shape, sampling, energy, max_angle, parity="odd"):
    """(y0, x0, ny, nx) of the centre crop ``downsample_to_max_angle`` keeps of
    an fftshifted pattern (propagation.py:424-439), or None for the whole grid."""
    ny, nx = shape
    dny, dnx = max_angle_gpts((ny, nx), sampling, energy2wavelength(float(energy)), max_angle, parity=parity)
    if (dny, dnx) == (ny, nx):
        return None
    return ny // 2 - dny // 2, nx // 2 - dnx // 2, dny, dnx


def _detector(shape, sampling, energy, max_angle, parity):
    if max_angle is None:
        return None
    if sampling is None:
        raise ValueError("max_angle needs the grid sampling")
    return detector_window(shape, _pair(sampling), energy, max_angle, parity)


def _upload_small(a: np.ndarray, dev) -> torch.Tensor:
    """A small host array on the device through pinned memory and a
    non-blocking copy: a pageable copy may wait for the work already queued on
    the stream (e.g. a whole scan) before it returns."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    return _to(t.pin_memory(), t.dtype, dev)


def _dp_shape(B, ny, nx, det):
    return (B, det[2], det[3]) if det is not None else (B, ny, nx)


def _accumulation(accumulate, B, dev):
    """Host-validated CSR of ``accumulate`` ((B,) pattern index per probe):
    (n_patterns, start (P+1,) int32, probes (B,) int32) on the device, the
    probes of each pattern in increasing order."""
    idx = accumulate.cpu().numpy() if isinstance(accumulate, torch.Tensor) else np.asarray(accumulate)
    idx = idx.reshape(-1)
    if idx.shape[0] != B:
        raise ValueError(f"accumulate needs one pattern index per probe ({B}), got {idx.shape[0]}")
    if not np.issubdtype(idx.dtype, np.integer):
        raise ValueError("accumulate must hold integer pattern indices")
    if idx.size and idx.min() < 0:
        raise ValueError("accumulate indices must be >= 0")
    P = int(idx.max()) + 1 if idx.size else 0
    order = np.argsort(idx, kind="stable").astype(np.int32)
    start = np.concatenate([[0], np.cumsum(np.bincount(idx, minlength=P))]).astype(np.int32)
    return P, _upload_small(start, dev), _upload_small(order, dev)


def accumulate_patterns(dp: torch.Tensor, accumulate) -> torch.Tensor:
    """Sum per-probe diffraction patterns ``dp`` (B, ...) into
    (max(accumulate) + 1, ...) patterns: pattern p is the float32 sum of the
    patterns of the probes b with ``accumulate[b] == p``, added in increasing b
    (deterministic).  The incoherent frozen-phonon average per scan position
    that the reference's callers form by summing simulate_fresnel_as patterns
    over configurations, as one device kernel (``wap_pattern_accumulate``)."""
    dev = dp.device
    B = dp.shape[0]
    P, start, order = _accumulation(accumulate, B, dev)
    plane = int(np.prod(dp.shape[1:]))
    dpc = dp.contiguous()
    out = torch.empty((P,) + tuple(dp.shape[1:]), dtype=torch.float32, device=dev)
    if P == 0:
        return out
    _lib.check(_lib.lib().wap_pattern_accumulate(_ptr(dpc), B, plane, _ptr(start), _ptr(order), P, _ptr(out), None,
                                                 _stream()))
    return out


def scan_class(V, psi, pos, dr, H, H_lo, dz, energy, exit_wave, dp, det=None, group=None):
    """``wap_scan_class`` for one grid class of device tensors; the probe-group
    size defaults to the autotuned one for the grid (0: the scheduler's own)."""
    D, N, n, _ = V.shape
    if group is None:
        from . import autotune
        group = autotune.balanced_group(autotune.lookup_scan(n), exit_wave.shape[0])
    y0, x0, dny, dnx = det if det is not None else (0, 0, 0, 0)
    return _lib.ScanClass(n, N, D, exit_wave.shape[0], V.data_ptr(), dr.data_ptr() if dr is not None else None,
                          psi.data_ptr(), pos.data_ptr() if pos is not None else None, H.data_ptr(),
                          H_lo.data_ptr() if H_lo is not None else None, float(dz), float(energy),
                          exit_wave.data_ptr(), dp.data_ptr() if dp is not None else None, int(group),
                          y0, x0, dny, dnx)


def _scan_run(V, psi, pos, dr, H, H_lo, dz, energy, exit_wave, dp, det=None, check=True):
    """Run a batched forward through the persistent scheduler (cached per shape).

    The scheduler's bounded waits report an expiry in a device status word
    instead of faulting.  ``check=True`` waits for the run and raises WapError
    if a wait expired; ``check=False`` returns at once and leaves the status
    to ``check_errors()`` (or to the next call, which raises for any finished
    deferred run that failed)."""
    D, N, n, _ = V.shape
    B = exit_wave.shape[0]
    dev = torch.cuda.current_device()
    key = (dev, n, N, D, B)
    cls = (_lib.ScanClass * 1)()
    cls[0] = scan_class(V, psi, pos, dr, H, H_lo, dz, energy, exit_wave, dp, det)
    L = _lib.lib()
    arr = ctypes.cast(cls, ctypes.c_void_p)
    with _scans_lock:
        ent = _scans.get(key)
        if ent is None:
            h = ctypes.c_void_p()
            _lib.check(L.wap_scan_create(ctypes.byref(h), 1, arr))
            ent = _scans[key] = (h, StreamOrder())
        else:
            _lib.check(L.wap_scan_bind(ent[0], 1, arr))
        h, order = ent
        cur = order.begin(torch.cuda.current_stream(dev))
        _lib.check(L.wap_scan_run(h, ctypes.c_void_p(cur.cuda_stream)))
        token = _lib.scan_status_begin(h, f"persistent scan of {B} probes on {n}x{n}, {N} slices", stream=cur)
        order.end(cur)
    if check:
        _lib.scan_status_end(token)
    else:
        _lib.defer_status(token)


def check_errors() -> None:
    """Raise WapError for a scheduler run issued with ``check=False`` whose
    bounded waits expired (waits for those runs; clears them)."""
    _lib.check_errors()


def release_caches() -> None:
    """Free the device memory the library keeps between calls: cached plans
    (twiddles, WPM workspaces), cached forward scans (transmission tables,
    interleaved propagators), idle pooled gradient scans and cached splits of
    complex128 transfer functions."""
    torch.cuda.synchronize()
    with _split_lock:
        _split_cache.clear()
    with _scans_lock:
        for h, _ in _scans.values():
            _lib.lib().wap_scan_destroy(h)
        _scans.clear()
    with _plans_lock:
        for p in _plans.values():
            p.close()
        _plans.clear()
    from . import autograd
    autograd.release_pool()


def simulate_fresnel_as(potential, probe, prop_kernel, slice_thickness, energy, *,
                        return_wavefronts: bool = True, positions=None, draw=None,
                        max_angle=None, sampling=None, parity="odd", check: bool = True, accumulate=None):
    """Fresnel / angular-spectrum multislice (propagation.py:305-352).

    Returns ``(exit_wave, diffraction_pattern, wavefronts)`` where
    ``diffraction_pattern = |fftshift(fft2(exit_wave))|^2`` and
    ``wavefronts`` stacks the wave after every slice (``None`` when
    ``return_wavefronts=False``).  With ``max_angle`` (mrad) and ``sampling``
    the pattern is ``downsample_to_max_angle(pattern, sampling,
    wavelength, max_angle, parity)``, stored cropped by the kernel.

    ``accumulate`` ((B,) ints): the returned patterns are summed per index
    (``accumulate_patterns``), e.g. the frozen-phonon draws of each scan
    position into one float32 pattern per position; exit waves stay per probe.

    Calls that run on the persistent scheduler (many probes of one probe) or
    as one cooperative launch (one or two probes on a square 256 grid; on a
    128 grid they run as one thread-block cluster per probe, without
    device-side waits) raise WapError if one of their bounded device-side
    waits expired; with
    ``check=False`` the call returns without waiting for the GPU and the
    failure is raised by ``check_errors()`` or by a later call.
    """
    dev = _device()
    _lib.poll_errors()
    V, psi, per_probe, pos, dr, B, N, ny, nx, batched = _prepare(potential, probe, positions, draw, dev)
    if N < 1:
        raise ValueError("need at least one array to stack")  # jnp.stack([]) in the reference
    H, H_lo = split_transfer(prop_kernel, dev)
    if H.shape != (ny, nx):
        raise ValueError(f"prop_kernel shape {tuple(H.shape)} does not match grid {(ny, nx)}")
    det = _detector((ny, nx), sampling, energy, max_angle, parity)
    exit_wave = torch.empty((B, ny, nx), dtype=torch.complex64, device=dev)
    dp = torch.empty(_dp_shape(B, ny, nx, det), dtype=torch.float32, device=dev)
    if (not return_wavefronts and ny == nx and ny in SCAN_SIZES and B >= SCAN_MIN_PROBES
            and not per_probe):
        # many probes of one shared probe: the persistent batched scheduler
        _scan_run(V, psi, pos, dr, H, H_lo, slice_thickness, energy, exit_wave, dp, det, check=check)
        if accumulate is not None:
            dp = accumulate_patterns(dp, accumulate)
        if not batched:
            exit_wave, dp = exit_wave[0], dp[0]
        return exit_wave, dp, None
    plan = get_plan(ny, nx, B, _lib.WAP_OP_FRESNEL_AS)
    plan.set_detector(det)
    stack = torch.empty((B, N, ny, nx), dtype=torch.complex64, device=dev) if return_wavefronts else None
    cur = plan.begin()
    _lib.check(_lib.lib().wap_multislice_fwd(
        plan.handle, _ptr(V), N, V.shape[0], _ptr(dr), _ptr(psi), B, 1 if per_probe else 0,
        _ptr(pos), _ptr(H), _ptr(H_lo), float(slice_thickness), float(energy), _ptr(exit_wave), _ptr(dp),
        _ptr(stack), ctypes.c_void_p(cur.cuda_stream)))
    if B <= CHAIN_MAX_PROBES and ny == nx and ny in CHAIN_SIZES and _lib.plan_status_pending(plan.handle):
        # one or two probes ran as one cooperative launch whose grid-wide waits are bounded
        token = _lib.scan_status_begin(plan.handle, f"one-launch chain of {B} probe(s) on {ny}x{nx}, {N} slices",
                                       source="wap_plan_status_async", stream=cur)
        plan.end(cur)
        if check:
            _lib.scan_status_end(token)
        else:
            _lib.defer_status(token)
    else:
        plan.end(cur)
    if accumulate is not None:
        dp = accumulate_patterns(dp, accumulate)
    if not batched:
        exit_wave, dp = exit_wave[0], dp[0]
        stack = stack[0] if stack is not None else None
    return exit_wave, dp, stack


simulate_fresnel_as_jit = simulate_fresnel_as
# README of the reference calls the Fresnel/AS simulator `simulate_fresnel`
simulate_fresnel = simulate_fresnel_as


def simulate_wpm(potential, probe, slice_thickness, energy, sampling, n_bins=128, power_spacing=2.0, *,
                 return_wavefronts: bool = True, positions=None, draw=None, max_angle=None, parity="odd",
                 accumulate=None):
    """WPM adaptive-binning multislice (propagation.py:358-387).

    Per slice: n_bins reference refractive indices spaced
    n_min + (n_max - n_min) t^power_spacing, one angular-spectrum propagate
    per reference, smoothstep blend of the two bracketing fields per pixel
    (propagation.py:215-256).  ``sampling`` = (dy, dx).  ``max_angle`` (mrad):
    the pattern comes back cropped as by ``downsample_to_max_angle``.
    ``accumulate``: patterns summed per index, as in ``simulate_fresnel_as``.
    """
    dev = _device()
    V, psi, per_probe, pos, dr, B, N, ny, nx, batched = _prepare(potential, probe, positions, draw, dev)
    if N < 1:
        raise ValueError("need at least one array to stack")
    n_bins = int(n_bins)
    if n_bins < 2:
        raise ValueError("n_bins must be >= 2")
    dy, dx = _pair(sampling)
    plan = get_plan(ny, nx, B, _lib.WAP_OP_WPM, n_bins)
    det = _detector((ny, nx), sampling, energy, max_angle, parity)
    plan.set_detector(det)
    exit_wave = torch.empty((B, ny, nx), dtype=torch.complex64, device=dev)
    dp = torch.empty(_dp_shape(B, ny, nx, det), dtype=torch.float32, device=dev)
    stack = torch.empty((B, N, ny, nx), dtype=torch.complex64, device=dev) if return_wavefronts else None
    cur = plan.begin()
    _lib.check(_lib.lib().wap_wpm_fwd(
        plan.handle, _ptr(V), N, V.shape[0], _ptr(dr), _ptr(psi), B, 1 if per_probe else 0,
        _ptr(pos), float(slice_thickness), float(energy), dy, dx, float(power_spacing),
        _ptr(exit_wave), _ptr(dp), _ptr(stack), ctypes.c_void_p(cur.cuda_stream)))
    plan.end(cur)
    if accumulate is not None:
        dp = accumulate_patterns(dp, accumulate)
    if not batched:
        exit_wave, dp = exit_wave[0], dp[0]
        stack = stack[0] if stack is not None else None
    return exit_wave, dp, stack


simulate_wpm_jit = simulate_wpm


def Propagator(u, H):
    """ifft2(H * fft2(u)) (propagation.py:178-181): one slice of zero potential,
    whose transmission is exactly 1."""
    dev = _device()
    u = _to(u, torch.complex64, dev)
    ny, nx = u.shape[-2:]
    V = torch.zeros((1, ny, nx), dtype=torch.float32, device=dev)
    out, _, _ = simulate_fresnel_as(V, u, H, 1.0, 100e3, return_wavefronts=False)
    return out


def wpm_propagation_kernel_vmap(Ek, n_vals, k0, k_perp2, dz) -> torch.Tensor:
    """ifft2(exp(i dz sqrt((n k0)^2 - k_perp^2)) Ek) for every n in ``n_vals``
    (propagation.py:159-171): (len(n_vals), ny, nx) complex64.  The propagator
    is evaluated in float64 and applied as complex64 hi + lo parts; the inverse
    transform runs in the pass kernels."""
    dev = _device()
    X = _to(Ek, torch.complex64, dev)
    if X.ndim != 2:
        raise ValueError("Ek must be one (ny, nx) spectrum")
    ny, nx = X.shape
    kp2 = _to(k_perp2, torch.float64, dev).reshape(-1)
    if kp2.numel() != ny * nx:
        raise ValueError("k_perp2 must have the shape of Ek")
    nv = np.atleast_1d(np.asarray(n_vals.cpu() if isinstance(n_vals, torch.Tensor) else n_vals, dtype=np.float64))
    plan = get_plan(ny, nx, 1, _lib.WAP_OP_FRESNEL_AS)
    out = torch.empty((nv.size, ny, nx), dtype=torch.complex64, device=dev)
    H = torch.empty(ny * nx, dtype=torch.complex128, device=dev)
    L = _lib.lib()
    cur = plan.begin()
    st = ctypes.c_void_p(cur.cuda_stream)
    try:
        for i, n in enumerate(nv):
            _lib.check(L.wap_line_transfer(_lib.WAP_TF_ANGULAR, ny * nx, _ptr(kp2), float(n) * float(k0),
                                           float(dz), _ptr(H), st))
            Hh, Hl = split_transfer(H.view(ny, nx), dev, cache=False)
            _lib.check(L.wap_spectrum_propagate(plan.handle, _ptr(X), 1, _ptr(Hh), _ptr(Hl), _ptr(out[i]), st))
    finally:
        plan.end(cur)
    return out


def wpm_propagation_kernel(Ek, n_val, k0, k_perp2, dz) -> torch.Tensor:
    """One homogeneous-index WPM propagate of a spectrum (propagation.py:159-167)."""
    return wpm_propagation_kernel_vmap(Ek, [float(n_val)], k0, k_perp2, dz)[0]


def aperture_probe(ny: int, nx: int, sampling, energy: float, alpha_mrad: float, defocus: float = 0.0,
                   centred: bool = True) -> torch.Tensor:
    """Convergent probe built on the device: (ny, nx) complex64.

    A hard aperture |f| lambda < alpha with the defocus phase
    exp(-i pi lambda df |f|^2) inside it (float64), inverse-transformed by the
    library's transforms, normalised to sum |psi|^2 = ny nx and, if
    ``centred``, rolled to the grid centre (the origin ``move_probe``
    measures positions from).  The reference's callers build probes on the
    host with abTEM (e.g. wpm/cbed.ipynb); this is the probe model of the
    benchmark configurations, without a host round trip."""
    dev = _device()
    ps_y, ps_x = _pair(sampling)
    plan = get_plan(int(ny), int(nx), 1, _lib.WAP_OP_FRESNEL_AS)
    out = torch.empty((int(ny), int(nx)), dtype=torch.complex64, device=dev)
    cur = plan.begin()
    _lib.check(_lib.lib().wap_aperture_probe(plan.handle, ps_y, ps_x, float(energy), float(alpha_mrad),
                                             float(defocus), 1 if centred else 0, _ptr(out),
                                             ctypes.c_void_p(cur.cuda_stream)))
    plan.end(cur)
    return out


def get_abtem_transmit(potential, energy):
    """propagation.py:286-299 builds transmission functions from abTEM
    potential objects; abTEM is not part of this package.  Build the potential
    with ``gaussian_potential`` (or pass a potential array to the simulators,
    which form the transmission on the device)."""
    raise NotImplementedError("get_abtem_transmit needs abTEM potentials; use gaussian_potential or pass a "
                              "potential array to simulate_fresnel_as / simulate_wpm")


def _potential_from_index(n_map: torch.Tensor, energy: float) -> torch.Tensor:
    """Invert n(V) of propagation.py:66-81: E+V = -E0 + sqrt(E0^2 + n^2 (2 E E0 + E^2))."""
    E0 = electron_rest_energy()
    n = n_map.to(torch.float64)
    return (-E0 + torch.sqrt(E0 * E0 + n * n * (2 * energy * E0 + energy * energy))) - energy


def wpm_step_adaptive(wave, n_map, dz, energy, ps, n_bins=256, power_spacing=2.0):
    """One adaptive-binning WPM step (propagation.py:215-256).

    Returns (new_wave, w, idx_L, n_refs) like the reference; ``new_wave`` comes
    from the WPM kernels, the auxiliary outputs are evaluated on the device
    from ``n_map`` with the reference's formulas.
    """
    dev = _device()
    n_map = _to(n_map, torch.float64, dev)
    V = _potential_from_index(n_map, float(energy)).to(torch.float32)[None]
    new_wave, _, _ = simulate_wpm(V, wave, dz, energy, ps, n_bins=n_bins, power_spacing=power_spacing,
                                  return_wavefronts=False)
    n_refs = get_polynomial_bins(n_map.min(), n_map.max(), n_bins, power_spacing)
    idx_R = torch.clamp(torch.searchsorted(n_refs, n_map.reshape(-1)).reshape(n_map.shape), 1, n_bins - 1)
    idx_L = idx_R - 1
    n_L, n_R = n_refs[idx_L], n_refs[idx_R]
    denom = n_R - n_L
    w = smoothstep((n_map - n_L) / torch.where(denom == 0, torch.ones_like(denom), denom))
    return new_wave, w, idx_L, n_refs


# ---------------------------------------------------------------------------
# detector crop (propagation.py:394-439)
# ---------------------------------------------------------------------------
def max_angle_gpts(shape, sampling, wavelength, max_angle_mrad, parity="odd"):
    """Cropped grid size matching max_angle_mrad (propagation.py:394-421)."""
    ny, nx = shape
    dx, dy = float(sampling[0]), float(sampling[1])
    max_freq = float(max_angle_mrad) / (float(wavelength) * 1000.0)
    half_x = int(math.floor(max_freq / (1.0 / (nx * dx))))
    half_y = int(math.floor(max_freq / (1.0 / (ny * dy))))
    half_x = max(0, min(half_x, nx // 2))
    half_y = max(0, min(half_y, ny // 2))
    if parity == "even":
        new_nx, new_ny = 2 * half_x, 2 * half_y
    else:
        new_nx, new_ny = 2 * half_x + 1, 2 * half_y + 1
    return max(1, min(new_ny, ny)), max(1, min(new_nx, nx))


def downsample_to_max_angle(pattern, sampling, wavelength, max_angle_mrad, parity="odd"):
    """Centre-crop an fftshifted pattern to max_angle_mrad (propagation.py:424-439);
    works on the last two axes of NumPy arrays or torch tensors."""
    ny, nx = pattern.shape[-2:]
    new_ny, new_nx = max_angle_gpts((ny, nx), sampling, wavelength, max_angle_mrad, parity=parity)
    if (new_ny, new_nx) == (ny, nx):
        return pattern
    y0 = ny // 2 - new_ny // 2
    x0 = nx // 2 - new_nx // 2
    return pattern[..., y0:y0 + new_ny, x0:x0 + new_nx]
