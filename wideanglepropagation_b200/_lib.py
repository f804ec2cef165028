"""ctypes binding of libwap.so (the C ABI declared in include/wap.h).

The shared library is built in-tree (``python -m wideanglepropagation_b200.build``
or ``__graft_entry__.build()``).  There is no fallback: if the library is
missing or cannot be loaded, every compute entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libwap.so")

WAP_OK = 0
WAP_ERR_ARG = -1
WAP_ERR_UNSUPPORTED = -2
WAP_ERR_CUDA = -3
WAP_ERR_TIMEOUT = -4

WAP_OP_FRESNEL_AS = 0
WAP_OP_WPM = 1
WAP_TF_FRESNEL = 0
WAP_TF_ANGULAR = 1

(WAP_KNOB_ELEMS, WAP_KNOB_TWIDDLES, WAP_KNOB_TW_SMEM, WAP_KNOB_PSI, WAP_KNOB_GROUP, WAP_KNOB_CHAIN,
 WAP_KNOB_SUSPEND, WAP_KNOB_H_HI, WAP_KNOB_CLUSTER) = range(9)
WAP_TW_FULL = 1
WAP_TW_HI = 2

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double

# name -> (restype, argtypes); mirrors include/wap.h
SIGNATURES = {
    "wap_version": (ctypes.c_char_p, []),
    "wap_last_error": (ctypes.c_char_p, []),
    "wap_plan_create": (_I, [ctypes.POINTER(_P), _I, _I, _I, _I, _I]),
    "wap_plan_destroy": (_I, [_P]),
    "wap_plan_set_config": (_I, [_P, _I, _I, _I]),
    "wap_plan_set_detector": (_I, [_P, _I, _I, _I, _I]),
    "wap_gaussian_potential": (_I, [_I, _I, _I, _D, _D, _P, _P, _D, _D, _P, _P]),
    "wap_aperture_probe": (_I, [_P, _D, _D, _D, _D, _D, _I, _P, _P]),
    "wap_pattern_accumulate": (_I, [_P, _I, ctypes.c_longlong, _P, _P, _I, _P, _P, _P]),
    "wap_spectrum_propagate": (_I, [_P, _P, _I, _P, _P, _P, _P]),
    "wap_scan_grad_backward_ex": (_I, [_P, _P, _P, _P, _P]),
    "wap_fp32_probe": (_I, [_I, _I, _P, _P]),
    "wap_line_transfer": (_I, [_I, _I, _P, _D, _D, _P, _P]),
    "wap_line_propagate": (_I, [_I, _I, _P, _P, _P, _I, _P, _P]),
    "wap_line_wpm": (_I, [_I, _I, _P, _P, _D, _P, _D, _P, _P]),
    "wap_wpm_naive_step": (_I, [_I, _I, _P, _P, _D, _D, _D, _D, _P, _P, _P]),
    "wap_plan_get_config": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "wap_transfer_function": (_I, [_I, _I, _I, _D, _D, _D, _D, _P, _I, _P, _P]),
    "wap_multislice_fwd": (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _P, _P, _P, _D, _D, _P, _P, _P, _P]),
    "wap_wpm_fwd": (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _P, _D, _D, _D, _D, _D, _P, _P, _P, _P]),
    "wap_multislice_fwd_ckpt": (_I, [_P, _P, _I, _I, _P, _P, _I, _I, _P, _P, _P, _D, _D, _P, _P, _P, _I, _P]),
    "wap_multislice_bwd": (_I, [_P, _P, _I, _I, _P, _I, _P, _P, _D, _D, _P, _P, _I, _P, _P, _P, _P, _P]),
    "wap_multislice_fwd_noalloc": (_I, [_P, _I, _I, _I, _P, _I, _I, _P, _P, _P, _D, _D, _P, _P, _P, _P]),
    "wap_scan_create": (_I, [ctypes.POINTER(_P), _I, _P]),
    "wap_scan_run": (_I, [_P, _P]),
    "wap_scan_grad_create": (_I, [ctypes.POINTER(_P), _P, _I]),
    "wap_scan_grad_backward": (_I, [_P, _P, _P, _P]),
    "wap_scan_bind": (_I, [_P, _I, _P]),
    "wap_scan_status": (_I, [_P, ctypes.POINTER(_I)]),
    "wap_scan_status_async": (_I, [_P, _P, _P]),
    "wap_plan_status_async": (_I, [_P, _P, _P]),
    "wap_plan_status_pending": (_I, [_P, ctypes.POINTER(_I)]),
    "wap_scan_debug_override": (_I, [_I, _I]),
    "wap_scan_info": (_I, [_P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "wap_scan_destroy": (_I, [_P]),
    "wap_scan_debug_stall": (_I, [_P, _I, ctypes.c_longlong]),
    "wap_scan_debug_checks": (_I, [_P, _I, _P]),
    "wap_launch_count": (ctypes.c_longlong, []),
    "wap_profile_enable": (_I, [_I]),
    "wap_profile_reset": (_I, []),
    "wap_profile_read": (_I, [_I, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_D), ctypes.POINTER(_D)]),
}

KIND_ROW, KIND_COL, KIND_WPM_COL, KIND_WPM_ROW, KIND_WPM_BINS, KIND_SCHED, KIND_TRANS = range(7)
KIND_NAMES = {KIND_ROW: "row_pass_kernel", KIND_COL: "col_pass_kernel", KIND_WPM_COL: "wpm_col_kernel",
              KIND_WPM_ROW: "wpm_row_kernel", KIND_WPM_BINS: "wpm_bins_kernel", KIND_SCHED: "scan_persistent_kernel",
              KIND_TRANS: "trans_table_kernel"}

class ScanClass(ctypes.Structure):
    """Mirror of ``wap_scan_class`` (include/wap.h)."""
    _fields_ = [("n", _I), ("n_slices", _I), ("n_draws", _I), ("n_probes", _I),
                ("V", _P), ("draw", _P), ("psi0", _P), ("positions", _P), ("H", _P), ("H_lo", _P),
                ("dz", _D), ("energy", _D), ("exit", _P), ("dp", _P), ("group", _I),
                ("det_y0", _I), ("det_x0", _I), ("det_ny", _I), ("det_nx", _I)]


_lib = None
_lock = threading.Lock()


class WapError(RuntimeError):
    """A CUDA-side failure reported by libwap.so."""


def lib():
    """Load libwap.so once; raise if it is absent (no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"libwap.so not found at {LIB_PATH}; build it with "
                    "`python -m wideanglepropagation_b200.build` (the multislice path "
                    "has no CPU fallback)")
            h = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(h, name)
                fn.restype = res
                fn.argtypes = args
            _lib = h
    return _lib


def check(rc: int) -> None:
    """Translate a WAP_* status into the reference's Python exception types."""
    if rc == WAP_OK:
        return
    msg = lib().wap_last_error().decode(errors="replace")
    if rc in (WAP_ERR_ARG, WAP_ERR_UNSUPPORTED):
        raise ValueError(msg)
    raise WapError(f"libwap error {rc}: {msg}")


# Device-side status of persistent-scheduler runs whose check was deferred
# (check=False): (event after the status copy, pinned host word, what ran).
_pending: list = []
_pending_lock = threading.Lock()


# Reusable (event, pinned status word, numpy view of it) triples per device:
# a token takes one and gives it back once its status has been read, so a call
# pays neither a pinned allocation nor an event creation.
_token_pool: dict = {}


def _token_parts(device_index: int):
    with _pending_lock:
        pool = _token_pool.get(device_index)
        if pool:
            return pool.pop()
    import torch
    word = torch.zeros(1, dtype=torch.int32, pin_memory=True)
    return torch.cuda.Event(), word, word.numpy()


def scan_status_begin(handle, what: str, source: str = "wap_scan_status_async", stream=None):
    """Enqueue, on ``stream`` (default: the current one), a copy of a scan's
    (or, with source="wap_plan_status_async", a plan's one-launch chain's)
    status word into pinned host memory and record an event after it; returns
    the token that ``scan_status_end`` or ``defer_status`` take."""
    import torch
    if stream is None:
        stream = torch.cuda.current_stream()
    di = stream.device.index
    ev, word, view = _token_parts(di)
    view[0] = 0
    check(getattr(lib(), source)(handle, ctypes.c_void_p(word.data_ptr()), ctypes.c_void_p(stream.cuda_stream)))
    ev.record(stream)
    return ev, word, what, view, di


def _raise_status(token) -> None:
    ev, word, what, view, di = token
    ev.synchronize()
    st = int(view[0])
    with _pending_lock:
        _token_pool.setdefault(di, []).append((ev, word, view))
    if st != WAP_OK:
        kind = "a bounded device-side wait expired" if st == WAP_ERR_TIMEOUT else "the kernel reported an error"
        raise WapError(f"libwap error {st}: {what}: {kind}; its outputs are incomplete")


def plan_status_pending(handle) -> bool:
    """Whether the last forward on the plan ran the one-launch chain (the only
    single-probe path with device-side waits, so the only one with a status)."""
    v = ctypes.c_int(0)
    check(lib().wap_plan_status_pending(handle, ctypes.byref(v)))
    return bool(v.value)


def scan_status_end(token) -> None:
    """Wait for the status copy of ``token`` and raise WapError if the run failed."""
    _raise_status(token)


def defer_status(token) -> None:
    """Keep ``token`` for ``check_errors`` (and the next checked call)."""
    with _pending_lock:
        _pending.append(token)


def check_errors() -> None:
    """Wait for every deferred scheduler status and raise WapError for the
    first run that failed (all deferred statuses are consumed)."""
    with _pending_lock:
        tokens = list(_pending)
        _pending.clear()
    first = None
    for t in tokens:
        try:
            _raise_status(t)
        except WapError as e:
            first = first or e
    if first is not None:
        raise first


def poll_errors() -> None:
    """Raise WapError for a deferred run that has already finished and failed;
    never blocks (runs still in flight stay pending)."""
    with _pending_lock:
        done = [t for t in _pending if t[0].query()]
        for t in done:
            _pending.remove(t)
    for t in done:
        _raise_status(t)


def version() -> str:
    return lib().wap_version().decode()


def profile_enable(on: bool) -> None:
    check(lib().wap_profile_enable(1 if on else 0))


def profile_reset() -> None:
    check(lib().wap_profile_reset())


def profile_read(kind: int):
    """(launches, device ms, algorithmic bytes) recorded for one pass kind."""
    n, ms, by = ctypes.c_longlong(), ctypes.c_double(), ctypes.c_double()
    check(lib().wap_profile_read(kind, ctypes.byref(n), ctypes.byref(ms), ctypes.byref(by)))
    return n.value, ms.value, by.value


def launch_count() -> int:
    """Kernels launched by libwap.so in this process so far."""
    return int(lib().wap_launch_count())
