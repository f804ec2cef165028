"""Launch-shape autotuner for the multislice passes.

Candidates per grid: elements per thread of the row pass (``row_e``), of the
column pass (``col_e``) and columns per column-pass CTA (``col_w``).  Each is
timed on the device with CUDA events over a short synthetic multislice; the
winner is cached in ``autotune_cache.json`` keyed by GPU name, grid, op and
bin count, and applied to every plan created afterwards.
"""
from __future__ import annotations

import json
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
CACHE_PATH = os.environ.get("WAP_AUTOTUNE_CACHE", os.path.join(HERE, "autotune_cache.json"))
_lock = threading.Lock()
_cache = None


def _gpu_name() -> str:
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device()) if torch.cuda.is_available() else "none"


def _key(ny, nx, op, n_bins, batch_class="any") -> str:
    return f"{_gpu_name()}|{ny}x{nx}|op{op}|K{n_bins}|{batch_class}"


def _load() -> dict:
    global _cache
    if _cache is None:
        try:
            with open(CACHE_PATH) as f:
                _cache = json.load(f)
        except (OSError, ValueError):
            _cache = {}
    return _cache


def lookup(ny, nx, op, n_bins=0):
    """Cached (row_e, col_e, col_w) for this GPU and grid, or None."""
    with _lock:
        v = _load().get(_key(ny, nx, op, n_bins))
    return tuple(v) if v else None


def store(ny, nx, op, n_bins, cfg) -> None:
    with _lock:
        c = _load()
        c[_key(ny, nx, op, n_bins)] = list(cfg)
        tmp = CACHE_PATH + ".tmp"
        with open(tmp, "w") as f:
            json.dump(c, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE_PATH)


def candidates(ny, nx):
    """Valid (row_e, col_e, col_w) launch shapes for an ny x nx grid."""
    out = []
    for row_e in (8, 16):
        if nx // row_e > 256 or nx < row_e:
            continue
        for col_e in (8, 16):
            T = ny // col_e
            for col_w in (4, 8, 16, 32):
                if col_w > nx or col_w * T > 512 or ny * col_w * 8 > 160 * 1024:
                    continue
                out.append((row_e, col_e, col_w))
    return out
