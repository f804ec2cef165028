"""Launch-shape autotuner for the multislice passes and the persistent scheduler.

Per-pass kernels — candidates per grid: elements per thread of the row pass
(``row_e``), of the column pass (``col_e``) and columns per column-pass CTA
(``col_w``), for batched calls and for one- or two-probe calls.  Persistent
scheduler — the probe-group size (probes advanced together through every pass:
enough tiles per pass to keep the resident CTAs busy, few enough that the
group's waves stay in L2).  Each candidate is timed on the device with CUDA
events over a short synthetic multislice; the winner is cached in
``autotune_cache.json`` keyed by GPU name, grid, op, bin count and batch class,
and applied to every plan or scan created afterwards.
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


SINGLE_MAX = 2   # calls with at most this many probes use the "single" launch shapes


def batch_class(batch: int) -> str:
    """'single' for one or two probes (few CTAs per pass: the shape must spread
    them over the SMs), 'any' otherwise."""
    return "single" if batch <= SINGLE_MAX else "any"


def _load() -> dict:
    global _cache
    if _cache is None:
        try:
            with open(CACHE_PATH) as f:
                _cache = json.load(f)
        except (OSError, ValueError):
            _cache = {}
    return _cache


def lookup(ny, nx, op, n_bins=0, cls="any"):
    """Cached (row_e, col_e, col_w) for this GPU, grid and batch class (falling
    back to the 'any' entry), or None."""
    with _lock:
        c = _load()
        v = c.get(_key(ny, nx, op, n_bins, cls)) or c.get(_key(ny, nx, op, n_bins))
    return tuple(v) if v else None


def store(ny, nx, op, n_bins, cfg, cls="any") -> None:
    with _lock:
        c = _load()
        c[_key(ny, nx, op, n_bins, cls)] = list(cfg)
        tmp = CACHE_PATH + ".tmp"
        with open(tmp, "w") as f:
            json.dump(c, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE_PATH)


def candidates(ny, nx):
    """Valid (row_e, col_e, col_w) launch shapes for an ny x nx grid."""
    out = []
    for row_e in (4, 8, 16):
        if nx // row_e > 256 or nx < row_e:
            continue
        for col_e in (4, 8, 16):
            T = ny // col_e
            for col_w in (2, 4, 8, 16, 32):
                if col_w > nx or col_w * T > 512 or ny * col_w * 8 > 160 * 1024:
                    continue
                out.append((row_e, col_e, col_w))
    return out


def _time_config(plan, run, reps=3):
    import torch
    run()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        s.record()
        run()
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    return best


def tune(ny: int, nx: int, op: int = 0, n_bins: int = 0, batch: int | None = None, n_slices: int = 6,
         verbose: bool = False):
    """Time every candidate launch shape on a synthetic multislice of ``batch``
    probes and cache the fastest; returns (config, {config: ms})."""
    import numpy as np
    import torch
    from . import _lib
    from .propagation import get_plan, simulate_fresnel_as, simulate_wpm
    if batch is None:
        batch = max(1, (64 * 2 ** 20) // (ny * nx * 8)) if op == 0 else 1
    rng = np.random.default_rng(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    V = torch.as_tensor(rng.uniform(0, 30, (n_slices, ny, nx)).astype(np.float32), device=dev)
    probe = torch.ones((ny, nx), dtype=torch.complex64, device=dev)
    pos = torch.as_tensor(np.stack([rng.integers(0, ny, batch), rng.integers(0, nx, batch)], 1).astype(np.int32),
                          device=dev)
    H = torch.exp(1j * torch.as_tensor(rng.uniform(-3, 3, (ny, nx)), device=dev)).to(torch.complex128)
    plan = get_plan(ny, nx, batch, op, n_bins)
    old = plan.config()

    def run():
        if op == _lib.WAP_OP_WPM:
            simulate_wpm(V, probe, 2.0, 300e3, (0.05, 0.05), n_bins, 1.0, return_wavefronts=False, positions=pos)
        else:
            simulate_fresnel_as(V, probe, H, 2.0, 300e3, return_wavefronts=False, positions=pos)

    times = {}
    for cfg in candidates(ny, nx):
        try:
            plan.set_config(*cfg)
        except ValueError:
            continue
        times[cfg] = _time_config(plan, run)
        if verbose:
            print(f"  {ny}x{nx} op{op} {cfg}: {times[cfg]:.3f} ms", flush=True)
    best = min(times, key=times.get)
    plan.set_config(*best) if best else plan.set_config(*old)
    store(ny, nx, op, n_bins, best, batch_class(batch))
    return best, times


def default_scan_group(n: int) -> int:
    """The scheduler's built-in probe-group size: 4 x the resident CTAs (3 per
    SM) in tiles, a tile being 4096 pixels (16 elements x 256 threads)."""
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    row_tiles = max(1, n * n // 4096)
    return max(1, -(-4 * 3 * sms // row_tiles))


def balanced_group(group: int, batch: int) -> int:
    """A probe-group size adjusted so that ``batch`` probes split into
    round(batch / group) groups of equal size (a short last group would run
    its dependency chain with most SMs idle); 0 stays 0 (the scheduler's own
    rule, which balances the same way)."""
    if group <= 0 or batch <= 0:
        return group
    ng = max(1, (batch + group // 2) // group)
    return -(-batch // ng)


def lookup_scan(n: int) -> int:
    """Cached probe-group size of the persistent scheduler for n x n grids (0: built-in)."""
    with _lock:
        v = _load().get(_key(n, n, "scan", 0))
    return int(v[0]) if v else 0


def tune_scan(n: int, n_slices: int = 8, verbose: bool = False):
    """Time the persistent scheduler on a synthetic n x n scan at probe-group
    sizes around the built-in one; cache and return the fastest."""
    import numpy as np
    import torch
    from .scan import BatchedScan, DeviceClass
    from .propagation import transfer_pair
    g0 = default_scan_group(n)
    cands = sorted({max(1, g0 // 4), max(1, g0 // 2), max(1, (3 * g0) // 4), g0, (3 * g0) // 2, 2 * g0})
    B = 8 * g0
    dev = torch.device("cuda", torch.cuda.current_device())
    gen = torch.Generator(device=dev).manual_seed(0)
    V = torch.rand((1, n_slices, n, n), generator=gen, device=dev) * 30
    probe = torch.ones((n, n), dtype=torch.complex64, device=dev)
    pos = torch.randint(0, n, (B, 2), generator=gen, device=dev, dtype=torch.int32)
    H, H_lo = transfer_pair("as", n, n, (0.05, 0.05), 2.0, 300e3)
    cls = DeviceClass(n, n, n_slices, 1, B, 2.0, 300e3, V, probe, pos, torch.zeros(B, dtype=torch.int32, device=dev),
                      H, H_lo, torch.empty((B, n, n), dtype=torch.complex64, device=dev),
                      torch.empty((B, n, n), dtype=torch.float32, device=dev))
    times = {}
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for g in cands:
        bs = BatchedScan([cls], mode="persistent", groups=[g])
        bs.step()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(3):
            s.record()
            bs.step()
            e.record()
            torch.cuda.synchronize()
            best = min(best, s.elapsed_time(e))
        times[g] = best
        if verbose:
            print(f"  scan {n}x{n} group {g}: {best:.3f} ms", flush=True)
        del bs
    best = min(times, key=times.get)
    with _lock:
        c = _load()
        c[_key(n, n, "scan", 0)] = [int(best)]
        tmp = CACHE_PATH + ".tmp"
        with open(tmp, "w") as f:
            json.dump(c, f, indent=1, sort_keys=True)
        os.replace(tmp, CACHE_PATH)
    return best, times


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser(description="autotune the multislice launch shapes on this GPU")
    ap.add_argument("--grids", default="256,512,1024", help="comma-separated square grid sizes")
    ap.add_argument("--wpm-bins", default="16", help="comma-separated WPM bin counts to tune (empty: none)")
    ap.add_argument("--single", action="store_true", help="tune the single-probe shapes (batch 1) instead")
    ap.add_argument("--scan", action="store_true", help="tune the persistent scheduler's probe-group size instead")
    args = ap.parse_args(argv)
    if args.scan:
        for n in [int(v) for v in args.grids.split(",") if v]:
            best, _ = tune_scan(n, verbose=True)
            print(f"{n}x{n} scan group best {best} (built-in {default_scan_group(n)})", flush=True)
        print(f"cache: {CACHE_PATH}")
        return
    b = 1 if args.single else None
    for n in [int(v) for v in args.grids.split(",") if v]:
        best, _ = tune(n, n, 0, 0, batch=b, verbose=True)
        print(f"{n}x{n} fresnel/as best {best}", flush=True)
        for k in [int(v) for v in args.wpm_bins.split(",") if v]:
            best, _ = tune(n, n, 1, k, batch=b, verbose=True)
            print(f"{n}x{n} wpm K={k} best {best}", flush=True)
    print(f"cache: {CACHE_PATH}")


if __name__ == "__main__":
    main()
