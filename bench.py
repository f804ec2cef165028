"""Benchmark: batched uneven 4D-STEM multislice scan on B200.

Workload (one "step"): 1024 probes on 256x256 windows (16x16 raster x 4
frozen-phonon draws, 80 slices) plus 64 probes on 512x512 windows (8x8
raster, 150 slices), diamond [100] lattice, 300 keV, angular-spectrum
propagator, 25 mrad / -50 A probes, complex64 waves, float32 diffraction
patterns - 91 520 slice-steps per step.

Printed JSON line (rank 0):
  value       slice-steps/s of the batched path, inputs resident in HBM
  e2e         the same through the public API (simulate_fresnel_as with
              positions/draws) from pinned host buffers, host<->device copies
              of the potential and of the diffraction patterns inside the
              timed region (downloads on a second stream, overlapping the
              next grid class's call)
  plain       slice-steps/s of the one-probe-per-launch path (same kernels)
  grad_over_fwd  t(forward + adjoint gradient) / t(forward) on the
              512^2, 64-slice, 64-probe inverse problem (checkpoint every 8)
  err_vs_fp64 rel-L2 of exit wave and diffraction pattern vs the FP64 oracle
              (probe 0 of each grid class, as the headline scan left them)
  roofline    dominant pass kernel: algorithmic bytes / device time vs the
              measured HBM copy bandwidth
  cpu_baseline  the NumPy/SciPy FP64 restatement on the host cores

``--impl reference`` times that CPU restatement alone as the reference arm.
Multi-GPU (torchrun): the 1088 probes are sharded across the ranks in
contiguous blocks per grid class (strong scaling: the whole job's work is
fixed), no collective inside the multislice; the e2e leg runs the sharded
public API (frozen-phonon draws summed per position on the rank that owns the
position) and each rank downloads its own patterns; time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "slice-steps/s at 1 B200 batched vs plain; grad/fwd cost; err vs FP64"
WORKLOAD = ("batched uneven 4D-STEM scan: 1024 probes 256^2 x 80 slices (16x16 raster x 4 phonon draws) "
            "+ 64 probes 512^2 x 150 slices (8x8 raster); diamond [100], 300 keV, angular spectrum")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="wap", choices=["wap", "reference"])
    ap.add_argument("--small", action="store_true", help="tiny workload (testing the harness)")
    ap.add_argument("--no-extras", action="store_true", help="skip plain/grad/err/cpu sections")
    ap.add_argument("--profile-grad", action="store_true",
                    help="gradient case for ncu captures: the 512^2 x 64-slice inverse problem on a 4x4 probe "
                         "raster (16 probes), checkpoint every 8, two forward + backward steps through the "
                         "persistent scheduler")
    ap.add_argument("--profile-wpm", action="store_true",
                    help="WPM case for ncu captures: C3 (512^2, K=16, plane wave) at 3 slices, two calls")
    ap.add_argument("--profile-single", action="store_true",
                    help="single-probe case for ncu captures: C2 (1024^2 AS, plane wave) at 10 slices, two calls")
    ap.add_argument("--profile-cluster", action="store_true",
                    help="cluster-kernel case for ncu captures: one Fresnel probe on 128^2, 20 slices (C1's slice "
                         "count and probe on the grid the cluster kernel serves), two calls")
    ap.add_argument("--profile-chain", action="store_true",
                    help="chain-kernel case for ncu captures: C1 (Fresnel 256^2, 20 slices, one probe), two calls")
    ap.add_argument("--table", action="store_true",
                    help="per-configuration table (C1 Fresnel 256^2, C2 AS 1024^2, C3 WPM 512^2; one probe): B200 "
                         "time, CPU FP64/FP32 restatement on a bounded sample, error vs the FP64 oracle at full "
                         "size, roofline fraction; prints one JSON object")
    ap.add_argument("--mode", default="persistent", choices=["persistent", "batched", "graph"],
                    help="batched execution mode timed as the headline")
    ap.add_argument("--traffic-case", action="store_true",
                    help="DRAM-traffic case for ncu counter captures: the headline classes at their full slice "
                         "counts with fewer probes (228 on 256^2 = two probe groups of 114, 32 on 512^2 = one "
                         "group), one warm-up and one step, no extras; the library's bytes per pixel-slice-step "
                         "are the same per probe group as in the full step")
    ap.add_argument("--class-only", type=int, default=0, choices=[0, 256, 512],
                    help="with --traffic-case: keep only the class of this grid size (per-class profiles)")
    ap.add_argument("--profile-case", action="store_true",
                    help="reduced scan for ncu captures: 512 probes 256^2 x 4 slices + 32 probes 512^2 x 4 "
                         "slices (waves 256 + 64 MB, above L2), one warm-up and one step, no extras")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def mix_rate(t_per_step_by_class, counts):
    """slice-steps/s of the workload mix given seconds per slice-step per class."""
    total = sum(counts)
    return total / sum(t * n for t, n in zip(t_per_step_by_class, counts))


# ---------------------------------------------------------------- CPU side
def cpu_reference_sample(classes_host, scale=1, mode="fp64"):
    """Time the oracle restatement on a bounded sample of each grid class
    (16*scale probes of the 256^2 class, 2*scale of the 512^2 class, 8 slices).

    Returns (slice-steps/s for the workload mix, cores, sample description,
    seconds the sample took, slice-steps in the sample)."""
    from oracle import propagation_oracle as O
    cores = os.cpu_count() or 1
    O.set_workers(cores)
    per_step = []
    desc = []
    wall, steps = 0.0, 0
    for w in classes_host:
        H = O.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
        nb = (16 if w.ny <= 256 else 2) * scale
        ns = 8
        probes = np.stack([O.move_probe(w.probe, tuple(p)) for p in w.positions[:nb]])
        t0 = time.perf_counter()
        O.simulate_fresnel_as(w.potential[0, :ns], probes, H, w.dz, w.energy, mode=mode, return_wavefronts=False)
        dt = time.perf_counter() - t0
        wall += dt
        steps += nb * ns
        per_step.append(dt / (nb * ns))
        desc.append(f"{nb} probes x {ns} slices at {w.ny}^2")
    rate = mix_rate(per_step, [w.n_probes * w.n_slices for w in classes_host])
    return (rate, cores, "; ".join(desc) + f" (oracle {mode}, scipy.fft workers={cores}), scaled to the workload mix",
            wall, steps)


def run_reference(args, classes_host, rank):
    """The reference arm: the CPU restatement on a bounded sample per step.
    ``ms_per_step`` is the measured wall time of one sample (what each of the
    timed steps ran); ``value`` scales the sample's per-class rates to the
    workload mix (the full workload is not run on the host)."""
    if rank != 0:
        return
    rates, walls = [], []
    for i in range(args.warmup + args.steps):
        r, cores, desc, wall, steps = cpu_reference_sample(classes_host)
        if i >= args.warmup:
            rates.append(r)
            walls.append(wall)
    v = statistics.median(rates)
    total = sum(c.n_probes * c.n_slices for c in classes_host)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "slice-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.median(walls),
            "ms_per_step_note": (f"measured wall time of one step's sample ({steps} slice-steps); value scales the "
                                 f"sample's per-class rates to the {total}-slice-step workload mix, which would take "
                                 f"{total / v:.1f} s per step on these cores"),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "c128",
            "data": "synthetic", "config": {"workload": WORKLOAD},
            "cpu_baseline": {"value": v, "unit": "slice-steps/s", "cores": cores, "kind": "port", "sample": desc,
                             "sample_s": statistics.median(walls), "sample_slice_steps": steps},
            "e2e": {"value": v, "unit": "slice-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- clocks
class ClockSampler:
    def __init__(self, index=0):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [l.strip().split(", ") for l in open(self.f.name) if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for n, v in zip(names, r[5:9]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- GPU side
def profile_grad():
    import torch
    import wideanglepropagation_b200 as wap
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    w = wap.synthetic.inverse_problem(0, n=512, n_slices=64, n_side=4)
    dev = torch.device("cuda", 0)
    H = wap.fresnel_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    probe = torch.as_tensor(w.probe).to(dev)
    pos = torch.as_tensor(w.positions).to(dev)
    Vt = torch.as_tensor(w.potential[0]).to(dev)
    _, target, _ = wap.simulate_fresnel_as(Vt, probe, H, w.dz, w.energy, positions=pos, return_wavefronts=False)
    V = torch.zeros_like(Vt, requires_grad=True)
    for _ in range(2):
        V.grad = None
        _, dp = simulate_fresnel_as_differentiable(V, probe, H, w.dz, w.energy, positions=pos, ckpt_every=8)
        ((dp - target) ** 2).sum().backward()
    torch.cuda.synchronize()
    print(json.dumps({"profile_grad": "ok", "grad_norm": float(V.grad.norm())}))


def main():
    args = parse()
    if args.profile_grad:
        profile_grad()
        return
    if args.table:
        baseline_table()
        return
    if args.profile_wpm:
        profile_wpm()
        return
    if args.profile_single:
        profile_single()
        return
    if args.profile_cluster:
        profile_cluster()
        return
    if args.profile_chain:
        profile_chain()
        return
    rank, world, local = dist_env()
    import wideanglepropagation_b200.synthetic as S
    if args.profile_case:
        classes_host = [S.batched_scan_class(0, 256, 4, 16, 2), S.batched_scan_class(1, 512, 4, 4, 2)]
        args.steps, args.warmup, args.no_extras = 1, 1, True
    elif args.traffic_case:
        import dataclasses
        full = S.batched_scan(0)
        classes_host = [dataclasses.replace(full[0], positions=full[0].positions[:228],
                                            draw_of_probe=full[0].draw_of_probe[:228]),
                        dataclasses.replace(full[1], positions=full[1].positions[:32],
                                            draw_of_probe=full[1].draw_of_probe[:32])]
        if args.class_only:
            classes_host = [w for w in classes_host if w.ny == args.class_only]
        args.steps, args.warmup, args.no_extras = 1, 1, True
    else:
        classes_host = S.batched_scan(0, small=args.small)

    if args.impl == "reference":
        run_reference(args, classes_host, rank)
        return
    total_ss_job = sum(w.n_probes * w.n_slices for w in classes_host)
    job_classes = classes_host
    if world > 1:
        classes_host = [_shard_class(w, rank, world) for w in classes_host]

    import torch
    import torch.distributed as dist
    from wideanglepropagation_b200 import _lib
    import wideanglepropagation_b200 as wap
    from wideanglepropagation_b200.scan import BatchedScan, to_device_class

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    _lib.lib()
    launches0 = _lib.launch_count()
    classes = [to_device_class(w, dev) for w in classes_host]
    scan = BatchedScan(classes, mode=args.mode)
    total_ss = scan.slice_steps()

    # --- headline: batched, inputs resident in HBM --------------------------
    for _ in range(args.warmup):
        scan.step()
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local)
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = _lib.launch_count()
    torch.cuda.synchronize()
    start.record()
    for _ in range(args.steps):
        scan.step()
    stop.record()
    torch.cuda.synchronize()
    l1 = _lib.launch_count()
    clk = clocks.stop()
    # graph replays bypass the library's host-side counter: count the nodes
    graph_launches = scan.launches() * args.steps if args.mode in ("graph", "persistent") else 0
    barrier()
    ms = max_over_ranks(start.elapsed_time(stop))
    ms_per_step = ms / args.steps
    value = total_ss_job / (ms_per_step / 1e3)
    gpu_launches = (l1 - l0) + graph_launches

    extras = {}
    # --- roofline: per-pass device time with the library's event tracing -----
    _lib.profile_reset()
    _lib.profile_enable(True)
    for _ in range(max(1, min(args.steps, 3))):
        scan._eager()      # eager launches so that the tracer records them
    torch.cuda.synchronize()
    _lib.profile_enable(False)
    kinds = {}
    for k, name in _lib.KIND_NAMES.items():
        n, kms, by = _lib.profile_read(k)
        if n:
            kinds[name] = (n, kms, by)
    _lib.profile_reset()
    dom = max(kinds, key=lambda k: kinds[k][1])
    n, kms, by = kinds[dom]
    peak, peak_src = _peak_hbm()
    achieved = by / (kms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": dom, "peak_source": peak_src,
                "launches": n, "avg_launch_us": 1e3 * kms / n,
                "share": {k: v[1] / sum(x[1] for x in kinds.values()) for k, v in kinds.items()}}
    roofline["traffic"], roofline["traffic_source"] = _ncu_traffic(
        dom, sum(w.n_probes * w.n_slices * w.ny * w.nx for w in classes_host))
    # FP32 side: algorithmic flops of one launch (10 N log2 N + 24 N per
    # slice-step of an N-pixel Fresnel/AS grid) against the measured FMA peak;
    # time_frac = max(bytes / HBM peak, flops / FP32 peak) / launch time
    fp32_peak = _fp32_peak()
    flops = sum(w.n_probes * w.n_slices * (10.0 * w.ny * w.nx * np.log2(w.ny * w.nx) + 24.0 * w.ny * w.nx)
                for w in classes_host)
    launch_s = kms / n / 1e3
    roofline["fp32"] = {"achieved": flops / launch_s / 1e12, "peak": fp32_peak, "unit": "TFLOP/s",
                        "frac": flops / launch_s / 1e12 / fp32_peak, "flops_per_launch": flops,
                        "peak_source": "FMA probe (wap_fp32_probe) in this run"}
    roofline["time_frac"] = max(by / n / (peak * 1e9), flops / (fp32_peak * 1e12)) / launch_s

    if scan.sched is not None:
        st = scan.sched.status()
        if st != 0:
            raise RuntimeError(f"persistent scan reported status {st}")
    # the extras and the CPU baseline belong to the single-GPU line: with N ranks
    # the others would idle at the next collective while rank 0 runs them
    extras_on = not args.no_extras and world == 1
    if extras_on:
        # first: the exit waves are still the headline scan's (the per-pass leg rewrites them)
        extras.update(_err_vs_fp64(classes, classes_host))
        extras.update(_plain(classes, args))
        extras.update(_per_pass(classes, args))
        extras.update(_configs())
        extras.update(_grad_ratio(args))
        extras.update(_lines())
        extras.update(_potential_builder())
        extras.update(_lippmann_schwinger())

    # --- e2e through the public API from pinned host buffers ------------------
    e2e = _e2e(job_classes, args, dev, barrier, max_over_ranks, world, rank)
    if extras_on:
        # the same with a 50 mrad detector: the crop is fused into the last column pass
        extras["e2e_detector_50mrad"] = _e2e(job_classes, args, dev, barrier, max_over_ranks, world, rank,
                                             max_angle=50.0)
        # the same from atom lists: the potential and the probe are built on the device
        extras["e2e_from_atoms"] = _e2e(job_classes, args, dev, barrier, max_over_ranks, world, rank,
                                        from_atoms=True)
        # per-probe patterns (no per-position accumulation of the draws)
        extras["e2e_per_probe_patterns"] = _e2e(job_classes, args, dev, barrier, max_over_ranks, world, rank,
                                                accumulate=False)

    cpu = None
    if rank == 0 and extras_on:
        r, cores, desc, wall, steps = cpu_reference_sample(classes_host, scale=4, mode="fp64")
        cpu = {"value": r, "unit": "slice-steps/s", "cores": cores, "kind": "port", "sample": desc,
               "sample_s": wall, "sample_slice_steps": steps}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "slice-steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
                "scaling": "strong" if world > 1 else "weak",
                "vs_baseline": None, "dtype": "c64", "data": "synthetic",
                "config": {"workload": WORKLOAD, "slice_steps_per_step": total_ss_job,
                           "pixel_slice_steps_per_step": sum(w.n_probes * w.n_slices * w.ny * w.nx
                                                             for w in job_classes),
                           "l2": "inputs larger than L2 (potential 241 MB, waves 640 MB per step)",
                           "mode": {"persistent": "one persistent kernel per step (device ticket queue, TMA tiles), "
                                                  "CUDA-graph replay",
                                    "batched": "per-pass launches over all probes of a class",
                                    "graph": "per-pass launches, CUDA-graph replay"}[args.mode],
                           "parallelism": f"probe shards x{world}" + (" (strong scaling: the job's probes split "
                                                                      "across ranks)" if world > 1 else ""),
                           "patterns": "e2e: the 4 frozen-phonon draws of each 256^2 position summed in float32 "
                                       "(one pattern per position); the 512^2 class has one draw"},
                "e2e": e2e, "gpu_launches": gpu_launches, "roofline": roofline, "clocks": clk,
                "cpu_baseline": cpu}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def _sources_sha256():
    """Digest of the scan kernel's translation unit: wap_sched.cu and every
    header it includes, followed recursively (the build a profile of that
    kernel was taken on)."""
    import hashlib
    import re
    csrc = os.path.join(ROOT, "wideanglepropagation_b200", "csrc")
    seen, order = set(), []

    def visit(path):
        path = os.path.normpath(path)
        if path in seen or not os.path.exists(path):
            return
        seen.add(path)
        order.append(path)
        for inc in re.findall(r'^#include "([^"]+)"', open(path).read(), re.M):
            visit(os.path.join(os.path.dirname(path), inc))

    visit(os.path.join(csrc, "wap_sched.cu"))
    h = hashlib.sha256()
    for f in sorted(order, key=os.path.basename):
        h.update(os.path.basename(f).encode())
        h.update(open(f, "rb").read())
    return h.hexdigest()


def _ncu_traffic(kernel, pixel_slice_steps):
    """DRAM bytes per launch of ``kernel``: the committed ncu record's bytes per
    pixel-slice-step (a capture of --traffic-case) times this launch's
    pixel-slice-steps, with where it came from; traffic None when the record
    was taken on other library sources than these."""
    p = os.path.join(ROOT, "profiles", "scan_kernel_dram_traffic.txt")
    if not os.path.exists(p):
        return None, "no committed DRAM-traffic record"
    rec = {}
    for line in open(p):
        if line.startswith("#") or ":" not in line:
            continue
        k, v = line.split(":", 1)
        rec[k.strip()] = v.strip()
    if rec.get("kernel") != kernel:
        return None, f"the committed record is of {rec.get('kernel')}, not {kernel}"
    src = "profiles/scan_kernel_dram_traffic.txt (ncu dram__bytes_read.sum + dram__bytes_write.sum of " \
          "bench.py --traffic-case, scaled by pixel-slice-steps)"
    if rec.get("sources_sha256") != _sources_sha256():
        return None, src + ": taken on other library sources than this build, not used"
    return float(rec["bytes_per_pixel_slice_step"]) * pixel_slice_steps, src


def _plain(classes, args):
    import torch
    from wideanglepropagation_b200.scan import BatchedScan
    # one probe per launch sequence on a subset of each class (timing scales per slice-step)
    plain = BatchedScan(classes, mode="plain", plain_subset=16)
    plain.step()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per = []
    for c in classes:
        sub = BatchedScan([c], mode="plain", plain_subset=16)
        s.record()
        sub.step()
        e.record()
        torch.cuda.synchronize()
        per.append(s.elapsed_time(e) / 1e3 / sub.slice_steps())
    rate = mix_rate(per, [c.slice_steps for c in classes])
    # batched per class for the same comparison
    bper = []
    for c in classes:
        sub = BatchedScan([c], mode="batched")
        sub.step()
        s.record()
        sub.step()
        e.record()
        torch.cuda.synchronize()
        bper.append(s.elapsed_time(e) / 1e3 / sub.slice_steps())
    return {"plain": {"value": rate, "unit": "slice-steps/s", "sample": "16 probes per class, one probe per launch"},
            "per_class_slice_steps_per_s": {f"{c.ny}x{c.nx}": {"batched": 1 / b, "plain": 1 / p}
                                            for c, b, p in zip(classes, bper, per)}}


def profile_wpm():
    import torch
    import wideanglepropagation_b200 as wap
    w = wap.synthetic.wpm_fcc(0, n_slices=3)
    dev = torch.device("cuda", 0)
    V = torch.as_tensor(w.potential[0], device=dev)
    pr = torch.as_tensor(w.probe, device=dev)
    for _ in range(2):
        wap.simulate_wpm(V, pr, w.dz, w.energy, (w.ps, w.ps), w.n_bins, w.power_spacing, return_wavefronts=False)
    torch.cuda.synchronize()
    print(json.dumps({"profile_wpm": "ok"}))


def profile_single():
    import torch
    import wideanglepropagation_b200 as wap
    w = wap.synthetic.angular_spectrum_diamond(0, n_slices=10)
    dev = torch.device("cuda", 0)
    V = torch.as_tensor(w.potential[0], device=dev)
    pr = torch.as_tensor(w.probe, device=dev)
    H = wap.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    for _ in range(2):
        wap.simulate_fresnel_as(V, pr, H, w.dz, w.energy, return_wavefronts=False)
    torch.cuda.synchronize()
    print(json.dumps({"profile_single": "ok"}))


def profile_cluster():
    import torch
    import wideanglepropagation_b200 as wap
    w = wap.synthetic.plain_fresnel(0)
    n = 128
    dev = torch.device("cuda", 0)
    V = torch.as_tensor(w.potential[0][:, :n, :n].copy(), device=dev)
    pr = torch.as_tensor(wap.synthetic.aperture_probe(n, n, w.ps, w.energy, 20.0, -30.0), device=dev)
    H = wap.fresnel_propagation_kernel(n, n, (w.ps, w.ps), w.dz, w.energy)
    for _ in range(2):
        wap.simulate_fresnel_as(V, pr, H, w.dz, w.energy, return_wavefronts=False)
    torch.cuda.synchronize()
    print(json.dumps({"profile_cluster": "ok"}))


def profile_chain():
    """C1 (Fresnel 256^2, 20 slices, one probe) through simulate_fresnel_as,
    two calls: the case of the one-launch cooperative chain kernel."""
    import torch
    import wideanglepropagation_b200 as wap
    w = wap.synthetic.plain_fresnel(0)
    dev = torch.device("cuda", 0)
    V = torch.as_tensor(w.potential[0], device=dev)
    pr = torch.as_tensor(w.probe, device=dev)
    H = wap.fresnel_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    for _ in range(2):
        wap.simulate_fresnel_as(V, pr, H, w.dz, w.energy, return_wavefronts=False)
    torch.cuda.synchronize()
    print(json.dumps({"profile_chain": "ok"}))


def baseline_table():
    """One row per single-probe configuration: device time through the public
    API (inputs resident, no wavefront stack), error vs the FP64 oracle on
    the full configuration, the oracle in FP64 and FP32 on the host cores
    (best of 3 after a warm-up, reduced slice counts, per slice-step), and the
    roofline fraction: the roofline time max(bytes / HBM peak, flops / FP32
    peak) over the measured time, with 20 B per pixel-slice-step and the
    flops 10 N log2 N + 24 N per slice-step (Fresnel / AS) or
    (K + 1) 5 N log2 N + 30 K N (WPM), N the pixels of the grid; the HBM and
    FP32 fractions beside it."""
    import torch
    import wideanglepropagation_b200 as wap
    from oracle import propagation_oracle as O
    S = wap.synthetic
    dev = torch.device("cuda", torch.cuda.current_device())
    cores = os.cpu_count() or 1
    O.set_workers(cores)
    peak, src = _peak_hbm()
    fp32 = _fp32_peak()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timeit(fn, reps):
        fn()
        torch.cuda.synchronize()
        s.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        wap.check_errors()
        return s.elapsed_time(e) / reps

    def cpu_rate(fn, n_slices):
        fn()
        best = min(_wall(fn) for _ in range(3))
        return n_slices / best

    rows = {}
    for name, w, kind, cpu_slices in (("C1_fresnel_256_N20", S.plain_fresnel(0), "fresnel", 20),
                                      ("C2_as_1024_N100", S.angular_spectrum_diamond(0), "as", 10),
                                      ("C3_wpm_512_N200_K16", S.wpm_fcc(0), "wpm", 4)):
        V = torch.as_tensor(w.potential[0], device=dev)
        pr = torch.as_tensor(w.probe, device=dev)
        Vh = w.potential[0].astype(np.float64)
        if kind == "wpm":
            gpu = lambda: wap.simulate_wpm(V, pr, w.dz, w.energy, (w.ps, w.ps), w.n_bins, w.power_spacing,
                                           return_wavefronts=False)
            ref = O.simulate_wpm(Vh, w.probe, w.dz, w.energy, (w.ps, w.ps), w.n_bins, w.power_spacing,
                                 mode="fp64", return_wavefronts=False)
            cpu = {m: cpu_rate(lambda m=m: O.simulate_wpm(Vh[:cpu_slices], w.probe, w.dz, w.energy, (w.ps, w.ps),
                                                         w.n_bins, w.power_spacing, mode=m, return_wavefronts=False),
                               cpu_slices) for m in ("fp64", "fp32")}
        else:
            tf = O.fresnel_propagation_kernel if kind == "fresnel" else O.angular_spectrum_propagation_kernel
            H = (wap.fresnel_propagation_kernel if kind == "fresnel" else wap.angular_spectrum_propagation_kernel)(
                w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
            Ho = tf(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
            gpu = lambda: wap.simulate_fresnel_as(V, pr, H, w.dz, w.energy, return_wavefronts=False, check=False)
            ref = O.simulate_fresnel_as(Vh, w.probe, Ho, w.dz, w.energy, mode="fp64", return_wavefronts=False)
            cpu = {m: cpu_rate(lambda m=m: O.simulate_fresnel_as(Vh[:cpu_slices], w.probe, Ho, w.dz, w.energy,
                                                                mode=m, return_wavefronts=False), cpu_slices)
                   for m in ("fp64", "fp32")}
        ms = timeit(gpu, 20 if kind == "fresnel" else 5 if kind == "as" else 2)
        ex, dp, _ = gpu()
        npx = w.ny * w.nx
        flops = w.n_slices * ((w.n_bins + 1) * 5.0 * npx * np.log2(npx) + 30.0 * w.n_bins * npx if kind == "wpm"
                              else 10.0 * npx * np.log2(npx) + 24.0 * npx)
        t_bytes = 20.0 * npx * w.n_slices / (peak * 1e9)
        t_flops = flops / (fp32 * 1e12)
        rows[name] = {
            "gpu_ms_per_call": ms, "gpu_slice_steps_per_s": w.n_slices / (ms / 1e3),
            "roofline_frac": max(t_bytes, t_flops) / (ms / 1e3),
            "roofline_bound": "hbm" if t_bytes >= t_flops else "fp32",
            "hbm_frac": t_bytes / (ms / 1e3), "fp32_frac": t_flops / (ms / 1e3),
            "err_vs_fp64_exit": float(O.rel_l2(ex.cpu().numpy(), ref[0])),
            "err_vs_fp64_dp": float(O.rel_l2(dp.cpu().numpy(), ref[1])),
            "cpu_fp64_slice_steps_per_s": cpu["fp64"], "cpu_fp32_slice_steps_per_s": cpu["fp32"],
            "cpu_sample_slices": cpu_slices, "cores": cores}
    print(json.dumps({"table": rows, "peak_gbs": peak, "peak_source": src, "fp32_tflops": fp32,
                      "fp32_source": "FMA probe (wap_fp32_probe) in this run"}), flush=True)


def _wall(fn):
    t0 = time.perf_counter()
    fn()
    return time.perf_counter() - t0


def _configs():
    """Single-call timings of the other workloads through the public API
    (inputs resident on the device), with their error vs the FP64 oracle
    measured separately by the GPU tests."""
    import torch
    import wideanglepropagation_b200 as wap
    S = wap.synthetic
    dev = torch.device("cuda", torch.cuda.current_device())
    out = {}
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timeit(fn, reps):
        fn()
        torch.cuda.synchronize()
        s.record()
        for _ in range(reps):
            fn()
        e.record()
        torch.cuda.synchronize()
        wap.check_errors()
        return s.elapsed_time(e) / reps

    w = S.plain_fresnel(0)
    V = torch.as_tensor(w.potential[0], device=dev)
    pr = torch.as_tensor(w.probe, device=dev)
    H = wap.fresnel_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    # check=False: the status of each call's bounded waits is read once after
    # the timed calls (check_errors in timeit), not by a host wait per call
    ms = timeit(lambda: wap.simulate_fresnel_as(V, pr, H, w.dz, w.energy, check=False), 20)
    ms_ns = timeit(lambda: wap.simulate_fresnel_as(V, pr, H, w.dz, w.energy, return_wavefronts=False, check=False), 20)
    out["fresnel_256_N20_1probe"] = {"ms_per_call": ms, "ms_per_call_no_stack": ms_ns,
                                     "slice_steps_per_s": w.n_slices / (ms_ns / 1e3)}
    w = S.angular_spectrum_diamond(0)
    V = torch.as_tensor(w.potential[0], device=dev)
    pr = torch.as_tensor(w.probe, device=dev)
    H = wap.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    ms_ns = timeit(lambda: wap.simulate_fresnel_as(V, pr, H, w.dz, w.energy, return_wavefronts=False, check=False), 5)
    out["as_1024_N100_1probe"] = {"ms_per_call_no_stack": ms_ns, "slice_steps_per_s": w.n_slices / (ms_ns / 1e3),
                                  "pixel_slice_steps_per_s": w.n_slices * w.ny * w.nx / (ms_ns / 1e3)}
    w = S.wpm_fcc(0)
    V = torch.as_tensor(w.potential[0], device=dev)
    pr = torch.as_tensor(w.probe, device=dev)
    ms_ns = timeit(lambda: wap.simulate_wpm(V, pr, w.dz, w.energy, (w.ps, w.ps), 16, 1.0, return_wavefronts=False), 2)
    out["wpm_512_N200_K16_1probe"] = {"ms_per_call_no_stack": ms_ns, "slice_steps_per_s": w.n_slices / (ms_ns / 1e3)}
    return {"configs": out}


def _per_pass(classes, args):
    import torch
    from wideanglepropagation_b200.scan import BatchedScan
    sc = BatchedScan(classes, mode="batched")
    sc.step()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(2):
        sc.step()
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / 2
    return {"batched_per_pass": {"value": sc.slice_steps() / (ms / 1e3), "unit": "slice-steps/s",
                                 "ms_per_step": ms}}


def _grad_ratio(args):
    import torch
    import wideanglepropagation_b200 as wap
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    w = wap.synthetic.inverse_problem(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    H = wap.fresnel_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    probe = torch.as_tensor(w.probe).to(dev)
    pos = torch.as_tensor(w.positions).to(dev)
    Vt = torch.as_tensor(w.potential[0]).to(dev)
    _, target, _ = wap.simulate_fresnel_as(Vt, probe, H, w.dz, w.energy, positions=pos, return_wavefronts=False)
    V = torch.zeros_like(Vt, requires_grad=True)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def fwd():
        with torch.no_grad():
            return wap.simulate_fresnel_as(V, probe, H, w.dz, w.energy, positions=pos, return_wavefronts=False)

    def step(k):
        V.grad = None
        _, dp = simulate_fresnel_as_differentiable(V, probe, H, w.dz, w.energy, positions=pos, ckpt_every=k)
        ((dp - target) ** 2).sum().backward()

    out = {}
    for _ in range(2):
        fwd(); step(8); step(1)
    torch.cuda.synchronize()
    reps = 3
    s.record()
    for _ in range(reps):
        fwd()
    e.record()
    torch.cuda.synchronize()
    t_f = s.elapsed_time(e) / reps
    for k in (8, 1):
        s.record()
        for _ in range(reps):
            step(k)
        e.record()
        torch.cuda.synchronize()
        out[k] = s.elapsed_time(e) / reps / t_f
    return {"grad_over_fwd": out[8], "grad_over_fwd_ckpt1": out[1], "grad_fwd_ms": t_f,
            "grad_workload": "512^2, 64 slices x 2 A, 300 keV, 64 probes (8x8), L = sum(|FFT psi|^2 - I)^2"}


def _fp32_peak():
    """FP32 FMA throughput (TFLOP/s) of this GPU: 8 CTAs of 256 threads per SM,
    each thread 2^14 x 8 independent FMAs; best of five after three warm-ups."""
    import ctypes
    import torch
    from wideanglepropagation_b200 import _lib
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    blocks, iters = sms * 8, 1 << 14
    out = torch.empty(blocks * 256, dtype=torch.float32, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)

    def launch():
        _lib.check(_lib.lib().wap_fp32_probe(blocks, iters, ctypes.c_void_p(out.data_ptr()), stream))

    for _ in range(3):
        launch()
    best = None
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        launch()
        e.record()
        torch.cuda.synchronize()
        t = s.elapsed_time(e) / 1e3
        best = t if best is None else min(best, t)
    return blocks * 256 * iters * 8 * 2 / best / 1e12


def _peak_hbm():
    """Measured HBM copy bandwidth (GB/s) and its source; the pool's earlier
    measurement when the measured-peaks file is absent."""
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        return float(json.load(open(peaks_path))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _potential_builder():
    """Device potential builder on the C2 configuration (1024^2 diamond [100],
    100 slices: 419 MB of float32 written) vs the host NumPy builder (4 slices,
    scaled)."""
    import torch
    import wideanglepropagation_b200 as wap
    import wideanglepropagation_b200.synthetic as S
    n, N, ps, dz = 1024, 100, 0.05, 1.3575
    pos, sl = S.lattice_atoms(np.random.default_rng(0), N, n, n, ps, 5.43, S.DIAMOND_LAYERS, 0.08)
    for _ in range(2):
        V = wap.gaussian_potential(N, n, n, ps, pos, sl, 25.0, 0.25, scale=1 / dz)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 5
    s.record()
    for _ in range(reps):
        V = wap.gaussian_potential(N, n, n, ps, pos, sl, 25.0, 0.25, scale=1 / dz)
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / reps
    del V
    t0 = time.perf_counter()
    S.lattice_stack(np.random.default_rng(0), 4, n, n, ps, 5.43, S.DIAMOND_LAYERS, 25.0, 0.25, 0.08)
    host_ms = (time.perf_counter() - t0) * 1e3 * N / 4
    gbs = 4.0 * N * n * n / (ms / 1e3) / 1e9
    peak, src = _peak_hbm()
    return {"potential_builder_c2": {"ms": ms, "atoms": int(pos.shape[0]), "written_gbs": gbs, "peak_gbs": peak,
                                     "peak_source": src, "frac": gbs / peak, "host_numpy_ms": host_ms,
                                     "note": "includes the atom-list upload (pageable) in each call"}}


def _lippmann_schwinger():
    """Lippmann-Schwinger 2D solve of a 128^2 Gaussian-atom potential (padded
    256^2, convolutions on 512^2) at the reference's default tolerance, on the
    device and with the float64 oracle on the host cores."""
    import torch
    import wideanglepropagation_b200 as wap
    import wideanglepropagation_b200.synthetic as S
    from oracle import propagation_oracle as O
    V = S.random_gaussian_stack(np.random.default_rng(0), 1, 128, 128, 0.1, 30, 20.0, 0.3)[0] / 2.0
    wap.solve_scattering_2d_lippmann_schwinger(V, 200e3, 0.1)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    psi = wap.solve_scattering_2d_lippmann_schwinger(V, 200e3, 0.1)
    torch.cuda.synchronize()
    gpu_ms = (time.perf_counter() - t0) * 1e3
    O.set_workers(os.cpu_count() or 1)
    t0 = time.perf_counter()
    ref = O.solve_scattering_2d_lippmann_schwinger(V, 200e3, 0.1)
    cpu_ms = (time.perf_counter() - t0) * 1e3
    err = float(np.linalg.norm(psi.cpu().numpy() - ref) / np.linalg.norm(ref))
    return {"lippmann_schwinger_128": {"device_ms": gpu_ms, "oracle_cpu_ms": cpu_ms, "rel_vs_oracle": err,
                                        "note": "wall clock incl. the host kernel build; gmres_tol 1e-4, restart 70"}}


def _lines():
    """1D helpers: propagate_1d over 65536 lines of 2048 points (1 GiB in,
    1 GiB out: HBM-bound, 16 B per point) and the naive per-pixel WPM step on
    64^2 (direct float64 sums)."""
    import torch
    import wideanglepropagation_b200 as wap
    n, L = 2048, 65536
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev).manual_seed(0)
    psi = torch.randn((L, n), dtype=torch.complex64, device=dev, generator=g)
    kx = wap.get_kx_1d(n, 0.2)
    H = wap.angular_spectrum_kernel_1d(kx ** 2, 20.0, 3.0)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(3):
        wap.propagate_1d(psi, H)
    torch.cuda.synchronize()
    reps = 10
    s.record()
    for _ in range(reps):
        wap.propagate_1d(psi, H)
    e.record()
    torch.cuda.synchronize()
    ms = s.elapsed_time(e) / reps
    gbs = 16.0 * n * L / (ms / 1e3) / 1e9
    peak, peak_src = _peak_hbm()
    rng = np.random.default_rng(0)
    wave = rng.normal(size=(64, 64)) + 1j * rng.normal(size=(64, 64))
    nmap = 1.0 + 1e-4 * rng.random((64, 64))
    wap.wpm_step(wave, nmap, 2.0, 300e3, (0.05, 0.05))
    torch.cuda.synchronize()
    s.record()
    wap.wpm_step(wave, nmap, 2.0, 300e3, (0.05, 0.05))
    e.record()
    torch.cuda.synchronize()
    return {"lines_1d": {"propagate_1d_ms": ms, "lines": L, "n": n, "achieved_gbs": gbs, "peak_gbs": peak,
                         "peak_source": peak_src, "frac": gbs / peak, "bytes_per_point": 16},
            "wpm_naive_step_64x64_ms": s.elapsed_time(e)}


def _err_vs_fp64(classes, classes_host):
    import torch
    import wideanglepropagation_b200 as wap
    from oracle import propagation_oracle as O
    errs = {}
    for c, w in zip(classes, classes_host):
        b = 0
        H = O.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
        p0 = O.move_probe(w.probe, tuple(w.positions[b]))
        rex, rdp, _ = O.simulate_fresnel_as(w.potential[w.draw_of_probe[b]], p0, H, w.dz, w.energy,
                                            return_wavefronts=False)
        torch.cuda.synchronize()
        errs[f"{w.ny}x{w.nx}"] = {"exit": O.rel_l2(c.exit[b].cpu().numpy(), rex),
                                  "dp": O.rel_l2(c.dp[b].cpu().numpy(), rdp)}
    return {"err_vs_fp64": errs}


def _shard_class(w, rank, world):
    """This rank's contiguous block of a grid class's probes (strong scaling)."""
    import dataclasses
    from wideanglepropagation_b200.distributed import shard_bounds
    lo, hi = shard_bounds(w.n_probes, rank, world)
    return dataclasses.replace(w, positions=w.positions[lo:hi], draw_of_probe=w.draw_of_probe[lo:hi])


def _positions_of(w):
    """Pattern index of each probe: its scan position (draw-major probe order);
    None for a class with one draw (one probe per position already)."""
    D = w.potential.shape[0]
    if D == 1:
        return None
    P = w.n_probes // D
    return np.arange(w.n_probes) % P


def _e2e(classes_host, args, dev, barrier, max_over_ranks, world, rank=0, max_angle=None, from_atoms=False,
         accumulate=True):
    """The headline workload through the public API from pinned host buffers
    (sharded_simulate_fresnel_as: at one GPU simply simulate_fresnel_as), the
    draws of each position summed into one pattern (``accumulate``); with
    ``max_angle`` (mrad) the patterns come back cropped to that detector
    window (the crop fused into the last column pass); with ``from_atoms``
    each step uploads the atom lists instead of the potential and builds the
    potential and the probe on the device (gaussian_potential,
    aperture_probe)."""
    import torch
    import torch.distributed as dist
    import wideanglepropagation_b200 as wap
    import wideanglepropagation_b200.synthetic as S
    from wideanglepropagation_b200.distributed import probe_shard, sharded_simulate_fresnel_as
    host = []
    atoms = []
    h2d = d2h = 0
    for ci, w in enumerate(classes_host):
        V = torch.from_numpy(w.potential).pin_memory()
        acc = _positions_of(w) if accumulate else None
        mine, first, count = probe_shard(w.n_probes, rank, world, acc)
        if from_atoms:
            D, N = w.potential.shape[:2]
            side = int(round((w.n_probes // D) ** 0.5))
            pos, rows = S.batched_scan_class_atoms(ci, w.ny, N, side, D)   # the seeds of batched_scan(0)
            atoms.append((pos, rows, D, N))
            h2d += pos.nbytes // 2 * 3 + (N * D + 1) * 4                   # (M, 3) float64 + offsets
        else:
            h2d += V.numel() * 4 + w.probe.size * 8
        H = wap.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
        win = wap.detector_window((w.ny, w.nx), (w.ps, w.ps), w.energy, max_angle) if max_angle else None
        shape = (count, win[2], win[3]) if win else (count, w.ny, w.nx)
        q = torch.from_numpy(w.positions).pin_memory()
        d = torch.from_numpy(w.draw_of_probe).pin_memory()
        h2d += len(mine) * (8 + 4) + (len(mine) + count + 1) * 4 * (1 if accumulate else 0)
        out = torch.empty(shape, dtype=torch.float32).pin_memory()
        d2h += out.numel() * 4
        host.append((w, V, torch.from_numpy(w.probe).pin_memory(), q, d, H, out, acc))
    if world > 1:
        t = torch.tensor([h2d, d2h], dtype=torch.float64, device=dev)
        dist.all_reduce(t)
        h2d, d2h = int(t[0]), int(t[1])
    # patterns go back on a second stream, so that a class's download overlaps
    # the next class's multislice (the end of the timed region waits for it)
    down = torch.cuda.Stream()

    def step():
        for i, (w, V, p, q, d, H, out, acc) in enumerate(host):
            if from_atoms:
                pos, rows, D, N = atoms[i]
                V = wap.gaussian_potential(D * N, w.ny, w.nx, w.ps, pos, rows, 25.0, 0.25,
                                           scale=1 / w.dz).view(D, N, w.ny, w.nx)
                p = wap.aperture_probe(w.ny, w.nx, w.ps, w.energy, 25.0, -50.0)
            # check=False: the scheduler's status is read once per step below,
            # so the host does not wait for one class before queueing the next
            dp, _, _ = sharded_simulate_fresnel_as(V, p, H, w.dz, w.energy, positions=q, draw=d, accumulate=acc,
                                                   gather=False, max_angle=max_angle, sampling=(w.ps, w.ps),
                                                   check=False)
            down.wait_stream(torch.cuda.current_stream())
            with torch.cuda.stream(down):
                out.copy_(dp, non_blocking=True)
            dp.record_stream(down)
        # steps are pipelined like a stream of scans: the next step's uploads
        # and multislice overlap this step's last download (the downloads stay
        # in order on their stream); finished runs' statuses are checked here
        # without waiting, the rest after the loop
        wap.propagation._lib.poll_errors()

    def finish():
        torch.cuda.current_stream().wait_stream(down)

    for _ in range(max(1, args.warmup)):
        step()
    finish()
    torch.cuda.synchronize()
    wap.check_errors()
    barrier()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record()
    for _ in range(args.steps):
        step()
    finish()
    e.record()
    torch.cuda.synchronize()
    wap.check_errors()   # raises if a bounded device-side wait expired in any timed step
    ms = max_over_ranks(s.elapsed_time(e)) / args.steps
    total = sum(w.n_probes * w.n_slices for w in classes_host)
    api = "simulate_fresnel_as(positions=, draw=, accumulate=per position)" if accumulate else \
        "simulate_fresnel_as(positions=, draw=)"
    if max_angle:
        api = api[:-1] + f", max_angle={max_angle:g}, sampling=)"
    if world > 1:
        api = "sharded_simulate_fresnel_as over " + api
    if from_atoms:
        api = "gaussian_potential(atoms) + aperture_probe + " + api
    return {"value": total / (ms / 1e3), "unit": "slice-steps/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": d2h, "ms_per_step": ms, "api": api}


if __name__ == "__main__":
    main()
