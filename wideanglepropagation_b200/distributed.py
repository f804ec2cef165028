"""Multi-GPU probe sharding (one process per GPU, torch.distributed).

Every probe of a scan is an independent multislice (the reference's caller
loop of ``simulate_fresnel_as(V, move_probe(probe, pos), H, dz, E)``,
propagation.py:263-276, :305-352), so a scan shards by probes: rank r takes a
contiguous block of probe indices, the potential and the transfer function
are replicated, and the forward pass needs no collective.  The patterns are
gathered once (``all_gather`` over NCCL/NVLink on GPUs, gloo on CPU in the
tests).  When the patterns of several probes are summed into one
(``accumulate``, e.g. the frozen-phonon draws of a scan position) the shards
are blocks of output patterns, each with all of its probes, so every sum is
formed on one rank in the same order as on one GPU.  The gradient of a loss
summed over probes needs one all-reduce (sum, float32) of dL/dV.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np
import torch
import torch.distributed as dist


def shard_bounds(n_items: int, rank: int, world: int) -> tuple:
    """Contiguous block [lo, hi) of ``n_items`` owned by ``rank``; blocks differ
    in size by at most one and cover every item exactly once."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError(f"bad rank {rank} for world size {world}")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def shard(seq, rank: int, world: int):
    lo, hi = shard_bounds(len(seq), rank, world)
    return seq[lo:hi]


def _pinned(a: np.ndarray) -> torch.Tensor:
    """A host array as a pinned tensor (uploads without waiting for the queued
    work); plain CPU memory where no CUDA device is present (the CPU tests)."""
    t = torch.from_numpy(np.ascontiguousarray(a))
    return t.pin_memory() if torch.cuda.is_available() else t


def _rank_world(group) -> tuple:
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def reduce_gradient(grad: torch.Tensor, group: Optional[dist.ProcessGroup] = None) -> torch.Tensor:
    """Sum a per-rank dL/dV over all ranks in place (no-op without a process group)."""
    if dist.is_available() and dist.is_initialized() and dist.get_world_size(group) > 1:
        dist.all_reduce(grad, op=dist.ReduceOp.SUM, group=group)
    return grad


def sharded_gradient(potential: torch.Tensor, positions: Sequence, grad_fn: Callable,
                     group: Optional[dist.ProcessGroup] = None) -> torch.Tensor:
    """dL/dV of a loss summed over all probe positions.

    ``grad_fn(potential, local_positions) -> dL/dV`` evaluates this rank's
    shard (e.g. a backward through ``simulate_fresnel_as_differentiable``);
    the shard gradients are then summed over ranks.
    """
    rank, world = _rank_world(group)
    local = shard(positions, rank, world)
    g = grad_fn(potential, local) if len(local) else torch.zeros_like(potential)
    return reduce_gradient(g, group)


def probe_shard(n_probes: int, rank: int, world: int, accumulate=None):
    """This rank's probes: (probe indices, pattern-index offset, pattern count).

    Without ``accumulate`` a contiguous block of probes; with it, the probes of
    a contiguous block of output patterns (each pattern's probes stay on one
    rank), their pattern indices renumbered from 0."""
    if accumulate is None:
        lo, hi = shard_bounds(n_probes, rank, world)
        return np.arange(lo, hi), lo, hi - lo
    acc = np.asarray(accumulate.cpu() if isinstance(accumulate, torch.Tensor) else accumulate).reshape(-1)
    if acc.shape[0] != n_probes:
        raise ValueError(f"accumulate needs one pattern index per probe ({n_probes}), got {acc.shape[0]}")
    n_patterns = int(acc.max()) + 1 if acc.size else 0
    lo, hi = shard_bounds(n_patterns, rank, world)
    mine = np.nonzero((acc >= lo) & (acc < hi))[0]
    return mine, lo, hi - lo


def gather_blocks(local: torch.Tensor, counts: Sequence[int], group=None) -> torch.Tensor:
    """Concatenate every rank's leading-axis block (``counts[r]`` rows on rank
    r) in rank order, on every rank: one all_gather of blocks padded to the
    largest count."""
    rank, world = _rank_world(group)
    if world == 1:
        return local
    m = max(counts)
    pad = torch.zeros((m,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    pad[:local.shape[0]] = local
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[:c] for b, c in zip(bufs, counts)])


def sharded_simulate_fresnel_as(potential, probe, prop_kernel, slice_thickness, energy, *, positions, draw=None,
                                accumulate=None, gather: bool = True, return_exit: bool = False,
                                group: Optional[dist.ProcessGroup] = None, forward: Optional[Callable] = None,
                                **kwargs):
    """``simulate_fresnel_as`` over a scan sharded across the ranks of ``group``.

    Each rank runs its probes (``probe_shard``) with ``forward`` (default: the
    library's ``simulate_fresnel_as``; ``kwargs`` pass through, e.g.
    ``max_angle``/``sampling``/``check``), then the patterns are gathered in
    probe (or pattern) order on every rank.  Returns ``(patterns, exit_waves or
    None)``; with ``gather=False`` this rank's block and its first index
    instead.  No collective runs inside the multislice itself.
    """
    if forward is None:
        from .propagation import simulate_fresnel_as as forward
    rank, world = _rank_world(group)
    pos = np.asarray(positions.cpu() if isinstance(positions, torch.Tensor) else positions).reshape(-1, 2)
    B = pos.shape[0]
    mine, first, count = probe_shard(B, rank, world, accumulate)
    whole = len(mine) == B   # one rank (or all probes here): pass the caller's arrays through unchanged
    local_pos = positions if whole else _pinned(pos[mine])
    dr = None
    if draw is not None:
        dr = draw if whole else _pinned(np.asarray(draw.cpu() if isinstance(draw, torch.Tensor) else draw)
                                        .reshape(-1)[mine])
    acc_local = None
    if accumulate is not None:
        acc = np.asarray(accumulate.cpu() if isinstance(accumulate, torch.Tensor) else accumulate).reshape(-1)
        acc_local = acc[mine] - first
    if len(mine):
        ex, dp, _ = forward(potential, probe, prop_kernel, slice_thickness, energy, positions=local_pos,
                            draw=dr, accumulate=acc_local, return_wavefronts=False, **kwargs)
        if accumulate is not None and dp.shape[0] < count:
            # trailing patterns of this block that no probe maps to
            z = torch.zeros((count - dp.shape[0],) + tuple(dp.shape[1:]), dtype=dp.dtype, device=dp.device)
            dp = torch.cat([dp, z])
    else:
        ex = dp = None
    if not gather:
        return dp, (ex if return_exit else None), first
    counts = [probe_shard(B, r, world, accumulate)[2] for r in range(world)]
    if dp is None:
        raise ValueError("a rank without probes cannot infer the pattern shape; use fewer ranks than probes")
    out = gather_blocks(dp, counts, group)
    exits = None
    if return_exit:
        if accumulate is not None:
            raise ValueError("return_exit with accumulate: exit waves are per probe, patterns per position")
        exits = gather_blocks(ex, counts, group)
    return out, exits


class _SumGradientAcrossRanks(torch.autograd.Function):
    """Identity forward; the backward all-reduces dL/dV over the group, so a
    loss summed over every rank's probes gets its full gradient on each rank."""

    @staticmethod
    def forward(ctx, V, group):
        ctx.group = group
        return V.view_as(V)

    @staticmethod
    def backward(ctx, g):
        g = g.contiguous().clone()
        reduce_gradient(g, ctx.group)
        return g, None


def sharded_differentiable(potential: torch.Tensor, probe, prop_kernel, slice_thickness, energy, *, positions,
                           draw=None, group: Optional[dist.ProcessGroup] = None,
                           forward: Optional[Callable] = None, **kwargs):
    """This rank's (exit_waves, patterns) of a sharded differentiable scan.

    The probes are sharded like ``sharded_simulate_fresnel_as``; a loss formed
    from the returned local patterns and summed over ranks (each rank calling
    ``backward`` on its own part) leaves the gradient of the total loss in
    ``potential.grad`` on every rank: the potential passes through an identity
    whose backward is one all-reduce (sum) of dL/dV.  ``forward`` defaults to
    ``simulate_fresnel_as_differentiable``.  Returns (exit, dp, first probe)."""
    if forward is None:
        from .autograd import simulate_fresnel_as_differentiable as forward
    rank, world = _rank_world(group)
    pos = np.asarray(positions.cpu() if isinstance(positions, torch.Tensor) else positions).reshape(-1, 2)
    mine, first, _ = probe_shard(pos.shape[0], rank, world)
    dr = None
    if draw is not None:
        dr = np.asarray(draw.cpu() if isinstance(draw, torch.Tensor) else draw).reshape(-1)[mine]
    V = _SumGradientAcrossRanks.apply(potential, group) if world > 1 else potential
    ex, dp = forward(V, probe, prop_kernel, slice_thickness, energy, positions=pos[mine], draw=dr, **kwargs)
    return ex, dp, first
