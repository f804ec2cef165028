"""Multi-GPU probe sharding (one process per GPU, torch.distributed).

Every probe of a scan is an independent multislice, so a scan shards by
probes: rank r takes a contiguous block of probe indices, the potential and
transfer function are replicated, and the forward pass needs no collective.
The gradient of a loss summed over probes needs one all-reduce (sum, float32)
of dL/dV over the ranks (NCCL over NVLink on GPUs, gloo on CPU for tests).
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

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
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    local = shard(positions, rank, world)
    g = grad_fn(potential, local) if len(local) else torch.zeros_like(potential)
    return reduce_gradient(g, group)
