"""Probe sharding and gradient reduction across ranks (gloo, world size 2, CPU)."""
import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from wideanglepropagation_b200.distributed import reduce_gradient, shard, shard_bounds, sharded_gradient


@pytest.mark.parametrize("n,world", [(0, 2), (1, 2), (7, 2), (1088, 8), (64, 3)])
def test_shard_bounds_partition(n, world):
    seen = []
    for r in range(world):
        lo, hi = shard_bounds(n, r, world)
        seen += list(range(lo, hi))
        assert hi - lo in (n // world, n // world + 1)
    assert seen == list(range(n))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        positions = [(i, 2 * i) for i in range(11)]
        V = torch.zeros(3, 4, 4)

        def grad_fn(pot, local):
            # per-probe contribution that identifies the probe: slice 0 gets
            # sum of row indices, slice 1 the count
            g = torch.zeros_like(pot)
            g[0] += sum(p[0] for p in local)
            g[1] += len(local)
            return g

        g = sharded_gradient(V, positions, grad_fn)
        q.put((rank, float(g[0, 0, 0]), float(g[1, 0, 0]), len(shard(positions, rank, world))))
        t = torch.full((5,), float(rank + 1))
        reduce_gradient(t)
        assert torch.all(t == sum(range(1, world + 1)))
    finally:
        dist.destroy_process_group()


def test_sharded_gradient_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, s0, s1, n_local in res:
        assert s0 == sum(range(11)) and s1 == 11
    assert sum(r[3] for r in res) == 11
