"""Probe sharding and gradient reduction across ranks (gloo, world size 2, CPU)."""
import os
import socket

import numpy as np

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


def _tag_forward(potential, probe, H, dz, E, *, positions, draw=None, accumulate=None, return_wavefronts=False,
                 **kw):
    """CPU stand-in for simulate_fresnel_as: probe b's 'pattern' is a 2x3
    array filled with a tag of its position and draw, its 'exit wave' the
    same tag as a complex value; patterns summed per accumulate index in
    probe order, as the library does."""
    pos = np.asarray(positions)
    d = np.zeros(len(pos)) if draw is None else np.asarray(draw)
    tag = torch.tensor(pos[:, 0] * 1000.0 + pos[:, 1] + 0.25 * d, dtype=torch.float64)
    dp = tag[:, None, None].expand(len(pos), 2, 3).clone()
    ex = tag.to(torch.complex128)[:, None, None].expand(len(pos), 2, 3).clone()
    if accumulate is not None:
        acc = np.asarray(accumulate)
        out = torch.zeros((int(acc.max()) + 1, 2, 3), dtype=torch.float64)
        for b in range(len(pos)):
            out[acc[b]] += dp[b]
        dp = out
    return ex, dp, None


def _scan_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from wideanglepropagation_b200.distributed import sharded_differentiable, sharded_simulate_fresnel_as
        P, D = 7, 3                              # 7 positions x 3 draws, draw-major
        pos = np.array([[i, 3 * i] for i in range(P)] * D)
        draw = np.repeat(np.arange(D), P)
        res = {}
        dp, ex = sharded_simulate_fresnel_as(None, None, None, 1.0, 1.0, positions=pos, draw=draw,
                                             return_exit=True, forward=_tag_forward)
        res["plain"] = (dp.numpy(), ex.numpy())
        acc = np.arange(P * D) % P
        dpa, _ = sharded_simulate_fresnel_as(None, None, None, 1.0, 1.0, positions=pos, draw=draw, accumulate=acc,
                                             forward=_tag_forward)
        res["acc"] = dpa.numpy()
        loc, _, first = sharded_simulate_fresnel_as(None, None, None, 1.0, 1.0, positions=pos, draw=draw,
                                                    gather=False, forward=_tag_forward)
        res["local"] = (first, loc.shape[0])

        # gradient: loss_r = sum over this rank's probes of tag_b * sum(V)
        def fwd(V, probe, H, dz, E, positions, draw=None, **kw):
            _, dp, _ = _tag_forward(None, None, None, dz, E, positions=positions, draw=draw)
            return None, dp * V.sum()

        V = torch.ones(2, 2, dtype=torch.float64, requires_grad=True)
        _, dpl, _ = sharded_differentiable(V, None, None, 1.0, 1.0, positions=pos, draw=draw, forward=fwd)
        dpl.sum().backward()
        res["grad"] = V.grad.numpy()
        q.put((rank, res))
    finally:
        dist.destroy_process_group()


def test_sharded_scan_gloo():
    """World size 2 over gloo: the real partition and reassembly logic of the
    sharded scan (probe blocks, pattern blocks with every probe of a pattern on
    one rank, the gather in order) and the all-reduced gradient, with a CPU
    stand-in forward that tags each probe's output."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    procs = [ctx.Process(target=_scan_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    res = dict(q.get(timeout=10) for _ in range(world))
    P, D = 7, 3
    pos = np.array([[i, 3 * i] for i in range(P)] * D)
    draw = np.repeat(np.arange(D), P)
    ref_ex, ref_dp, _ = _tag_forward(None, None, None, 1, 1, positions=pos, draw=draw)
    _, ref_acc, _ = _tag_forward(None, None, None, 1, 1, positions=pos, draw=draw, accumulate=np.arange(P * D) % P)
    total_tag = float(ref_dp[:, 0, 0].sum()) * 6
    for r in range(world):
        dp, ex = res[r]["plain"]
        assert np.array_equal(dp, ref_dp.numpy()) and np.array_equal(ex, ref_ex.numpy())
        assert np.array_equal(res[r]["acc"], ref_acc.numpy())
        assert np.allclose(res[r]["grad"], total_tag)
    assert res[0]["local"] == (0, 11) and res[1]["local"] == (11, 10)


@pytest.mark.parametrize("B,world", [(21, 2), (1088, 8), (9, 4)])
def test_probe_shard_accumulate_keeps_patterns_whole(B, world):
    from wideanglepropagation_b200.distributed import probe_shard
    P = max(1, B // 3)
    acc = np.arange(B) % P
    seen = []
    for r in range(world):
        mine, first, count = probe_shard(B, r, world, acc)
        assert set(acc[mine]) <= set(range(first, first + count))
        seen += list(mine)
    assert sorted(seen) == list(range(B))
