"""Persistent batched scheduler (wap_scan_*): same results as the per-pass
path and the FP64 oracle, CUDA-graph replay, and bounded waits that report
a timeout instead of hanging (failure injected from the host)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from wideanglepropagation_b200 import _lib  # noqa: E402
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wap():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import wideanglepropagation_b200 as w
    return w


def _classes(wap, spec, seed=0):
    from wideanglepropagation_b200.scan import to_device_class
    S = wap.synthetic
    return [to_device_class(S.batched_scan_class(seed + i, n, ns, side, draws)) for i, (n, ns, side, draws) in enumerate(spec)]


def _run(wap, classes, mode, groups=None):
    from wideanglepropagation_b200.scan import BatchedScan
    sc = BatchedScan(classes, mode=mode, groups=groups)
    sc.step()
    torch.cuda.synchronize()
    if sc.sched is not None:
        assert sc.sched.status() == 0
    return [c.exit.clone() for c in classes], [c.dp.clone() for c in classes], sc


def rel(a, b):
    a = a.double() if not a.is_complex() else a.to(torch.complex128)
    b = b.double() if not b.is_complex() else b.to(torch.complex128)
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.mark.parametrize("spec", [
    [(128, 5, 4, 2), (256, 4, 2, 1)],          # uneven: two sizes, draws
    [(512, 3, 2, 1)],
    [(1024, 2, 1, 2)],
    [(256, 6, 3, 1), (128, 3, 2, 1), (512, 2, 1, 1)],
])
def test_persistent_matches_per_pass(wap, spec):
    """Same math as the per-pass kernels; the scheduler may use a different
    radix plan (elements per thread), so results agree to float32 FFT
    rounding (2e-6), not bit for bit."""
    classes = _classes(wap, spec)
    ex_b, dp_b, _ = _run(wap, classes, "batched")
    ex_p, dp_p, _ = _run(wap, classes, "persistent")
    for a, b in zip(ex_p, ex_b):
        assert rel(a, b) < 2e-6
    for a, b in zip(dp_p, dp_b):
        assert rel(a, b) < 2e-6


def test_persistent_vs_oracle_and_groups(wap):
    from oracle import propagation_oracle as O
    spec = [(256, 6, 3, 2), (128, 4, 2, 1)]
    classes = _classes(wap, spec, seed=3)
    host = [wap.synthetic.batched_scan_class(3 + i, *s) for i, s in enumerate(spec)]
    ex, dp, _ = _run(wap, classes, "persistent", groups=[5, 3])   # groups that do not divide B
    for c, w, e, d in zip(classes, host, ex, dp):
        H = O.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
        for b in (0, c.n_probes // 2, c.n_probes - 1):
            p0 = O.move_probe(w.probe, tuple(w.positions[b]))
            rex, rdp, _ = O.simulate_fresnel_as(w.potential[w.draw_of_probe[b]], p0, H, w.dz, w.energy,
                                                return_wavefronts=False)
            assert O.rel_l2(e[b].cpu().numpy(), rex) < 1e-5
            assert O.rel_l2(d[b].cpu().numpy(), rdp) < 1e-5


def test_graph_replay_is_repeatable(wap):
    from wideanglepropagation_b200.scan import BatchedScan
    classes = _classes(wap, [(256, 4, 4, 1), (512, 2, 2, 1)])
    sc = BatchedScan(classes, mode="persistent")
    sc.capture()
    sc.graph.replay()
    torch.cuda.synchronize()
    first = [c.dp.clone() for c in classes]
    for c in classes:
        c.dp.zero_()
    sc.graph.replay()
    torch.cuda.synchronize()
    assert sc.sched.status() == 0
    for a, c in zip(first, classes):
        assert torch.equal(a, c.dp)


def test_bounded_wait_reports_timeout(wap):
    """A dependency that nothing satisfies (set from the host) makes the
    bounded waits expire: the run returns WAP_ERR_TIMEOUT and the context stays
    usable for the next, normal run."""
    from wideanglepropagation_b200 import _lib
    from wideanglepropagation_b200.scan import BatchedScan
    classes = _classes(wap, [(128, 3, 2, 1)])
    ref_ex, _, _ = _run(wap, classes, "batched")
    sc = BatchedScan(classes, mode="persistent")
    sc.sched.debug_stall(1, 1 << 12)
    sc.sched.run()
    torch.cuda.synchronize()
    assert sc.sched.status() == _lib.WAP_ERR_TIMEOUT
    sc.sched.debug_stall(-1, 0)
    sc.sched.run()
    torch.cuda.synchronize()
    assert sc.sched.status() == 0
    assert rel(classes[0].exit, ref_ex[0]) < 2e-6


def test_scan_rejects_unsupported(wap):
    from wideanglepropagation_b200.scan import PersistentScan
    classes = _classes(wap, [(128, 2, 1, 1)])
    classes[0].ny = classes[0].nx = 64
    with pytest.raises(ValueError, match="128, 256, 512 or 1024"):
        PersistentScan(classes)


@pytest.mark.parametrize("n_slices,table", [(160, "hi"), (161, "full")])
def test_twiddle_table_gate(wap, n_slices, table):
    """Scans of at most 160 slices run the hi-only stage-twiddle table, longer
    ones hi + lo: the default run reproduces the forced table bit for bit on
    each side of the gate, and both tables stay within 1e-5 of the FP64 oracle."""
    from oracle import propagation_oracle as O
    L = _lib.lib()
    spec = [(128, n_slices, 3, 1)]
    host = wap.synthetic.batched_scan_class(5, *spec[0])
    H = O.angular_spectrum_propagation_kernel(host.ny, host.nx, (host.ps, host.ps), host.dz, host.energy)
    p0 = O.move_probe(host.probe, tuple(host.positions[0]))
    rex, _, _ = O.simulate_fresnel_as(host.potential[0], p0, H, host.dz, host.energy, return_wavefronts=False)
    ex_default, _, _ = _run(wap, _classes(wap, spec, seed=5), "persistent")
    out = {}
    try:
        for forced, knob in (("hi", _lib.WAP_TW_HI), ("full", _lib.WAP_TW_FULL)):
            _lib.check(L.wap_scan_debug_override(_lib.WAP_KNOB_TWIDDLES, knob))
            out[forced], _, _ = _run(wap, _classes(wap, spec, seed=5), "persistent")
            assert O.rel_l2(out[forced][0][0].cpu().numpy(), rex) < 1e-5
    finally:
        _lib.check(L.wap_scan_debug_override(_lib.WAP_KNOB_TWIDDLES, -1))
    assert torch.equal(ex_default[0], out[table][0])
    other = "full" if table == "hi" else "hi"
    assert not torch.equal(ex_default[0], out[other][0])


def test_scheduler_ignores_environment(wap, monkeypatch):
    """The scheduler's choices come from the library and explicit overrides
    only: variables in the environment change nothing."""
    spec = [(128, 4, 8, 1)]
    ex_default, _, _ = _run(wap, _classes(wap, spec, seed=7), "persistent")
    for k, v in (("WAP_SCHED_TW", "full"), ("WAP_SCHED_E", "8"), ("WAP_SCHED_GROUP", "3"),
                 ("WAP_SCHED_TWIDDLES", "global")):
        monkeypatch.setenv(k, v)
    ex_env, _, _ = _run(wap, _classes(wap, spec, seed=7), "persistent")
    assert torch.equal(ex_default[0], ex_env[0])


def test_api_raises_on_scheduler_timeout(wap):
    """simulate_fresnel_as on the persistent scheduler raises WapError when a
    bounded wait expires (a dependency nothing satisfies, short spin limit),
    defers it with check=False until check_errors(), and the next call
    succeeds with the FP64 oracle's result."""
    from oracle import propagation_oracle as O
    from wideanglepropagation_b200 import propagation as P
    host = wap.synthetic.batched_scan_class(3, 128, 4, 8, 1)
    H = wap.angular_spectrum_propagation_kernel(128, 128, (host.ps, host.ps), host.dz, host.energy)
    args = (host.potential[0], host.probe, H, host.dz, host.energy)
    kw = dict(positions=host.positions, return_wavefronts=False)
    ex0, _, _ = wap.simulate_fresnel_as(*args, **kw)
    torch.cuda.synchronize()
    key = (torch.cuda.current_device(), 128, host.n_slices, 1, host.n_probes)
    h, _ = P._scans[key]   # (scan handle, StreamOrder)
    L = _lib.lib()
    try:
        _lib.check(L.wap_scan_debug_stall(h, 1, 1 << 12))
        with pytest.raises(_lib.WapError, match="bounded device-side wait expired"):
            wap.simulate_fresnel_as(*args, **kw)
        wap.simulate_fresnel_as(*args, check=False, **kw)   # returns without waiting
        with pytest.raises(_lib.WapError, match="bounded device-side wait expired"):
            wap.check_errors()
        wap.check_errors()   # consumed
    finally:
        _lib.check(L.wap_scan_debug_stall(h, -1, 0))
    ex1, _, _ = wap.simulate_fresnel_as(*args, **kw)
    assert torch.equal(ex0, ex1)
    p0 = O.move_probe(host.probe, tuple(host.positions[5]))
    rex, _, _ = O.simulate_fresnel_as(host.potential[0], p0, H.cpu().numpy(), host.dz, host.energy,
                                      return_wavefronts=False)
    assert O.rel_l2(ex1[5].cpu().numpy(), rex) < 1e-5


def test_autograd_raises_on_scheduler_timeout(wap):
    """The differentiable path on the persistent scheduler raises WapError in
    the forward when a bounded wait expires, and works again afterwards."""
    from wideanglepropagation_b200 import autograd as A
    host = wap.synthetic.batched_scan_class(4, 128, 4, 8, 1)
    H = wap.angular_spectrum_propagation_kernel(128, 128, (host.ps, host.ps), host.dz, host.energy)
    V = torch.tensor(host.potential[0], device="cuda", requires_grad=True)

    def step():
        ex, dp = A.simulate_fresnel_as_differentiable(V, host.probe, H, host.dz, host.energy,
                                                      positions=host.positions, ckpt_every=2)
        dp.sum().backward()
        g = V.grad.clone()
        V.grad = None
        return g

    g0 = step()
    torch.cuda.synchronize()
    key = (torch.cuda.current_device(), 128, host.n_slices, 1, host.n_probes, 2)
    h, _ = A._pool[key][-1]   # (scan handle, StreamOrder)
    L = _lib.lib()
    try:
        _lib.check(L.wap_scan_debug_stall(h, 1, 1 << 12))
        with pytest.raises(_lib.WapError, match="bounded device-side wait expired"):
            step()
    finally:
        _lib.check(L.wap_scan_debug_stall(h, -1, 0))
    g1 = step()
    assert torch.allclose(g0, g1, rtol=1e-5, atol=1e-6 * float(g0.abs().max()))


def test_automatic_groups_are_balanced(wap):
    """With group 0 the library picks about 4 x the resident CTAs in tiles and
    evens it out over the batch: 64 probes on 512^2 (nominal 28 on 148 SMs)
    run as two groups of 32."""
    from wideanglepropagation_b200.scan import PersistentScan
    classes = _classes(wap, [(512, 2, 8, 1)])
    assert classes[0].n_probes == 64
    info = PersistentScan(classes, [0]).info()
    nominal = -(-4 * info["grid"] // (512 * 512 // 4096))
    ng = max(1, (64 + nominal // 2) // nominal)
    assert info["group0"] == -(-64 // ng)
    if info["grid"] == 444:
        assert info["group0"] == 32
