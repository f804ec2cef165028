"""Calls issued on different CUDA streams without synchronising in between.

The library keeps device workspace between calls in cached objects (plans:
transmission tables, chain counters, WPM fields; persistent scans: tables,
work queues, status words; pooled gradient scans).  Two calls of the same
shape issued back to back on two streams share that workspace; each cached
object therefore remembers the stream of its last use, and a use from another
stream first waits for what was issued there.  Every case here issues call A on one stream and call B
(same shapes, different inputs) on another stream at once, then compares both
results with the same calls run one after the other on one stream: the
kernels are the same, so the results must agree bit for bit (gradients, which
sum the probes' terms with atomics, to 1e-5 rel-L2).  The first call
of each pair is made long enough (slices, probes) that an unordered second
call would overlap it.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def wap():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import wideanglepropagation_b200 as w
    return w


def _inputs(n, N, D, seed):
    import wideanglepropagation_b200.synthetic as S
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.1, 2.0, 200e3
    V = np.stack([S.random_gaussian_stack(rng, N, n, n, ps, 12, 20.0, 0.3) for _ in range(D)])
    V = torch.from_numpy((V / dz).astype(np.float32)).cuda()
    probe = torch.from_numpy(S.aperture_probe(n, n, ps, E, 20.0, -30.0, dtype=np.complex64)).cuda()
    return V, probe, ps, dz, E


def _pair(fn, a, b):
    """fn(a), fn(b) on two streams issued back to back, and the same two calls
    on one stream one after the other."""
    torch.cuda.synchronize()
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    s1.wait_stream(torch.cuda.current_stream())
    s2.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s1):
        ra = fn(a)
    with torch.cuda.stream(s2):
        rb = fn(b)
    torch.cuda.synchronize()
    serial = (fn(a), fn(b))
    torch.cuda.synchronize()
    return (ra, rb), serial


def _same(x, y):
    for u, v in zip(x, y):
        if u is None:
            assert v is None
            continue
        assert torch.equal(u, v)


@pytest.mark.parametrize("n,B,N", [(128, 1, 40), (256, 2, 40), (256, 3, 30)])
def test_plan_paths_on_two_streams(wap, n, B, N):
    """Cluster (128^2, one probe), chain (256^2, two probes) and per-pass
    (three probes) forwards of one cached plan from two streams."""
    V, probe, ps, dz, E = _inputs(n, N, 1, 1)
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    rng = np.random.default_rng(2)
    pos = [torch.from_numpy(rng.integers(0, n, (B, 2)).astype(np.int32)).cuda() for _ in range(2)]
    Vs = [V[0], torch.flip(V[0], (0,)).contiguous()]

    def fn(i):
        ex, dp, _ = wap.simulate_fresnel_as(Vs[i], probe, H, dz, E, positions=pos[i], return_wavefronts=False)
        return ex, dp

    (ra, rb), (sa, sb) = _pair(fn, 0, 1)
    _same(ra, sa)
    _same(rb, sb)
    assert not torch.equal(sa[1], sb[1])


def test_persistent_scan_on_two_streams(wap):
    """Two batched scans of the same shape (one cached persistent scan) from two streams."""
    n, N, B = 256, 24, 64
    V, probe, ps, dz, E = _inputs(n, N, 2, 3)
    H = wap.angular_spectrum_propagation_kernel(n, n, (ps, ps), dz, E)
    rng = np.random.default_rng(4)
    pos = torch.from_numpy(rng.integers(0, n, (B, 2)).astype(np.int32)).cuda()
    draw = torch.from_numpy((np.arange(B) % 2).astype(np.int32)).cuda()
    Vs = [V, torch.flip(V, (0,)).contiguous()]

    def fn(i):
        ex, dp, _ = wap.simulate_fresnel_as(Vs[i], probe, H, dz, E, positions=pos, draw=draw,
                                            return_wavefronts=False)
        return ex, dp

    (ra, rb), (sa, sb) = _pair(fn, 0, 1)
    _same(ra, sa)
    _same(rb, sb)
    assert not torch.equal(sa[1], sb[1])


def test_wpm_on_two_streams(wap):
    n, N = 128, 12
    V, probe, ps, dz, E = _inputs(n, N, 1, 5)
    Vs = [V[0], 1.5 * V[0]]

    def fn(i):
        ex, dp, st = wap.simulate_wpm(Vs[i], probe, dz, E, (ps, ps), n_bins=8, power_spacing=1.0)
        return ex, dp, st

    (ra, rb), (sa, sb) = _pair(fn, 0, 1)
    _same(ra, sa)
    _same(rb, sb)


def test_gradient_scans_on_two_streams(wap):
    """Forward + backward of the differentiable multislice (pooled gradient
    scans, persistent scheduler) on two streams."""
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable as diff
    n, N, B = 128, 12, 16
    V, probe, ps, dz, E = _inputs(n, N, 1, 6)
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    rng = np.random.default_rng(7)
    pos = torch.from_numpy(rng.integers(0, n, (B, 2)).astype(np.int32)).cuda()
    Vs = [V[0], torch.flip(V[0], (1,)).contiguous()]

    def fn(i):
        x = Vs[i].clone().requires_grad_(True)
        _, dp = diff(x, probe, H, dz, E, positions=pos, ckpt_every=4)
        (dp * dp).sum().backward()
        return dp.detach(), x.grad

    (ra, rb), (sa, sb) = _pair(fn, 0, 1)
    # the patterns bit for bit; the gradients sum the probes' terms with
    # atomics (order-dependent rounding)
    for r, s_ in ((ra, sa), (rb, sb)):
        assert torch.equal(r[0], s_[0])
        err = float(torch.linalg.vector_norm(r[1] - s_[1]) / torch.linalg.vector_norm(s_[1]))
        assert err <= 1e-5, err
