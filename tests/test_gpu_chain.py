"""One-launch chain of a single probe (cooperative kernel, grid-wide barriers
between the passes): against the FP64 oracle and against the per-pass path
(one launch per pass, forced through wap_scan_debug_override), on every chain
size, with two probes, the wavefront stack and a detector window.  The
cluster kernel, which serves 128^2 and 256^2 by default, is switched off for
these tests.

Tolerance: rel-L2 <= 1e-5 against the oracle; the chain and the per-pass
launches may use different elements per thread (FFT radix plans), so they
agree to float32 FFT rounding (2e-6), not bit for bit.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
from wideanglepropagation_b200 import _lib  # noqa: E402

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def wap():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import wideanglepropagation_b200 as w
    # 128^2 / 256^2 probes take the cluster kernel by default: off here, so
    # that these sizes reach the chain
    L = _lib.lib()
    _lib.check(L.wap_scan_debug_override(_lib.WAP_KNOB_CLUSTER, 0))
    yield w
    _lib.check(L.wap_scan_debug_override(_lib.WAP_KNOB_CLUSTER, -1))


def rel(a, b):
    from oracle.propagation_oracle import rel_l2
    return rel_l2(a, b)


def _setup(n, N, seed):
    import wideanglepropagation_b200.synthetic as S
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.05 if n >= 512 else 0.1, 2.0, 200e3
    V = (S.random_gaussian_stack(rng, N, n, n, ps, 12, 20.0, 0.3) / dz).astype(np.float32)
    probe = S.aperture_probe(n, n, ps, E, 20.0, -30.0, dtype=np.complex64)
    return V, probe, ps, dz, E


def _per_pass(fn):
    L = _lib.lib()
    _lib.check(L.wap_scan_debug_override(_lib.WAP_KNOB_CHAIN, 0))
    try:
        return fn()
    finally:
        _lib.check(L.wap_scan_debug_override(_lib.WAP_KNOB_CHAIN, -1))


@pytest.mark.parametrize("n,N,elems", [(128, 9, 0), (256, 20, 0), (256, 8, 8), (512, 12, 4), (1024, 6, 8),
                                       (2048, 3, 16)])
def test_chain_single_probe(wap, n, N, elems):
    """elems = 0: the default (128^2 and 256^2 run the chain); otherwise the
    chain forced on with that many elements per thread (the A/B override,
    which also reaches the larger grids)."""
    from oracle import propagation_oracle as O
    V, probe, ps, dz, E = _setup(n, N, seed=n)
    H = wap.angular_spectrum_propagation_kernel(n, n, (ps, ps), dz, E)
    call = lambda: wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=(n <= 512))
    L = _lib.lib()
    if elems:
        _lib.check(L.wap_scan_debug_override(_lib.WAP_KNOB_CHAIN, elems))
    try:
        l0 = _lib.launch_count()
        ex, dp, st = call()
        torch.cuda.synchronize()
        launches = _lib.launch_count() - l0
    finally:
        _lib.check(L.wap_scan_debug_override(_lib.WAP_KNOB_CHAIN, -1))
    assert launches <= 2, launches   # transmission table + the chain kernel
    pex, pdp, pst = _per_pass(call)
    rex, rdp, rst = O.simulate_fresnel_as(V.astype(np.float64), probe, H.cpu().numpy(), dz, E,
                                          return_wavefronts=(n <= 512))
    assert rel(ex.cpu().numpy(), rex) < TOL
    assert rel(dp.cpu().numpy(), rdp) < TOL
    assert rel(ex.cpu().numpy(), pex.cpu().numpy()) < 2e-6
    if st is not None:
        assert rel(st.cpu().numpy(), rst) < TOL
        assert rel(st.cpu().numpy(), pst.cpu().numpy()) < 2e-6


def test_chain_two_probes_window(wap):
    """Two probes (positions and potential draws) with a detector window."""
    from oracle import propagation_oracle as O
    n = 256
    V0, probe, ps, dz, E = _setup(n, 7, seed=5)
    V1, _, _, _, _ = _setup(n, 7, seed=6)
    V = np.stack([V0, V1])
    pos = np.array([[10, 250], [128, 3]], np.int32)
    draw = np.array([1, 0], np.int32)
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    kw = dict(positions=pos, draw=draw, return_wavefronts=False, max_angle=40.0, sampling=(ps, ps))
    ex, dp, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, **kw)
    pex, pdp, _ = _per_pass(lambda: wap.simulate_fresnel_as(V, probe, H, dz, E, **kw))
    lam = O.energy2wavelength(E)
    for b in range(2):
        rex, rdp, _ = O.simulate_fresnel_as(V[draw[b]].astype(np.float64), O.move_probe(probe, tuple(pos[b])),
                                            H.cpu().numpy(), dz, E, return_wavefronts=False)
        assert rel(ex[b].cpu().numpy(), rex) < TOL
        assert rel(dp[b].cpu().numpy(), O.downsample_to_max_angle(rdp, (ps, ps), lam, 40.0)) < TOL
    assert rel(dp.cpu().numpy(), pdp.cpu().numpy()) < 2e-6


def test_chain_deferred_status_is_clean(wap):
    """check=False defers the chain's status to check_errors(), which finds
    no failure; repeated calls give identical results."""
    V, probe, ps, dz, E = _setup(256, 5, seed=8)
    H = wap.angular_spectrum_propagation_kernel(256, 256, (ps, ps), dz, E)
    outs = [wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=False, check=False)[0] for _ in range(3)]
    wap.check_errors()
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[1], outs[2])
