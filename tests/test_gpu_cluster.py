"""Cluster-resident multislice of single probes (the wave in the distributed
shared memory of one 16-CTA thread-block cluster per probe, one launch for all
slices): against the FP64 oracle and against the per-pass path (one launch per
pass, forced through wap_scan_debug_override), on 128^2 (the default) and
256^2 (through the override), with the wavefront stack, two probes with
positions and potential draws, a detector window, and every
elements-per-thread variant.

Tolerance: rel-L2 <= 1e-5 against the oracle; the cluster kernel and the
per-pass launches may use different elements per thread (FFT radix plans), so
they agree to float32 FFT rounding (2e-6), not bit for bit.
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
    return w


def rel(a, b):
    from oracle.propagation_oracle import rel_l2
    return rel_l2(a, b)


def _setup(n, N, seed):
    import wideanglepropagation_b200.synthetic as S
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.1, 2.0, 200e3
    V = (S.random_gaussian_stack(rng, N, n, n, ps, 12, 20.0, 0.3) / dz).astype(np.float32)
    probe = S.aperture_probe(n, n, ps, E, 20.0, -30.0, dtype=np.complex64)
    return V, probe, ps, dz, E


def _with(knobs, fn):
    L = _lib.lib()
    for k, v in knobs.items():
        _lib.check(L.wap_scan_debug_override(k, v))
    try:
        return fn()
    finally:
        for k in knobs:
            _lib.check(L.wap_scan_debug_override(k, -1))


PER_PASS = {_lib.WAP_KNOB_CLUSTER: 0, _lib.WAP_KNOB_CHAIN: 0}


@pytest.mark.parametrize("n,N,elems", [(128, 12, 0), (128, 7, 4), (256, 20, 16), (256, 9, 8)])
def test_cluster_single_probe(wap, n, N, elems):
    """elems = 0: the default (128^2 runs the cluster kernel); otherwise that
    many elements per thread through the override, which also reaches 256^2."""
    from oracle import propagation_oracle as O
    V, probe, ps, dz, E = _setup(n, N, seed=n + N)
    H = wap.angular_spectrum_propagation_kernel(n, n, (ps, ps), dz, E)
    call = lambda: wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=True)

    def counted():
        l0 = _lib.launch_count()
        out = call()
        torch.cuda.synchronize()
        return out, _lib.launch_count() - l0
    (ex, dp, st), launches = _with({_lib.WAP_KNOB_CLUSTER: elems} if elems else {}, counted)
    assert launches <= 2, launches   # transmission table + the cluster kernel
    pex, pdp, pst = _with(PER_PASS, call)
    rex, rdp, rst = O.simulate_fresnel_as(V.astype(np.float64), probe, H.cpu().numpy(), dz, E,
                                          return_wavefronts=True)
    assert rel(ex.cpu().numpy(), rex) < TOL
    assert rel(dp.cpu().numpy(), rdp) < TOL
    assert rel(st.cpu().numpy(), rst) < TOL
    assert rel(ex.cpu().numpy(), pex.cpu().numpy()) < 2e-6
    assert rel(st.cpu().numpy(), pst.cpu().numpy()) < 2e-6


@pytest.mark.parametrize("n,elems", [(128, 0), (256, 16)])
def test_cluster_two_probes_draws_window(wap, n, elems):
    """Two probes with positions and potential draws, a detector window, the
    Fresnel propagator, no stack."""
    from oracle import propagation_oracle as O
    V0, probe, ps, dz, E = _setup(n, 6, seed=11)
    V1, _, _, _, _ = _setup(n, 6, seed=12)
    V = np.stack([V0, V1])
    pos = np.array([[3, n - 6], [n // 2 + 2, 64]], np.int32)
    draw = np.array([1, 0], np.int32)
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    kw = dict(positions=pos, draw=draw, return_wavefronts=False, max_angle=40.0, sampling=(ps, ps))
    ex, dp, _ = _with({_lib.WAP_KNOB_CLUSTER: elems} if elems else {},
                      lambda: wap.simulate_fresnel_as(V, probe, H, dz, E, **kw))
    pex, pdp, _ = _with(PER_PASS, lambda: wap.simulate_fresnel_as(V, probe, H, dz, E, **kw))
    lam = O.energy2wavelength(E)
    for b in range(2):
        rex, rdp, _ = O.simulate_fresnel_as(V[draw[b]].astype(np.float64), O.move_probe(probe, tuple(pos[b])),
                                            H.cpu().numpy(), dz, E, return_wavefronts=False)
        assert rel(ex[b].cpu().numpy(), rex) < TOL
        assert rel(dp[b].cpu().numpy(), O.downsample_to_max_angle(rdp, (ps, ps), lam, 40.0)) < TOL
    assert rel(dp.cpu().numpy(), pdp.cpu().numpy()) < 2e-6


def test_cluster_repeatable(wap):
    """Repeated calls (the plan's cached table and fit check) give identical
    results; the chain kernel, forced, agrees."""
    V, probe, ps, dz, E = _setup(128, 5, seed=3)
    H = wap.angular_spectrum_propagation_kernel(128, 128, (ps, ps), dz, E)
    outs = [wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=False)[0] for _ in range(3)]
    assert torch.equal(outs[0], outs[1]) and torch.equal(outs[1], outs[2])
    chain = _with({_lib.WAP_KNOB_CLUSTER: 0},
                  lambda: wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=False)[0])
    assert rel(outs[0].cpu().numpy(), chain.cpu().numpy()) < 2e-6


def test_refused_cluster_launch_falls_back_to_chain(wap):
    """A cluster launch that the device refuses (injected on the host: knob
    value 1 makes the call treat the launch as refused without issuing it)
    leaves no error behind: the call runs on the chain kernel, bit for bit the
    chain's result, and so does every later call of that plan."""
    V, probe, ps, dz, E = _setup(128, 9, seed=21)
    H = wap.angular_spectrum_propagation_kernel(128, 128, (ps, ps), dz, E)
    call = lambda: wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=False)

    def counted():
        l0 = _lib.launch_count()
        out = call()
        torch.cuda.synchronize()
        return out, _lib.launch_count() - l0
    # whether the plan's last forward ran the chain kernel (it then has a status word to read)
    chain_ran = lambda: _lib.plan_status_pending(
        wap.propagation.get_plan(128, 128, 1, _lib.WAP_OP_FRESNEL_AS).handle)
    wap.release_caches()   # a plan of its own: the fallback is kept for the plan's life
    try:
        call()
        assert not chain_ran()   # the default: the cluster kernel
        (chain, _, _), _ = _with({_lib.WAP_KNOB_CLUSTER: 0}, counted)
        assert chain_ran()
        (ex, dp, _), launches = _with({_lib.WAP_KNOB_CLUSTER: 1}, counted)
        assert chain_ran()
        assert 1 <= launches <= 2, launches   # [transmission table +] the chain kernel, not the refused one
        assert torch.equal(ex, chain)
        (ex2, _, _), launches = counted()   # knob back to the default: the plan stays on the chain
        assert chain_ran()
        assert 1 <= launches <= 2, launches
        assert torch.equal(ex2, chain)
        wap.check_errors()
    finally:
        wap.release_caches()
