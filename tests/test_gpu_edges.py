"""Edge cases of the drop-in API on the device: empty inputs, the largest
grid, probe positions that wrap the grid edges on both execution paths,
odd batch sizes around the scheduler's threshold, and one slice."""
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


def _setup(n=128, N=3, seed=0):
    import wideanglepropagation_b200.synthetic as S
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.1, 2.0, 200e3
    V = (S.random_gaussian_stack(rng, N, n, n, ps, 8, 20.0, 0.3) / dz).astype(np.float32)
    probe = S.aperture_probe(n, n, ps, E, 20.0, -30.0, dtype=np.complex64)
    return V, probe, ps, dz, E


def test_empty_inputs_raise(wap):
    V, probe, ps, dz, E = _setup(64, 2)
    H = wap.fresnel_propagation_kernel(64, 64, (ps, ps), dz, E)
    with pytest.raises(ValueError):
        wap.simulate_fresnel_as(V[:0], probe, H, dz, E)                      # no slices
    with pytest.raises(ValueError):
        wap.simulate_fresnel_as(V, probe, H, dz, E, positions=np.zeros((0, 2), np.int32))   # no probes
    with pytest.raises(ValueError):
        wap.simulate_fresnel_as(V, probe[:, :32], H, dz, E)                  # probe / potential grids differ
    with pytest.raises(ValueError):
        wap.simulate_fresnel_as(V, probe, H[:32], dz, E)                     # transfer function grid differs


def test_largest_grid_single_probe(wap):
    """2048^2, the largest grid of the transform kernels, against the FP64 oracle."""
    from oracle import propagation_oracle as O
    n, N = 2048, 2
    V, probe, ps, dz, E = _setup(n, N, seed=3)
    H = wap.angular_spectrum_propagation_kernel(n, n, (ps, ps), dz, E)
    ex, dp, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=False)
    rex, rdp, _ = O.simulate_fresnel_as(V.astype(np.float64), probe, H.cpu().numpy(), dz, E, return_wavefronts=False)
    assert O.rel_l2(ex.cpu().numpy(), rex) < 1e-5
    assert O.rel_l2(dp.cpu().numpy(), rdp) < 1e-5


@pytest.mark.parametrize("B", [7, 8, 9])   # around the scheduler's threshold (8 probes)
def test_wrapping_positions_both_paths(wap, B):
    """Positions at and beyond the grid edges wrap like the reference's
    jnp.roll (move_probe); 7 probes run the per-pass kernels, 8 and 9 the
    persistent scheduler; every probe must equal its own single-probe run."""
    from oracle import propagation_oracle as O
    n = 128
    V, probe, ps, dz, E = _setup(n, 3, seed=1)
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    edge = np.array([[0, 0], [n - 1, n - 1], [0, n - 1], [n - 1, 0], [1, 64], [64, 127], [127, 1], [63, 0],
                     [5, 5]], np.int32)[:B]
    ex, dp, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, positions=edge, return_wavefronts=False)
    Ho = H.cpu().numpy()
    for b in range(B):
        p0 = O.move_probe(probe.astype(np.complex128), tuple(edge[b]))
        rex, rdp, _ = O.simulate_fresnel_as(V.astype(np.float64), p0, Ho, dz, E, return_wavefronts=False)
        assert O.rel_l2(ex[b].cpu().numpy(), rex) < 1e-5, b
        assert O.rel_l2(dp[b].cpu().numpy(), rdp) < 1e-5, b


def test_one_slice(wap):
    from oracle import propagation_oracle as O
    V, probe, ps, dz, E = _setup(256, 1, seed=2)
    H = wap.fresnel_propagation_kernel(256, 256, (ps, ps), dz, E)
    pos = np.array([[128, 128]] * 8 + [[3, 250]] * 8, np.int32)             # 16 probes: scheduler, one slice
    ex, dp, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, positions=pos, return_wavefronts=False)
    for b in (0, 15):
        p0 = O.move_probe(probe.astype(np.complex128), tuple(pos[b]))
        rex, _, _ = O.simulate_fresnel_as(V.astype(np.float64), p0, H.cpu().numpy(), dz, E, return_wavefronts=False)
        assert O.rel_l2(ex[b].cpu().numpy(), rex) < 1e-5


def test_release_caches_frees_and_recovers(wap):
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    V, probe, ps, dz, E = _setup(128, 3, seed=4)
    H = wap.fresnel_propagation_kernel(128, 128, (ps, ps), dz, E)
    pos = np.array([[i * 8, 100 - i * 5] for i in range(12)], np.int32)
    ex0, _, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, positions=pos, return_wavefronts=False)
    Vt = torch.tensor(V, device="cuda", requires_grad=True)
    _, dp = simulate_fresnel_as_differentiable(Vt, probe, H, dz, E, positions=pos)
    dp.sum().backward()
    g0 = Vt.grad.clone()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    wap.release_caches()
    assert torch.cuda.mem_get_info()[0] >= free0      # plans, scans and pooled gradient scans gone
    ex1, _, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, positions=pos, return_wavefronts=False)
    assert torch.equal(ex0, ex1)                      # rebuilt on demand, same numbers
    Vt.grad = None
    _, dp = simulate_fresnel_as_differentiable(Vt, probe, H, dz, E, positions=pos)
    dp.sum().backward()
    assert float((Vt.grad - g0).norm() / g0.norm()) < 1e-6


def test_fp32_probe_computes_its_chains(wap):
    """The roofline's FMA probe does the arithmetic it is credited with: each
    thread's 8 chains a <- a x + y, summed, match a float64 evaluation."""
    import ctypes
    from wideanglepropagation_b200 import _lib
    blocks, iters = 2, 64
    out = torch.empty(blocks * 256, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib().wap_fp32_probe(blocks, iters, ctypes.c_void_p(out.data_ptr()),
                                         ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    x, y = np.float64(np.float32(0.999999)), np.float64(np.float32(1e-6))
    a = (np.float64(np.float32(1e-3)) * np.arange(256)[:, None]).astype(np.float32).astype(np.float64) + np.arange(8)
    for _ in range(iters):
        a = a * x + y
    ref = np.tile(a.sum(axis=1), blocks)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-5)
    with pytest.raises(ValueError):
        _lib.check(_lib.lib().wap_fp32_probe(0, iters, ctypes.c_void_p(out.data_ptr()), None))


def test_transfer_split_cache_follows_changes(wap):
    """A complex128 transfer function on the device is split into hi + lo once
    and reused; an in-place change of it must not reuse the stale split."""
    rng = np.random.default_rng(5)
    n = 64
    V = torch.tensor(rng.uniform(0, 30, (3, n, n)).astype(np.float32), device="cuda")
    psi = torch.tensor((rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))).astype(np.complex64), device="cuda")
    H = wap.angular_spectrum_propagation_kernel(n, n, (0.05, 0.05), 2.0, 300e3)
    assert H.dtype == torch.complex128 and H.is_cuda
    e1, _, _ = wap.simulate_fresnel_as(V, psi, H, 2.0, 300e3, return_wavefronts=False)
    e2, _, _ = wap.simulate_fresnel_as(V, psi, H, 2.0, 300e3, return_wavefronts=False)
    assert torch.equal(e1, e2)
    H.mul_(torch.exp(1j * torch.linspace(0, 1, n * n, dtype=torch.float64, device="cuda")).reshape(n, n))
    e3, _, _ = wap.simulate_fresnel_as(V, psi, H, 2.0, 300e3, return_wavefronts=False)
    e4, _, _ = wap.simulate_fresnel_as(V, psi, H.clone(), 2.0, 300e3, return_wavefronts=False)
    assert torch.equal(e3, e4)
    assert not torch.equal(e1, e3)


def test_inference_mode_complex128_transfer(wap):
    """Calls under torch.inference_mode() with a complex128 device transfer
    function (an inference tensor, which has no version counter) work and give
    the same result as outside it, on the per-pass path, the scheduler path and
    the WPM line-transfer helper."""
    V, probe, ps, dz, E = _setup(128, 3, seed=2)
    pos = np.array([[64, 64], [10, 20], [100, 5], [3, 3], [64, 0], [0, 64], [127, 127], [50, 90]], np.int32)
    H0 = wap.angular_spectrum_propagation_kernel(128, 128, (ps, ps), dz, E)
    ref1 = wap.simulate_fresnel_as(V, probe, H0, dz, E, return_wavefronts=False)[0]
    ref8 = wap.simulate_fresnel_as(V, probe, H0, dz, E, positions=pos, return_wavefronts=False)[0]
    with torch.inference_mode():
        H = wap.angular_spectrum_propagation_kernel(128, 128, (ps, ps), dz, E)
        assert H.dtype == torch.complex128 and H.is_inference()
        for _ in range(2):   # a second call would hit a cache entry if one had been made
            ex1 = wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=False)[0]
            ex8 = wap.simulate_fresnel_as(V, probe, H, dz, E, positions=pos, return_wavefronts=False)[0]
            assert torch.equal(ex1, ref1) and torch.equal(ex8, ref8)
        kp2 = torch.rand(128, 128, dtype=torch.float64, device="cuda")
        X = torch.randn(128, 128, dtype=torch.complex64, device="cuda")
        out = wap.wpm_propagation_kernel_vmap(X, [1.0, 1.0001], 50.0, kp2, 2.0)
    assert torch.equal(out, wap.wpm_propagation_kernel_vmap(X, [1.0, 1.0001], 50.0, kp2, 2.0))


def test_transfer_split_cache_other_stream(wap):
    """A cached complex128 transfer-function split made on one stream is used
    correctly from another stream (the consumer waits for the split)."""
    V, probe, ps, dz, E = _setup(128, 3, seed=4)
    H = wap.angular_spectrum_propagation_kernel(128, 128, (ps, ps), dz, E)
    ref = wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=False)[0]
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        ex = wap.simulate_fresnel_as(V, probe, H, dz, E, return_wavefronts=False)[0]
    torch.cuda.current_stream().wait_stream(s)
    assert torch.equal(ex, ref)
