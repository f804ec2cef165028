"""Detector window fused into the diffraction epilogue.

``max_angle`` / ``sampling`` / ``parity`` make the last column pass store
only the centre crop that ``downsample_to_max_angle`` (propagation.py:424-439)
keeps.  The stored values are the same float32 numbers as the full pattern's,
so the fused crop must equal the crop of the full pattern exactly, on every
path that writes a pattern: the per-pass forward, the persistent scheduler,
WPM, and the adjoint seed of both gradient paths (where a loss on the cropped
pattern must give the gradient of the same loss on the full pattern's window).
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


def _case(n=128, N=5, n_side=4, seed=0):
    import wideanglepropagation_b200.synthetic as S
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.1, 2.0, 200e3
    V = (S.random_gaussian_stack(rng, N, n, n, ps, 12, 20.0, 0.3) / dz).astype(np.float32)
    probe = S.aperture_probe(n, n, ps, E, 20.0, 0.0, dtype=np.complex64)
    pos = S.raster_positions(n, n, n_side, n_side)
    return V, probe, pos, ps, dz, E


@pytest.mark.parametrize("parity", ["odd", "even"])
@pytest.mark.parametrize("angle", [30.0, 80.0])
def test_fused_crop_per_pass(wap, parity, angle):
    V, probe, pos, ps, dz, E = _case()
    n = V.shape[-1]
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    # return_wavefronts=True keeps the per-pass kernels
    _, dp_full, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, positions=pos[:3])
    ex, dp, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, positions=pos[:3], max_angle=angle, sampling=(ps, ps),
                                        parity=parity)
    ref = wap.downsample_to_max_angle(dp_full, (ps, ps), wap.energy2wavelength(E), angle, parity=parity)
    assert dp.shape == ref.shape and dp.shape[-1] < n
    assert torch.equal(dp, ref)


@pytest.mark.parametrize("parity", ["odd", "even"])
def test_fused_crop_persistent_scan(wap, parity):
    V, probe, pos, ps, dz, E = _case()
    n = V.shape[-1]
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    kw = dict(positions=pos, return_wavefronts=False)   # 16 probes, square: persistent scheduler
    _, dp_full, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, **kw)
    _, dp, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, max_angle=40.0, sampling=ps, parity=parity, **kw)
    ref = wap.downsample_to_max_angle(dp_full, (ps, ps), wap.energy2wavelength(E), 40.0, parity=parity)
    assert dp.shape == ref.shape
    assert torch.equal(dp, ref)
    # the cached scan is re-bound without a window afterwards
    _, dp_again, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, **kw)
    assert torch.equal(dp_again, dp_full)


def test_fused_crop_wpm(wap):
    V, probe, pos, ps, dz, E = _case(n=64, N=3)
    _, dp_full, _ = wap.simulate_wpm(V, probe, dz, E, (ps, ps), n_bins=8, power_spacing=1.0, positions=pos[:2])
    _, dp, _ = wap.simulate_wpm(V, probe, dz, E, (ps, ps), n_bins=8, power_spacing=1.0, positions=pos[:2],
                                max_angle=50.0)
    ref = wap.downsample_to_max_angle(dp_full, (ps, ps), wap.energy2wavelength(E), 50.0)
    assert dp.shape == ref.shape and dp.shape[-1] < 64
    assert torch.equal(dp, ref)


def test_window_covering_the_grid_is_no_crop(wap):
    V, probe, pos, ps, dz, E = _case(n=64, N=2)
    H = wap.fresnel_propagation_kernel(64, 64, (ps, ps), dz, E)
    _, dp, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, max_angle=1e6, sampling=ps)
    assert dp.shape == (64, 64)


@pytest.mark.parametrize("n_side", [2, 4])   # 4 probes: per-pass adjoint; 16: persistent gradient scan
def test_gradient_through_the_window(wap, n_side):
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    V, probe, pos, ps, dz, E = _case(n=128, N=6, n_side=n_side, seed=1)
    n = V.shape[-1]
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    dev = torch.device("cuda")
    y0, x0, wy, wx = wap.detector_window((n, n), (ps, ps), E, 45.0)
    rng = np.random.default_rng(7)
    target = torch.tensor(rng.random((len(pos), wy, wx)), dtype=torch.float32, device=dev)
    Vt = torch.tensor(V, device=dev)

    V1 = Vt.clone().requires_grad_(True)
    _, dpc = simulate_fresnel_as_differentiable(V1, probe, H, dz, E, positions=pos, ckpt_every=2, max_angle=45.0,
                                                sampling=ps)
    ((dpc - target) ** 2).sum().backward()

    V2 = Vt.clone().requires_grad_(True)
    _, dpf = simulate_fresnel_as_differentiable(V2, probe, H, dz, E, positions=pos, ckpt_every=2)
    ((dpf[..., y0:y0 + wy, x0:x0 + wx] - target) ** 2).sum().backward()

    assert torch.equal(dpc.detach(), dpf.detach()[..., y0:y0 + wy, x0:x0 + wx])
    rel = float((V1.grad - V2.grad).norm() / V2.grad.norm())
    assert rel < 1e-6, rel   # same kernels and seed values: equal up to atomic-add ordering


def test_bad_window_rejected(wap):
    from wideanglepropagation_b200 import _lib
    plan = wap.get_plan(64, 64, 1, _lib.WAP_OP_FRESNEL_AS)
    with pytest.raises(ValueError):
        _lib.check(_lib.lib().wap_plan_set_detector(plan.handle, 40, 0, 30, 10))
    with pytest.raises(ValueError):
        _lib.check(_lib.lib().wap_plan_set_detector(plan.handle, -1, 0, 10, 10))
    _lib.check(_lib.lib().wap_plan_set_detector(plan.handle, 0, 0, 0, 0))


@pytest.mark.parametrize("n_side", [2, 3])   # 4 probes: pass kernels; 9: persistent scheduler
def test_gradient_window_and_exit_loss(wap, n_side):
    """A loss on the cropped pattern and on the exit wave together: the seed
    scatters the window's dL/d(dp) and adds fft2(dL/d(exit) / 2); the result
    equals the full-grid pattern cropped by hand."""
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    V, probe, pos, ps, dz, E = _case(n=128, N=6, n_side=n_side, seed=2)
    n = V.shape[-1]
    H = wap.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    dev = torch.device("cuda")
    y0, x0, wy, wx = wap.detector_window((n, n), (ps, ps), E, 45.0)
    rng = np.random.default_rng(8)
    target = torch.tensor(rng.random((len(pos), wy, wx)), dtype=torch.float32, device=dev)
    c = torch.tensor(rng.normal(size=(len(pos), n, n)) + 1j * rng.normal(size=(len(pos), n, n)),
                     dtype=torch.complex64, device=dev)
    Vt = torch.tensor(V, device=dev)

    V1 = Vt.clone().requires_grad_(True)
    ex1, dpc = simulate_fresnel_as_differentiable(V1, probe, H, dz, E, positions=pos, ckpt_every=2, max_angle=45.0,
                                                  sampling=ps)
    (((dpc - target) ** 2).sum() + 1e-2 * (ex1 * c).real.sum()).backward()

    V2 = Vt.clone().requires_grad_(True)
    ex2, dpf = simulate_fresnel_as_differentiable(V2, probe, H, dz, E, positions=pos, ckpt_every=2)
    (((dpf[..., y0:y0 + wy, x0:x0 + wx] - target) ** 2).sum() + 1e-2 * (ex2 * c).real.sum()).backward()

    rel = float((V1.grad - V2.grad).norm() / V2.grad.norm())
    assert rel < 1e-6, rel
