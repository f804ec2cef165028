"""Grids whose sides are not powers of two (Bluestein transforms through the
power-of-two FFT core): Fresnel / angular-spectrum and WPM multislice on
100^2 (the reference notebook's gpts = 100), 96 x 160, 120^2, an odd prime
side and a mixed power-of-two / generic grid, against the FP64 oracle.

Bar: rel-L2 <= 1e-5 of exit wave, pattern and wavefront stack, as on
power-of-two grids.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-5


@pytest.fixture(scope="module")
def wap():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import wideanglepropagation_b200 as w
    return w


def np_(t):
    return t.detach().cpu().numpy()


def rel(a, b):
    from oracle.propagation_oracle import rel_l2
    return rel_l2(a, b)


def _setup(ny, nx, N, seed, ps=0.1, E=200e3, dz=2.0, atoms=12):
    import wideanglepropagation_b200.synthetic as S
    rng = np.random.default_rng(seed)
    V = np.stack([S.gaussian_slice(ny, nx, ps, rng.uniform(0, 1, (atoms, 2)) * [ny * ps, nx * ps], 20.0, 0.3)
                  for _ in range(N)]) / dz
    probe = S.aperture_probe(ny, nx, ps, E, 20.0, -30.0, dtype=np.complex64)
    return V.astype(np.float32), probe, ps, dz, E


@pytest.mark.parametrize("ny,nx,kind", [(100, 100, "fresnel"), (96, 160, "as"), (120, 120, "as"),
                                        (67, 67, "fresnel"), (128, 100, "as"), (1000, 1000, "as")])
def test_fresnel_as_generic_grid(wap, ny, nx, kind):
    from oracle import propagation_oracle as O
    N = 3 if ny == 1000 else 12
    V, probe, ps, dz, E = _setup(ny, nx, N, seed=ny + nx)
    tf = O.fresnel_propagation_kernel if kind == "fresnel" else O.angular_spectrum_propagation_kernel
    H = tf(ny, nx, (ps, ps), dz, E)
    ex, dp, st = wap.simulate_fresnel_as(V, probe, H, dz, E)
    rex, rdp, rst = O.simulate_fresnel_as(V, probe, H, dz, E)
    assert ex.shape == (ny, nx) and dp.shape == (ny, nx) and st.shape == (N, ny, nx)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL
    assert rel(np_(st), rst) < TOL


def test_generic_grid_probes_positions_draws_window(wap):
    """A batch on 100 x 120: per-probe positions (move_probe, wrapping),
    potential draws, a detector window and the device transfer function."""
    from oracle import propagation_oracle as O
    ny, nx, N = 100, 120, 6
    V0, probe, ps, dz, E = _setup(ny, nx, N, seed=3)
    V1, _, _, _, _ = _setup(ny, nx, N, seed=4)
    V = np.stack([V0, V1])
    pos = np.array([[50, 60], [0, 0], [99, 119], [13, 77], [70, 5]], np.int32)
    draw = np.array([0, 1, 1, 0, 1], np.int32)
    H = wap.angular_spectrum_propagation_kernel(ny, nx, (ps, ps), dz, E)
    kw = dict(positions=pos, draw=draw, return_wavefronts=False)
    ex, dp, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, **kw)
    _, dpw, _ = wap.simulate_fresnel_as(V, probe, H, dz, E, max_angle=30.0, sampling=(ps, ps), **kw)
    Hh = H.cpu().numpy()
    lam = O.energy2wavelength(E)
    for b in range(len(pos)):
        p0 = O.move_probe(probe, tuple(pos[b]))
        rex, rdp, _ = O.simulate_fresnel_as(V[draw[b]], p0, Hh, dz, E, return_wavefronts=False)
        assert rel(np_(ex[b]), rex) < TOL
        assert rel(np_(dp[b]), rdp) < TOL
        assert np.array_equal(np_(dpw[b]), O.downsample_to_max_angle(np_(dp[b]), (ps, ps), lam, 30.0))


@pytest.mark.parametrize("ny,nx,K,p", [(100, 100, 16, 1.0), (96, 160, 8, 2.0), (120, 120, 128, 2.0)])
def test_wpm_generic_grid(wap, ny, nx, K, p):
    from oracle import propagation_oracle as O
    V, probe, _, dz, E = _setup(ny, nx, 8, seed=ny * 3 + K, ps=0.05, E=300e3, dz=2.04)
    ps = 0.05
    ex, dp, st = wap.simulate_wpm(V, probe, dz, E, (ps, ps), n_bins=K, power_spacing=p)
    rex, rdp, rst = O.simulate_wpm(V, probe, dz, E, (ps, ps), n_bins=K, power_spacing=p)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL
    assert rel(np_(st), rst) < TOL


def test_generic_grid_unsupported_paths_raise(wap):
    """The gradient and the probe builder need power-of-two grids: they raise
    ValueError on a generic grid instead of computing something else."""
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    V, probe, ps, dz, E = _setup(100, 100, 3, seed=9)
    H = wap.fresnel_propagation_kernel(100, 100, (ps, ps), dz, E)
    Vt = torch.tensor(V, device="cuda", requires_grad=True)
    with pytest.raises(ValueError, match="power-of-two"):
        simulate_fresnel_as_differentiable(Vt, probe, H, dz, E)
    with pytest.raises(ValueError, match="power-of-two"):
        wap.aperture_probe(100, 100, ps, E, 20.0)
