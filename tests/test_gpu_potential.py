"""Device-side Gaussian-atom potential builder against the host builders of
the synthetic workloads (same atoms, float64 NumPy sums).

Tolerance: the device sums float32 products of float64-evaluated profiles,
so rel-L2 <= 1e-6 and max |diff| <= 1e-6 of the peak; atoms beyond 7 sigma
of a pixel are skipped (< 2.3e-11 of a peak each).
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


def _check(dev_V, host_V):
    d = dev_V.double().cpu().numpy()
    assert d.shape == host_V.shape
    assert np.linalg.norm(d - host_V) <= 1e-6 * np.linalg.norm(host_V)
    assert np.abs(d - host_V).max() <= 1e-6 * np.abs(host_V).max()


def test_diamond_lattice_matches_host(wap):
    import wideanglepropagation_b200.synthetic as S
    args = (8, 256, 256, 0.05, 5.43, S.DIAMOND_LAYERS)
    host = S.lattice_stack(np.random.default_rng(5), *args, 25.0, 0.25, 0.08) / 1.3575
    pos, sl = S.lattice_atoms(np.random.default_rng(5), *args, 0.08)
    _check(wap.gaussian_potential(8, 256, 256, 0.05, pos, sl, 25.0, 0.25, scale=1 / 1.3575), host)


@pytest.mark.parametrize("shape", [(64, 96), (50, 70), (33, 128)])
def test_random_stack_partial_tiles(wap, shape):
    import wideanglepropagation_b200.synthetic as S
    ny, nx = shape
    host = S.random_gaussian_stack(np.random.default_rng(1), 3, ny, nx, 0.1, 30, 20.0, 0.3)
    pos, sl = S.random_gaussian_atoms(np.random.default_rng(1), 3, ny, nx, 0.1, 30)
    _check(wap.gaussian_potential(3, ny, nx, 0.1, pos, sl, 20.0, 0.3), host)


def test_anisotropic_sampling_amplitudes_and_many_atoms(wap):
    rng = np.random.default_rng(2)
    ny, nx, py, px, sigma = 64, 48, 0.07, 0.11, 0.35
    M = 700                                         # > 128 per tile: several culling rounds
    pos = rng.uniform(0, 1, (M, 2)) * (ny * py, nx * px)
    sl = rng.integers(0, 2, M)
    amp = rng.uniform(5, 50, M)
    host = np.zeros((3, ny, nx))                    # slice 2 holds no atom
    y, x = np.arange(ny) * py, np.arange(nx) * px
    for (cy, cx), s, a in zip(pos, sl, amp):
        dy = (y - cy + ny * py / 2) % (ny * py) - ny * py / 2
        dx = (x - cx + nx * px / 2) % (nx * px) - nx * px / 2
        host[s] += a * np.exp(-(dy[:, None] ** 2 + dx[None, :] ** 2) / (2 * sigma ** 2))
    V = wap.gaussian_potential(3, ny, nx, (py, px), pos, sl, amp, sigma)
    _check(V[:2], host[:2])
    assert torch.count_nonzero(V[2]) == 0


def test_no_atoms(wap):
    V = wap.gaussian_potential(2, 32, 32, 0.1, np.zeros((0, 2)), np.zeros(0), 1.0, 0.3)
    assert torch.count_nonzero(V) == 0


def test_multislice_from_device_potential(wap):
    import wideanglepropagation_b200.synthetic as S
    n, N, ps, dz, E = 128, 6, 0.05, 1.3575, 300e3
    host = (S.lattice_stack(np.random.default_rng(9), N, n, n, ps, 5.43, S.DIAMOND_LAYERS, 25.0, 0.25, 0.08)
            / dz).astype(np.float32)
    pos, sl = S.lattice_atoms(np.random.default_rng(9), N, n, n, ps, 5.43, S.DIAMOND_LAYERS, 0.08)
    Vd = wap.gaussian_potential(N, n, n, ps, pos, sl, 25.0, 0.25, scale=1 / dz)
    probe = S.aperture_probe(n, n, ps, E, 25.0, -50.0, dtype=np.complex64)
    H = wap.angular_spectrum_propagation_kernel(n, n, (ps, ps), dz, E)
    a, _, _ = wap.simulate_fresnel_as(host, probe, H, dz, E, return_wavefronts=False)
    b, _, _ = wap.simulate_fresnel_as(Vd, probe, H, dz, E, return_wavefronts=False)
    assert float((a - b).norm() / a.norm()) < 1e-6


def test_bad_arguments(wap):
    with pytest.raises(ValueError):
        wap.gaussian_potential(2, 32, 32, 0.1, np.zeros((1, 2)), [2], 1.0, 0.3)   # slice index out of range
    with pytest.raises(ValueError):
        wap.gaussian_potential(2, 32, 32, 0.1, np.zeros((1, 2)), [0], 1.0, 0.0)   # sigma must be positive
