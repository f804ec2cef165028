"""1D line helpers (propagation.py:609-652) and the naive WPM step
(:184-212) on the device, against the reference-generated fixtures and the
oracle.

Tolerances: float64 transfer functions and the float64 naive step agree with
the fixtures to rounding (1e-12); the complex64 line transforms to 1e-5
rel-L2, the bar of the multislice path.
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


def rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_line_transfer_functions(wap, golden):
    n, dx, dy, k0 = golden["l1_meta"]
    kx = wap.get_kx_1d(int(n), dx)
    assert rel(kx, golden["l1_kx"]) < 1e-15
    assert rel(wap.fresnel_kernel_1d(kx ** 2, k0, dy), golden["l1_Hf"]) < 1e-13
    Ha = wap.angular_spectrum_kernel_1d(kx ** 2, k0, dy)
    assert Ha.dtype == torch.complex128
    assert rel(Ha, golden["l1_Ha"]) < 1e-13          # evanescent entries included


@pytest.mark.parametrize("which", ["f", "a"])
def test_propagate_1d(wap, golden, which):
    H = golden[f"l1_H{which}"]
    out = wap.propagate_1d(golden["l1_psi"], H)
    assert out.shape == golden["l1_psi"].shape
    assert rel(out, golden[f"l1_prop_{which}"]) < 1e-5


def test_wpm_kernel_1d(wap, golden):
    n, dx, dy, k0 = golden["l1_meta"]
    kx2 = golden["l1_kx"] ** 2
    psik = np.fft.fft(golden["l1_psi"][0])
    assert rel(wap.wpm_kernel_1d(psik, 1.3, k0, kx2, dy), golden["l1_wpm1"]) < 1e-5
    out = wap.wpm_kernel_1d_vmap(psik, golden["l1_nvals"], k0, kx2, dy)
    assert out.shape == golden["l1_wpmv"].shape
    assert rel(out, golden["l1_wpmv"]) < 1e-5


@pytest.mark.parametrize("n", [32, 256, 2048])
def test_propagate_1d_sizes_and_per_line_H(wap, n):
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(n)
    psi = rng.normal(size=(5, n)) + 1j * rng.normal(size=(5, n))
    kx = O.get_kx_1d(n, 0.2)
    H = np.stack([O.angular_spectrum_kernel_1d(kx ** 2, 9.0 + i, 3.0 + 0.5 * i) for i in range(5)])
    assert rel(wap.propagate_1d(psi, H), O.propagate_1d(psi, H)) < 1e-5
    assert rel(wap.propagate_1d(psi, H[0]), O.propagate_1d(psi, H[0])) < 1e-5


def test_unsupported_line_length(wap):
    with pytest.raises(ValueError):
        wap.propagate_1d(np.ones(48, np.complex64), np.ones(48, np.complex64))


def test_naive_wpm_step_matches_reference(wap, golden):
    ny, nx, ps, dz, E = golden["naive_meta"]
    out = wap.wpm_step(golden["naive_wave"], golden["naive_n"], dz, E, (ps, ps))
    assert out.dtype == torch.complex128
    assert rel(out, golden["naive_out"]) < 1e-11


def test_binned_wpm_converges_to_naive(wap):
    """The exactness check: the adaptive-binning step approaches the per-pixel
    step as the bins get finer, with the same error as the FP64 oracle's."""
    import wideanglepropagation_b200.synthetic as S
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(3)
    ny = nx = 32
    ps, dz, E = 0.05, 2.04, 300e3
    V = (S.random_gaussian_stack(rng, 1, ny, nx, ps, 3, 80.0, 0.2) / dz)[0]
    wave = S.aperture_probe(ny, nx, ps, E, 40.0, 0.0, dtype=np.complex128)
    nmap = O.electron_refractive_index(V, E)
    naive = wap.wpm_step(wave, nmap, dz, E, (ps, ps)).cpu().numpy()
    assert O.rel_l2(naive, O.wpm_step(wave, nmap, dz, E, (ps, ps))) < 1e-11
    errs = []
    for K in (16, 64, 256):
        binned = wap.wpm_step_adaptive(wave.astype(np.complex64), nmap, dz, E, (ps, ps), n_bins=K,
                                       power_spacing=1.0)[0]
        ref = O.wpm_step_adaptive(wave, nmap, dz, E, (ps, ps), n_bins=K, power_spacing=1.0)[0]
        e, e_ref = rel(binned, naive), O.rel_l2(ref, naive)
        assert abs(e - e_ref) < 0.1 * e_ref + 2e-6, (K, e, e_ref)
        errs.append(e)
    assert errs[0] > errs[1] > errs[2]


def test_wpm_propagation_kernel_2d(wap):
    """wpm_propagation_kernel(_vmap) (propagation.py:159-171) against the oracle,
    with evanescent components (k_perp beyond n k0 at the grid corners)."""
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(11)
    ny, nx = 64, 128
    Ek = np.fft.fft2(rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx)))
    k0, dz = 30.0, 0.8
    ky = 2 * np.pi * np.fft.fftfreq(ny, 0.1)
    kx = 2 * np.pi * np.fft.fftfreq(nx, 0.1)
    kp2 = ky[:, None] ** 2 + kx[None, :] ** 2
    assert (kp2 > (1.3 * k0) ** 2).any()
    ns = [1.0, 1.1, 1.3]
    out = wap.wpm_propagation_kernel_vmap(Ek, ns, k0, kp2, dz)
    for i, n in enumerate(ns):
        assert rel(out[i], O.wpm_propagation_kernel(Ek, n, k0, kp2, dz)) < 1e-5
    assert rel(wap.wpm_propagation_kernel(Ek, 1.1, k0, kp2, dz), O.wpm_propagation_kernel(Ek, 1.1, k0, kp2, dz)) < 1e-5
    with pytest.raises(NotImplementedError):
        wap.get_abtem_transmit(None, 300e3)
