"""Lippmann-Schwinger 2D solver (propagation.py:446-602): the Green's
function kernel (host float64, as the reference builds it), the device FFT
convolution (complex64 transforms: 1e-5), and the GMRES solve against the
reference-generated solution (tolerance-limited: 1e-4 at gmres_tol 1e-5)."""
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


def test_kernel_and_convolution(wap, golden):
    k0, h, n = golden["ls_meta"]
    n = int(n)
    Khat, emb = wap.build_lippmann_schwinger_kernel_2d(k0, h, h, n, n)
    assert emb == (2 * n, 2 * n)
    assert rel(Khat, golden["ls_Khat"]) < 1e-13
    # 24 -> embedding 48 (not a power of two: the Bluestein transforms), against
    # the reference's own convolution of the fixture source
    assert rel(wap.apply_convolution(golden["ls_src"], Khat, emb, (n, n)), golden["ls_conv"]) < 1e-5


@pytest.mark.parametrize("n", [16, 32])
def test_convolution_matches_oracle(wap, n):
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(n)
    src = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    k0 = 2 * np.pi / 0.3
    Khat_o, emb = O.build_lippmann_schwinger_kernel_2d(k0, 0.05, 0.05, n, n)
    Khat, _ = wap.build_lippmann_schwinger_kernel_2d(k0, 0.05, 0.05, n, n)
    ref = O.apply_convolution(src, Khat_o, emb, (n, n))
    assert rel(wap.apply_convolution(src, Khat, emb, (n, n)), ref) < 1e-5


def test_solve_matches_reference(wap, golden):
    E, ps, _ = golden["ls_solve_meta"]
    psi = wap.solve_scattering_2d_lippmann_schwinger(golden["ls_V"], E, ps, gmres_tol=1e-5)
    assert psi.shape == golden["ls_psi"].shape
    assert rel(psi, golden["ls_psi"]) < 1e-4


def test_solve_default_tolerance_vs_oracle(wap):
    import wideanglepropagation_b200.synthetic as S
    from oracle import propagation_oracle as O
    V = S.random_gaussian_stack(np.random.default_rng(4), 1, 32, 32, 0.1, 6, 20.0, 0.3)[0] / 2.0
    psi = wap.solve_scattering_2d_lippmann_schwinger(V, 200e3, 0.1)
    ref = O.solve_scattering_2d_lippmann_schwinger(V, 200e3, 0.1)
    assert rel(psi, ref) < 1e-3
    # the scattered part is not negligible: the solve does something
    y = (np.arange(64) * 0.1)
    inc = np.exp(1j * 2 * np.pi / 0.02508 * (y - y.mean()))[16:48]
    assert rel(psi, np.broadcast_to(inc, (32, 32))) > 1e-3
