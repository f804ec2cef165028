"""Parity at the benchmark configurations' full sizes and at the reference's
own default arguments.

* WPM, 512^2, K = 16 linear bins, all 200 slices (the WPM configuration);
* simulate_wpm with the reference defaults n_bins=128, power_spacing=2.0
  (wide_angle_propagation/propagation.py:358) on 128^2 and 256^2 grids, 24
  slices;
* wpm_step_adaptive with its default n_bins=256 (propagation.py:215) against
  the oracle's adaptive step;
* two full-length classes of the batched scan (256^2 x 80 slices and 512^2 x
  150 slices, 16 probes each) through the persistent scheduler, 3 probes per
  class against the FP64 oracle;
* the gradient configuration: 512^2, 64 slices, checkpoint every 8, 8 probes
  (the persistent gradient chain) against autograd of the complex128
  restatement and against central differences, h = 1e-3 V*A on 32 voxels.

Bar: rel-L2 <= 1e-5 of exit wave and pattern against the FP64 oracle;
gradients <= 1e-4 against autograd and <= 2e-3 against central differences
(their truncation error), as in test_gpu_grad.py.  The complex128 gradient
restatement runs on the device here (torch's FFTs, float64): on the host the
64 forward evaluations of the differences would take minutes.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

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


def test_wpm_config_full_length(wap):
    """512^2, K = 16 linear bins, FCC [100], all 200 slices."""
    from oracle import propagation_oracle as O
    w = wap.synthetic.wpm_fcc(0)
    assert w.n_slices == 200 and w.ny == 512 and w.n_bins == 16
    ex, dp, _ = wap.simulate_wpm(w.potential[0], w.probe, w.dz, w.energy, (w.ps, w.ps), 16, 1.0,
                                 return_wavefronts=False)
    rex, rdp, _ = O.simulate_wpm(w.potential[0], w.probe, w.dz, w.energy, (w.ps, w.ps), 16, 1.0,
                                 return_wavefronts=False)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL


@pytest.mark.parametrize("n", [128, 256])
def test_wpm_reference_defaults(wap, n):
    """simulate_wpm(..., n_bins=128, power_spacing=2.0): the reference's own
    defaults, 24 slices; a convergent probe, so the pattern is not trivial."""
    from oracle import propagation_oracle as O
    w = wap.synthetic.wpm_fcc(3, n_slices=24, n=n)
    probe = wap.synthetic.aperture_probe(n, n, w.ps, w.energy, 25.0, -40.0, dtype=np.complex64)
    ex, dp, st = wap.simulate_wpm(w.potential[0], probe, w.dz, w.energy, (w.ps, w.ps))
    rex, rdp, rst = O.simulate_wpm(w.potential[0], probe, w.dz, w.energy, (w.ps, w.ps))
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL
    assert rel(np_(st), rst) < TOL


def test_wpm_step_adaptive_default_bins(wap):
    """wpm_step_adaptive with its default n_bins=256, power_spacing=2.0 against
    the oracle's adaptive step (new wave, weights, left indices, bins)."""
    from oracle import propagation_oracle as O
    w = wap.synthetic.wpm_fcc(5, n_slices=1, n=256)
    rng = np.random.default_rng(5)
    wave = (rng.normal(size=(256, 256)) + 1j * rng.normal(size=(256, 256))).astype(np.complex64)
    n_map = O.electron_refractive_index(w.potential[0, 0].astype(np.float64), w.energy)
    new, wgt, idx, refs = wap.wpm_step_adaptive(wave, n_map, w.dz, w.energy, (w.ps, w.ps))
    rnew, rw, ridx, rrefs = O.wpm_step_adaptive(wave.astype(np.complex128), n_map, w.dz, w.energy, (w.ps, w.ps))
    assert len(rrefs) == 256
    assert rel(np_(new), rnew) < TOL
    assert np.array_equal(np_(idx), ridx)
    assert np.max(np.abs(np_(wgt) - rw)) < 1e-9
    assert np.max(np.abs(np_(refs) - rrefs)) < 1e-14


@pytest.fixture(scope="module")
def scan_classes(wap):
    """Two full-length classes of the batched scan, 16 probes each: 256^2 x 80
    slices (4 x 4 raster, 1 draw) and 512^2 x 150 slices (4 x 4 raster)."""
    S = wap.synthetic
    return [S.batched_scan_class(0, 256, 80, 4, 1), S.batched_scan_class(1, 512, 150, 4, 1)]


@pytest.mark.parametrize("ci", [0, 1])
def test_scan_full_length_classes(wap, scan_classes, ci):
    """The persistent scheduler (public API, >= 8 probes) on a full-length
    class: probes 0, 7 and 15 against the FP64 oracle."""
    from oracle import propagation_oracle as O
    w = scan_classes[ci]
    assert w.n_probes == 16
    H = wap.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    ex, dp, _ = wap.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy, positions=w.positions,
                                        return_wavefronts=False)
    Hh = H.cpu().numpy()
    for b in (0, 7, 15):
        p0 = O.move_probe(w.probe, tuple(w.positions[b]))
        rex, rdp, _ = O.simulate_fresnel_as(w.potential[0], p0, Hh, w.dz, w.energy, return_wavefronts=False)
        assert rel(np_(ex[b]), rex) < TOL, b
        assert rel(np_(dp[b]), rdp) < TOL, b


@pytest.fixture(scope="module")
def grad_problem(wap):
    """512^2, 64 slices x 2 A, 300 keV, 8 probes (a 2 x 4 raster of the 8 x 8
    one), target from a seed-drawn Gaussian-atom stack, unknown = 0.4 x another
    seed-drawn stack (at V = 0 most voxels' gradients vanish)."""
    import wideanglepropagation_b200.synthetic as S
    from oracle import propagation_oracle as O
    w = S.inverse_problem(0)
    rng = np.random.default_rng(7)
    V0 = 0.4 * S.random_gaussian_stack(rng, w.n_slices, w.ny, w.nx, w.ps, 30, 20.0, 0.3) / w.dz
    pos = w.positions[::8][:8]
    H = O.fresnel_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    return w, V0, pos, H


def _oracle_loss(V, probe, H, dz, E, target, pos):
    from oracle import torch_oracle as T
    _, dp = T.simulate(V, probe, H, dz, E, pos, device="cuda")
    return ((dp - target) ** 2).sum()


def test_gradient_config(wap, grad_problem):
    """dL/dV of L = sum (|FFT psi_exit|^2 - I)^2 on the gradient configuration
    (checkpoint every 8, persistent gradient chain) against complex128
    autograd, and against central differences (h = 1e-3 V*A) on 32 voxels."""
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    w, V0, pos, H = grad_problem
    dz, E = w.dz, w.energy
    with torch.no_grad():
        _, tgt = T.simulate(torch.tensor(w.potential[0], dtype=torch.float64, device="cuda"), w.probe, H, dz, E, pos,
                            device="cuda")
    # the library's adjoint
    V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
    _, dp = simulate_fresnel_as_differentiable(V, w.probe, H, dz, E, positions=pos, ckpt_every=8)
    L = ((dp.double() - tgt) ** 2).sum()
    L.backward()
    g = V.grad.double()
    # autograd of the complex128 restatement
    Vr = torch.tensor(V0, dtype=torch.float64, device="cuda", requires_grad=True)
    Lr = _oracle_loss(Vr, w.probe, H, dz, E, tgt, pos)
    Lr.backward()
    gr = Vr.grad
    assert abs(float(L) - float(Lr)) / float(Lr) < 1e-4
    err = float(torch.linalg.vector_norm(g - gr) / torch.linalg.vector_norm(gr))
    assert err < 1e-4, err
    # central differences on 32 voxels (weighted towards large gradients)
    rng = np.random.default_rng(2)
    flat = np.abs(gr.cpu().numpy()).ravel()
    idx = rng.choice(flat.size, 32, replace=False, p=flat / flat.sum())
    h = 1e-3 / dz
    Vd = torch.tensor(V0, dtype=torch.float64, device="cuda")
    num = []
    with torch.no_grad():
        for i in idx:
            flat_v = Vd.view(-1)
            old = float(flat_v[i])
            flat_v[i] = old + h
            Lp = float(_oracle_loss(Vd, w.probe, H, dz, E, tgt, pos))
            flat_v[i] = old - h
            Lm = float(_oracle_loss(Vd, w.probe, H, dz, E, tgt, pos))
            flat_v[i] = old
            num.append((Lp - Lm) / (2 * h))
    num = np.array(num)
    ana = g.cpu().numpy().ravel()[idx]
    assert np.linalg.norm(num - ana) / np.linalg.norm(num) < 2e-3
