"""Adjoint multislice (wap_multislice_bwd) against torch-complex128 autograd
of the restated reference and against central finite differences.

Tolerances: rel-L2 of dL/dV <= 1e-4 vs autograd (float32 kernels, long
chains of FFTs); central FD with h = 1e-3 V*A agrees to 2e-3 relative on the
sampled voxels (FD truncation error dominates).
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


def _problem(n=64, N=9, n_side=2, seed=0):
    import wideanglepropagation_b200.synthetic as S
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.1, 2.0, 300e3
    Vt = (S.random_gaussian_stack(rng, N, n, n, ps, 4, 20.0, 0.3) / dz)
    V0 = 0.5 * (S.random_gaussian_stack(rng, N, n, n, ps, 4, 20.0, 0.3) / dz)
    probe = S.aperture_probe(n, n, ps, E, 25.0, -50.0, dtype=np.complex64)
    pos = S.raster_positions(n, n, n_side, n_side)
    H = O.fresnel_propagation_kernel(n, n, (ps, ps), dz, E)
    from oracle import torch_oracle as T
    _, target = T.simulate(torch.tensor(Vt), probe, H, dz, E, pos)
    return Vt, V0, probe, pos, H, dz, E, target.numpy()


@pytest.mark.parametrize("ckpt", [1, 3, 4, 9])
def test_grad_matches_autograd(wap, ckpt):
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    Vt, V0, probe, pos, H, dz, E, target = _problem()
    L_ref, g_ref = T.loss_and_grad(V0, probe, H, dz, E, target, pos)
    V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
    ex, dp = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, ckpt_every=ckpt)
    L = ((dp - torch.tensor(target, device="cuda", dtype=torch.float32)) ** 2).sum()
    L.backward()
    g = V.grad.cpu().numpy()
    assert abs(float(L) - L_ref) / L_ref < 1e-4
    err = np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)
    assert err < 1e-4, err


def test_grad_exit_wave_loss(wap):
    """A loss on the complex exit wave (torch complex-gradient convention).

    Re(sum c psi) with random complex c sums terms of random sign, so the
    float32 result carries more relative error: tolerance 5e-4."""
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    Vt, V0, probe, pos, H, dz, E, target = _problem(N=5)
    rng = np.random.default_rng(1)
    c = (rng.normal(size=(len(pos), 64, 64)) + 1j * rng.normal(size=(len(pos), 64, 64)))
    Vr = torch.tensor(V0, requires_grad=True)
    ex_r, dp_r = T.simulate(Vr, probe, H, dz, E, pos)
    Lr = (ex_r * torch.tensor(c)).real.sum() + 1e-3 * (dp_r ** 2).sum()
    Lr.backward()
    V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
    ex, dp = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, ckpt_every=2)
    L = (ex * torch.tensor(c, dtype=torch.complex64, device="cuda")).real.sum() + 1e-3 * (dp.double() ** 2).sum()
    L.backward()
    err = np.linalg.norm(V.grad.cpu().numpy() - Vr.grad.numpy()) / np.linalg.norm(Vr.grad.numpy())
    assert err < 5e-4, err


def test_grad_central_differences(wap):
    """dL/dV against central FD, h = 1e-3 V*A (= 1e-3/dz V) on 32 voxels, FP64 oracle loss."""
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    Vt, V0, probe, pos, H, dz, E, target = _problem(N=6)
    V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
    _, dp = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, ckpt_every=2)
    ((dp - torch.tensor(target, device="cuda", dtype=torch.float32)) ** 2).sum().backward()
    g = V.grad.cpu().numpy()
    rng = np.random.default_rng(2)
    # voxels weighted towards where the gradient is large
    flat = np.abs(g).ravel()
    idx = rng.choice(flat.size, 32, replace=False, p=flat / flat.sum())
    h = 1e-3 / dz
    num, ana = [], []
    for i in idx:
        vp = V0.copy().ravel(); vp[i] += h
        vm = V0.copy().ravel(); vm[i] -= h
        Lp, _ = T.loss_and_grad(vp.reshape(V0.shape), probe, H, dz, E, target, pos)
        Lm, _ = T.loss_and_grad(vm.reshape(V0.shape), probe, H, dz, E, target, pos)
        num.append((Lp - Lm) / (2 * h))
        ana.append(g.ravel()[i])
    num, ana = np.array(num), np.array(ana)
    assert np.linalg.norm(num - ana) / np.linalg.norm(num) < 2e-3


def test_grad_with_draws(wap):
    """Two potential draws: each probe's contribution lands in its own draw."""
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    Vt, V0, probe, pos, H, dz, E, target = _problem(N=4)
    V2 = np.stack([V0, 0.7 * V0])
    draw = np.array([0, 1, 1, 0], np.int32)
    V = torch.tensor(V2, dtype=torch.float32, device="cuda", requires_grad=True)
    _, dp = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, draw=draw, ckpt_every=2)
    tgt = torch.tensor(target, device="cuda", dtype=torch.float32)
    ((dp - tgt) ** 2).sum().backward()
    g = V.grad.cpu().numpy()
    for d in range(2):
        sel = np.nonzero(draw == d)[0]
        _, gr = T.loss_and_grad(V2[d], probe, H, dz, E, target[sel], pos[sel])
        assert np.linalg.norm(g[d] - gr) / np.linalg.norm(gr) < 1e-4


def _scan_problem(n=128, N=9, n_side=3, seed=4):
    import wideanglepropagation_b200.synthetic as S
    from oracle import propagation_oracle as O
    from oracle import torch_oracle as T
    rng = np.random.default_rng(seed)
    ps, dz, E = 0.08, 2.0, 300e3
    Vt = S.random_gaussian_stack(rng, N, n, n, ps, 6, 20.0, 0.3) / dz
    V0 = 0.5 * (S.random_gaussian_stack(rng, N, n, n, ps, 6, 20.0, 0.3) / dz)
    probe = S.aperture_probe(n, n, ps, E, 25.0, -50.0, dtype=np.complex64)
    pos = S.raster_positions(n, n, n_side, n_side)
    H = O.angular_spectrum_propagation_kernel(n, n, (ps, ps), dz, E)
    _, target = T.simulate(torch.tensor(Vt), probe, H, dz, E, pos)
    return V0, probe, pos, H, dz, E, target.numpy()


@pytest.mark.parametrize("ckpt", [1, 3, 4, 9])
def test_persistent_gradient_matches_autograd(wap, ckpt):
    """>= 8 probes on a 128^2 grid: forward, checkpoints, recompute and adjoint
    all run in the persistent scheduler."""
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    V0, probe, pos, H, dz, E, target = _scan_problem()
    assert len(pos) >= 8
    L_ref, g_ref = T.loss_and_grad(V0, probe, H, dz, E, target, pos)
    V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
    _, dp = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, ckpt_every=ckpt)
    L = ((dp - torch.tensor(target, device="cuda", dtype=torch.float32)) ** 2).sum()
    L.backward()
    err = np.linalg.norm(V.grad.cpu().numpy() - g_ref) / np.linalg.norm(g_ref)
    assert abs(float(L) - L_ref) / L_ref < 1e-4
    assert err < 1e-4, err


def test_persistent_gradient_two_pending_graphs(wap):
    """Two forwards before their backwards get separate scan buffers."""
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    V0, probe, pos, H, dz, E, target = _scan_problem(N=5, seed=6)
    tgt = torch.tensor(target, device="cuda", dtype=torch.float32)
    V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
    _, dp1 = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, ckpt_every=2)
    _, dp2 = simulate_fresnel_as_differentiable(V * 0.5, probe, H, dz, E, positions=pos, ckpt_every=2)
    (((dp1 - tgt) ** 2).sum() + ((dp2 - tgt) ** 2).sum()).backward()
    Vr = torch.tensor(V0, requires_grad=True)
    _, d1 = T.simulate(Vr, probe, H, dz, E, pos)
    _, d2 = T.simulate(Vr * 0.5, probe, H, dz, E, pos)
    tr = torch.tensor(target)
    (((d1 - tr) ** 2).sum() + ((d2 - tr) ** 2).sum()).backward()
    err = np.linalg.norm(V.grad.cpu().numpy() - Vr.grad.numpy()) / np.linalg.norm(Vr.grad.numpy())
    assert err < 1e-4, err


@pytest.mark.parametrize("ckpt,dp_weight", [(3, 1e-3), (9, 1e-3), (2, 0.0)])
def test_persistent_gradient_exit_wave_loss(wap, ckpt, dp_weight):
    """A loss on the exit wave through the persistent scheduler: the seed adds
    fft2(dL/d(exit) / 2) to the diffraction term (or stands alone when the
    loss ignores the pattern).  Tolerance 5e-4 as for the per-pass case."""
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import SCAN_MIN_PROBES, simulate_fresnel_as_differentiable
    V0, probe, pos, H, dz, E, target = _scan_problem(N=7, seed=8)
    assert len(pos) >= SCAN_MIN_PROBES
    n = V0.shape[-1]
    rng = np.random.default_rng(2)
    c = rng.normal(size=(len(pos), n, n)) + 1j * rng.normal(size=(len(pos), n, n))
    Vr = torch.tensor(V0, requires_grad=True)
    ex_r, dp_r = T.simulate(Vr, probe, H, dz, E, pos)
    Lr = (ex_r * torch.tensor(c)).real.sum()
    if dp_weight:
        Lr = Lr + dp_weight * (dp_r ** 2).sum()
    Lr.backward()
    V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
    ex, dp = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, ckpt_every=ckpt)
    L = (ex * torch.tensor(c, dtype=torch.complex64, device="cuda")).real.sum()
    if dp_weight:
        L = L + dp_weight * (dp.double() ** 2).sum()
    L.backward()
    err = np.linalg.norm(V.grad.cpu().numpy() - Vr.grad.numpy()) / np.linalg.norm(Vr.grad.numpy())
    assert err < 5e-4, err


@pytest.mark.parametrize("cfg", [(4, 4, 4), (4, 16, 2), (16, 4, 8)])
def test_grad_small_element_shapes(wap, cfg):
    """The adjoint on the 4-elements-per-thread pass shapes (row E, column E,
    column width) that the one/two-probe launch shapes may use."""
    from oracle import torch_oracle as T
    from wideanglepropagation_b200 import _lib
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    Vt, V0, probe, pos, H, dz, E, target = _problem(N=5, seed=3)
    L_ref, g_ref = T.loss_and_grad(V0, probe, H, dz, E, target, pos)
    plan = wap.get_plan(64, 64, len(pos), _lib.WAP_OP_FRESNEL_AS)
    old = plan.config()
    try:
        plan.set_config(*cfg)
        V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
        _, dp = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, ckpt_every=2)
        L = ((dp - torch.tensor(target, device="cuda", dtype=torch.float32)) ** 2).sum()
        L.backward()
        assert plan.config() == cfg
    finally:
        plan.set_config(*old)
    err = np.linalg.norm(V.grad.cpu().numpy() - g_ref) / np.linalg.norm(g_ref)
    assert err < 1e-4, err


def test_grad_non_square_grid(wap):
    """The pass-kernel adjoint on a 64 x 128 grid (the persistent scheduler
    takes square grids only) against the autograd of the torch restatement."""
    import wideanglepropagation_b200.synthetic as S
    from oracle import propagation_oracle as O
    from oracle import torch_oracle as T
    from wideanglepropagation_b200.autograd import simulate_fresnel_as_differentiable
    rng = np.random.default_rng(21)
    ny, nx, N, ps, dz, E = 64, 128, 5, 0.1, 2.0, 300e3
    Vt = S.random_gaussian_stack(rng, N, ny, nx, ps, 4, 20.0, 0.3) / dz
    V0 = 0.5 * S.random_gaussian_stack(rng, N, ny, nx, ps, 4, 20.0, 0.3) / dz
    probe = S.aperture_probe(ny, nx, ps, E, 25.0, -50.0, dtype=np.complex64)
    pos = np.array([[20, 40], [32, 64], [50, 100]], dtype=np.int32)
    H = O.fresnel_propagation_kernel(ny, nx, (ps, ps), dz, E)
    _, target = T.simulate(torch.tensor(Vt), probe, H, dz, E, pos)
    L_ref, g_ref = T.loss_and_grad(V0, probe, H, dz, E, target.numpy(), pos)
    V = torch.tensor(V0, dtype=torch.float32, device="cuda", requires_grad=True)
    _, dp = simulate_fresnel_as_differentiable(V, probe, H, dz, E, positions=pos, ckpt_every=2)
    L = ((dp - torch.tensor(target.numpy(), device="cuda", dtype=torch.float32)) ** 2).sum()
    L.backward()
    assert abs(float(L) - L_ref) / L_ref < 1e-4
    err = np.linalg.norm(V.grad.cpu().numpy() - g_ref) / np.linalg.norm(g_ref)
    assert err < 1e-4, err
