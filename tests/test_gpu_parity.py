"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle.

Tolerance: rel-L2 <= 1e-5 on the complex exit wave vs the reference
algorithm in float64 (the oracle); the same bound on the diffraction pattern
and the wavefront stack.
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


# ---------------------------------------------------------------- golden
def test_golden_fresnel(wap, golden):
    ny, nx, ps, N, dz, E = golden["fres_meta"]
    ex, dp, st = wap.simulate_fresnel_as(golden["fres_V"], golden["fres_probe"], golden["fres_H"], dz, E)
    assert rel(np_(ex), golden["fres_exit"]) < TOL
    assert rel(np_(dp), golden["fres_dp"]) < TOL
    assert rel(np_(st), golden["fres_stack"]) < TOL


def test_golden_as_nonsquare(wap, golden):
    ny, nx, ps, N, dz, E = golden["as_meta"]
    ex, dp, st = wap.simulate_fresnel_as(golden["as_V"], golden["as_probe"], golden["as_H"], dz, E)
    assert ex.shape == (32, 64)
    assert rel(np_(ex), golden["as_exit"]) < TOL
    assert rel(np_(dp), golden["as_dp"]) < TOL
    assert rel(np_(st), golden["as_stack"]) < TOL


@pytest.mark.parametrize("K,p", [(16, 1.0), (8, 2.0)])
def test_golden_wpm(wap, golden, K, p):
    ny, nx, ps, N, dz, E = golden["wpm_meta"]
    ex, dp, st = wap.simulate_wpm(golden["wpm_V"], golden["wpm_probe"], dz, E, (ps, ps), n_bins=K, power_spacing=p)
    assert rel(np_(ex), golden[f"wpm_K{K}_exit"]) < TOL
    assert rel(np_(dp), golden[f"wpm_K{K}_dp"]) < TOL
    assert rel(np_(st), golden[f"wpm_K{K}_stack"]) < TOL


def test_golden_wpm_step(wap, golden):
    ny, nx, ps, N, dz, E = golden["wpm_meta"]
    from oracle import propagation_oracle as O
    nmap = O.electron_refractive_index(golden["wpm_V"][0], E)
    nw, w, iL, nrefs = wap.wpm_step_adaptive(golden["wstep_wave0"], nmap, dz, E, (ps, ps), 12, 2.0)
    assert rel(np_(nw), golden["wstep_out"]) < TOL
    assert np.array_equal(np_(iL), golden["wstep_idxL"])
    assert np.allclose(np_(w), golden["wstep_w"], atol=1e-12)
    nw, w, iL, _ = wap.wpm_step_adaptive(golden["wstep_wave0"], np.full((int(ny), int(nx)), nmap.mean()),
                                         dz, E, (ps, ps), 4, 1.0)
    assert np.all(np_(iL) == 0)


def test_transfer_functions(wap, golden):
    H = wap.fresnel_propagation_kernel(48, 64, (0.11, 0.09), 2.0, 200e3)
    assert H.dtype == torch.complex128
    assert rel(np_(H), golden["H_fres_48x64"]) < 1e-13
    assert rel(np_(wap.angular_spectrum_propagation_kernel(48, 64, (0.11, 0.09), 1.5, 300e3)),
               golden["H_as_48x64"]) < 1e-13
    assert rel(np_(wap.angular_spectrum_propagation_kernel(32, 32, (0.01, 0.01), 0.7, 300e3)),
               golden["H_as_evan_32x32"]) < 1e-13


# ---------------------------------------------------------------- known answers
@pytest.mark.parametrize("n", [32, 64, 128, 256, 512, 1024, 2048])
def test_vacuum_is_exact_propagator_power(wap, n):
    """V = 0: exit = ifft2(H^N fft2(psi0)) for every supported size."""
    rng = np.random.default_rng(n)
    psi = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))).astype(np.complex64)
    H = np.exp(1j * rng.uniform(-np.pi, np.pi, (n, n)))
    N = 3
    ex, dp, _ = wap.simulate_fresnel_as(np.zeros((N, n, n), np.float32), psi, H.astype(np.complex64), 1.0, 200e3,
                                        return_wavefronts=False)
    want = np.fft.ifft2(H.astype(np.complex64).astype(np.complex128) ** N * np.fft.fft2(psi.astype(np.complex128)))
    assert rel(np_(ex), want) < 2e-6
    want_dp = np.abs(np.fft.fftshift(np.fft.fft2(want))) ** 2
    assert rel(np_(dp), want_dp) < 4e-6


@pytest.mark.parametrize("shape", [(32, 2048), (2048, 32), (64, 128), (256, 32)])
def test_nonsquare_sizes(wap, shape):
    from oracle import propagation_oracle as O
    ny, nx = shape
    rng = np.random.default_rng(7)
    V = rng.uniform(0, 30, (2, ny, nx)).astype(np.float32)
    psi = (rng.normal(size=shape) + 1j * rng.normal(size=shape)).astype(np.complex64)
    H = O.fresnel_propagation_kernel(ny, nx, (0.05, 0.07), 1.5, 300e3)
    ex, dp, st = wap.simulate_fresnel_as(V, psi, H, 1.5, 300e3)
    rex, rdp, rst = O.simulate_fresnel_as(V, psi, H, 1.5, 300e3)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL
    assert rel(np_(st), rst) < TOL


def test_plane_wave_constant_potential(wap):
    """Constant V: uniform phase N 2 pi (n-1) dz / lam times the carrier H[0,0]^N."""
    from oracle import propagation_oracle as O
    n, N, dz, E, v0 = 128, 7, 2.0, 200e3, 13.0
    H = O.fresnel_propagation_kernel(n, n, (0.1, 0.1), dz, E)
    ex, _, _ = wap.simulate_fresnel_as(np.full((N, n, n), v0, np.float32), np.ones((n, n), np.complex64),
                                       H, dz, E, return_wavefronts=False)
    dn = O.electron_refractive_index(np.float64(v0), E) - 1
    want = np.exp(1j * N * 2 * np.pi * dn * dz / O.energy2wavelength(E)) * H[0, 0] ** N
    assert np.max(np.abs(np_(ex) - want)) < 2e-6


def test_unitarity(wap):
    rng = np.random.default_rng(3)
    n = 256
    psi = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))).astype(np.complex64)
    H = np.exp(1j * rng.uniform(-3, 3, (n, n))).astype(np.complex64)
    V = rng.uniform(0, 50, (40, n, n)).astype(np.float32)
    ex, _, _ = wap.simulate_fresnel_as(V, psi, H, 2.0, 200e3, return_wavefronts=False)
    assert abs(np.linalg.norm(np_(ex)) / np.linalg.norm(psi) - 1) < 1e-5


# ---------------------------------------------------------------- workloads
def test_plain_fresnel_full(wap):
    """256^2, 20 slices, 200 keV, Fresnel (the CPU-runnable workload) in full."""
    from oracle import propagation_oracle as O
    w = wap.synthetic.plain_fresnel(0)
    H = O.fresnel_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    ex, dp, st = wap.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy)
    rex, rdp, rst = O.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL
    assert rel(np_(st), rst) < TOL
    # the device transfer function (complex128) gives the same result
    Hd = wap.fresnel_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    ex2, _, _ = wap.simulate_fresnel_as(w.potential[0], w.probe, Hd, w.dz, w.energy)
    assert rel(np_(ex2), rex) < TOL


def test_angular_spectrum_full(wap):
    """1024^2, 100 slices, 300 keV, diamond [100], angular spectrum, in full."""
    from oracle import propagation_oracle as O
    w = wap.synthetic.angular_spectrum_diamond(0)
    H = O.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    ex, dp, _ = wap.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy, return_wavefronts=False)
    rex, rdp, _ = O.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy, return_wavefronts=False)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL


def test_wpm_fcc_reduced(wap):
    """512^2, K=16 linear bins, FCC [100]; 12 of the 200 slices (FP64 oracle cost)."""
    from oracle import propagation_oracle as O
    w = wap.synthetic.wpm_fcc(0, n_slices=12)
    ex, dp, st = wap.simulate_wpm(w.potential[0], w.probe, w.dz, w.energy, (w.ps, w.ps), 16, 1.0)
    rex, rdp, rst = O.simulate_wpm(w.potential[0], w.probe, w.dz, w.energy, (w.ps, w.ps), 16, 1.0)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL
    assert rel(np_(st), rst) < TOL


def test_wpm_evanescent(wap):
    """Fine sampling puts part of the spectrum beyond k0 (complex-sqrt branch)."""
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(11)
    n, ps, dz, E = 64, 0.004, 0.5, 300e3
    V = (rng.uniform(0, 40, (3, n, n))).astype(np.float32)
    psi = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))).astype(np.complex64)
    ex, dp, _ = wap.simulate_wpm(V, psi, dz, E, (ps, ps), 8, 2.0)
    rex, rdp, _ = O.simulate_wpm(V, psi, dz, E, (ps, ps), 8, 2.0)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL


def test_batched_scan_positions_and_draws(wap):
    from oracle import propagation_oracle as O
    cls = wap.synthetic.batched_scan(0, small=True)[0]
    H = O.angular_spectrum_propagation_kernel(cls.ny, cls.nx, (cls.ps, cls.ps), cls.dz, cls.energy)
    ex, dp, _ = wap.simulate_fresnel_as(cls.potential, cls.probe, H, cls.dz, cls.energy, positions=cls.positions,
                                        draw=cls.draw_of_probe, return_wavefronts=False)
    assert ex.shape == (cls.n_probes, cls.ny, cls.nx)
    for b in range(0, cls.n_probes, 5):
        p0 = O.move_probe(cls.probe, tuple(cls.positions[b]))
        rex, rdp, _ = O.simulate_fresnel_as(cls.potential[cls.draw_of_probe[b]], p0, H, cls.dz, cls.energy,
                                            return_wavefronts=False)
        assert rel(np_(ex[b]), rex) < TOL
        assert rel(np_(dp[b]), rdp) < TOL


def test_wpm_batched_probes(wap):
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(5)
    n = 64
    V = rng.uniform(0, 40, (2, n, n)).astype(np.float32)
    probe = O.move_probe(np.fft.fftshift(np.fft.ifft2((rng.random((n, n)) < 0.2).astype(np.complex128))), (n // 2, n // 2))
    pos = np.array([[10, 20], [32, 32], [63, 0]], np.int32)
    ex, dp, st = wap.simulate_wpm(V, probe, 2.0, 300e3, (0.05, 0.05), 8, 1.0, positions=pos)
    for b in range(3):
        rex, rdp, rst = O.simulate_wpm(V, O.move_probe(probe, tuple(pos[b])), 2.0, 300e3, (0.05, 0.05), 8, 1.0)
        assert rel(np_(ex[b]), rex) < TOL
        assert rel(np_(st[b]), rst) < TOL


def test_launch_configs_agree(wap):
    """Every autotuner candidate computes the same result."""
    from wideanglepropagation_b200 import autotune, _lib
    from oracle import propagation_oracle as O
    n = 256
    rng = np.random.default_rng(9)
    V = rng.uniform(0, 30, (3, n, n)).astype(np.float32)
    psi = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))).astype(np.complex64)
    H = O.fresnel_propagation_kernel(n, n, (0.1, 0.1), 2.0, 200e3)
    rex, _, _ = O.simulate_fresnel_as(V, psi, H, 2.0, 200e3, return_wavefronts=False)
    plan = wap.get_plan(n, n, 1, _lib.WAP_OP_FRESNEL_AS)
    old = plan.config()
    try:
        for cfg in autotune.candidates(n, n):
            plan.set_config(*cfg)
            ex, _, _ = wap.simulate_fresnel_as(V, psi, H, 2.0, 200e3, return_wavefronts=False)
            assert rel(np_(ex), rex) < TOL, cfg
    finally:
        plan.set_config(*old)


def test_unsupported_size_raises(wap):
    """Sides beyond 1024 that are not powers of two (and below 17) are not
    implemented; every other size is (the Bluestein path covers 17..1024)."""
    for ny, nx in ((12, 64), (1500, 64)):
        with pytest.raises(ValueError, match="unsupported grid"):
            wap.simulate_fresnel_as(np.zeros((1, ny, nx), np.float32), np.ones((ny, nx), np.complex64),
                                    np.ones((ny, nx), np.complex64), 1.0, 200e3)


def test_pinned_host_inputs_upload_on_a_side_stream(wap):
    """Pinned host arrays (uploaded on a side stream that the caller's stream
    waits for) give the same result as device arrays, also when the upload is
    queued behind a long call on the caller's stream."""
    import wideanglepropagation_b200.synthetic as S
    ws = S.batched_scan(0, small=True)
    w = ws[1]
    H = wap.angular_spectrum_propagation_kernel(w.ny, w.nx, (w.ps, w.ps), w.dz, w.energy)
    dev = torch.device("cuda")
    Vd, pd = torch.as_tensor(w.potential, device=dev), torch.as_tensor(w.probe, device=dev)
    qd, dd = torch.as_tensor(w.positions, device=dev), torch.as_tensor(w.draw_of_probe, device=dev)
    ref_ex, ref_dp, _ = wap.simulate_fresnel_as(Vd, pd, H, w.dz, w.energy, positions=qd, draw=dd,
                                                return_wavefronts=False)
    Vh = torch.from_numpy(w.potential).pin_memory()
    big = torch.zeros((16, 512, 512), dtype=torch.float32, device=dev)
    Hb = wap.fresnel_propagation_kernel(512, 512, (0.05, 0.05), 2.0, 300e3)
    for _ in range(2):
        wap.simulate_fresnel_as(big, torch.ones((512, 512), dtype=torch.complex64, device=dev), Hb, 2.0, 300e3,
                                return_wavefronts=False)   # keeps the caller's stream busy
        ex, dp, _ = wap.simulate_fresnel_as(Vh, torch.from_numpy(w.probe).pin_memory(), H, w.dz, w.energy,
                                            positions=torch.from_numpy(w.positions).pin_memory(),
                                            draw=torch.from_numpy(w.draw_of_probe).pin_memory(),
                                            return_wavefronts=False)
        assert torch.equal(ex, ref_ex) and torch.equal(dp, ref_dp)


def test_wpm_strong_phase(wap):
    """A strong potential in thick slices: bin phases well above 0.5 rad, so the
    column pass's exp(i phi) takes its sincosf branch next to the Taylor one."""
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(12)
    n, ps, dz, E = 64, 0.05, 5.0, 300e3
    V = rng.uniform(0, 2000, (3, n, n)).astype(np.float32)
    psi = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))).astype(np.complex64)
    ex, dp, _ = wap.simulate_wpm(V, psi, dz, E, (ps, ps), 8, 1.0)
    rex, rdp, _ = O.simulate_wpm(V, psi, dz, E, (ps, ps), 8, 1.0)
    assert rel(np_(ex), rex) < TOL
    assert rel(np_(dp), rdp) < TOL


@pytest.mark.parametrize("ny,nx", [(64, 64), (1024, 1024), (128, 512)])
def test_every_launch_shape_other_grids(wap, ny, nx):
    """Every launch shape the autotuner may pick (4, 8 or 16 elements per
    thread, 2 to 32 columns per column CTA), on a small, a large and a
    non-square grid, against the oracle."""
    from wideanglepropagation_b200 import autotune, _lib
    from oracle import propagation_oracle as O
    rng = np.random.default_rng(13)
    V = rng.uniform(0, 30, (2, ny, nx)).astype(np.float32)
    psi = (rng.normal(size=(ny, nx)) + 1j * rng.normal(size=(ny, nx))).astype(np.complex64)
    H = O.angular_spectrum_propagation_kernel(ny, nx, (0.05, 0.05), 2.0, 300e3)
    rex, rdp, _ = O.simulate_fresnel_as(V, psi, H, 2.0, 300e3, return_wavefronts=False)
    plan = wap.get_plan(ny, nx, 1, _lib.WAP_OP_FRESNEL_AS)
    old = plan.config()
    tried = 0
    try:
        for cfg in autotune.candidates(ny, nx):
            try:
                plan.set_config(*cfg)
            except ValueError:
                continue   # a shape the kernels cannot launch on this grid
            ex, dp, _ = wap.simulate_fresnel_as(V, psi, H, 2.0, 300e3, return_wavefronts=False)
            assert rel(np_(ex), rex) < TOL, cfg
            assert rel(np_(dp), rdp) < TOL, cfg
            tried += 1
    finally:
        plan.set_config(*old)
    assert tried > 0


def test_every_wpm_launch_shape(wap):
    """The WPM passes at every launch shape a WPM plan accepts (8 or 16
    elements per thread, 2 to 32 columns per column CTA) against the oracle."""
    from wideanglepropagation_b200 import autotune, _lib
    from oracle import propagation_oracle as O
    n, K = 128, 8
    rng = np.random.default_rng(14)
    V = rng.uniform(0, 60, (3, n, n)).astype(np.float32)
    psi = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))).astype(np.complex64)
    rex, rdp, _ = O.simulate_wpm(V, psi, 2.0, 300e3, (0.05, 0.05), K, 1.0, return_wavefronts=False)
    plan = wap.get_plan(n, n, 1, _lib.WAP_OP_WPM, K)
    old = plan.config()
    with pytest.raises(ValueError):
        plan.set_config(4, 8, 8)
    tried = 0
    try:
        for cfg in autotune.candidates(n, n):
            try:
                plan.set_config(*cfg)
            except ValueError:
                continue   # 4 elements per thread: Fresnel/AS plans only
            ex, dp, _ = wap.simulate_wpm(V, psi, 2.0, 300e3, (0.05, 0.05), K, 1.0, return_wavefronts=False)
            assert rel(np_(ex), rex) < TOL, cfg
            assert rel(np_(dp), rdp) < TOL, cfg
            tried += 1
    finally:
        plan.set_config(*old)
    assert tried > 0
