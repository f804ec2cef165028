"""Device probe builder (wap_aperture_probe) against its host restatement, and
per-position accumulation of diffraction patterns (wap_pattern_accumulate)
against the summed FP64 oracle patterns.

Probe tolerance: rel-L2 <= 1e-6 (one complex64 inverse transform of a float64
spectrum).  Accumulated patterns: rel-L2 <= 1e-5 against the sum of the
oracle's per-probe patterns (the multislice bar), and bit-exact against
summing the library's own per-probe patterns in probe order.
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
    from oracle.propagation_oracle import rel_l2
    return rel_l2(a, b)


@pytest.mark.parametrize("ny,nx,ps,E,alpha,df,centred", [
    (256, 256, 0.1, 200e3, 20.0, 0.0, True),        # the Fresnel configuration's probe
    (256, 256, 0.05, 300e3, 25.0, -50.0, True),     # the batched scan's probe
    (512, 512, 0.05, 300e3, 25.0, -50.0, False),
    (128, 256, 0.07, 80e3, 30.0, 120.0, True),      # non-square grid
])
def test_aperture_probe_matches_host(wap, ny, nx, ps, E, alpha, df, centred):
    S = wap.synthetic
    ref = S.aperture_probe(ny, nx, ps, E, alpha, df, centred=centred, dtype=np.complex128)
    p = wap.aperture_probe(ny, nx, ps, E, alpha, df, centred=centred)
    assert p.dtype == torch.complex64 and p.shape == (ny, nx)
    assert rel(p.cpu().numpy(), ref) < 1e-6
    assert abs(float((p.abs() ** 2).sum()) / (ny * nx) - 1) < 1e-5


def test_aperture_probe_in_a_scan(wap):
    """A scan started from the device probe equals one started from the host
    probe to float rounding of the probe."""
    w = wap.synthetic.batched_scan_class(2, 128, 4, 3, 1)
    H = wap.angular_spectrum_propagation_kernel(128, 128, (w.ps, w.ps), w.dz, w.energy)
    pd = wap.aperture_probe(128, 128, w.ps, w.energy, 25.0, -50.0)
    ex_d, dp_d, _ = wap.simulate_fresnel_as(w.potential[0], pd, H, w.dz, w.energy, positions=w.positions,
                                            return_wavefronts=False)
    ex_h, dp_h, _ = wap.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy, positions=w.positions,
                                            return_wavefronts=False)
    assert rel(ex_d.cpu().numpy(), ex_h.cpu().numpy()) < 1e-6
    assert rel(dp_d.cpu().numpy(), dp_h.cpu().numpy()) < 1e-6


@pytest.mark.parametrize("n,side,draws", [(128, 3, 3), (256, 2, 4)])
def test_accumulate_draws_per_position(wap, n, side, draws):
    """Probes b = d * P + p (draw d of position p): the patterns of each
    position's draws summed in float32, on the scheduler path; against the
    sum of the FP64 oracle's patterns and bit-exact against summing the
    library's per-probe patterns in probe order."""
    from oracle import propagation_oracle as O
    w = wap.synthetic.batched_scan_class(6, n, 5, side, draws)
    P = side * side
    B = w.n_probes
    assert B == P * draws and B >= 8
    acc = np.arange(B) % P
    H = wap.angular_spectrum_propagation_kernel(n, n, (w.ps, w.ps), w.dz, w.energy)
    args = (w.potential, w.probe, H, w.dz, w.energy)
    kw = dict(positions=w.positions, draw=w.draw_of_probe, return_wavefronts=False)
    ex, dp_acc, _ = wap.simulate_fresnel_as(*args, accumulate=acc, **kw)
    ex1, dp, _ = wap.simulate_fresnel_as(*args, **kw)
    assert dp_acc.shape == (P, n, n) and ex.shape == (B, n, n)
    assert torch.equal(ex, ex1)
    manual = dp[0:P].clone()
    for d in range(1, draws):
        manual += dp[d * P:(d + 1) * P]
    assert torch.equal(dp_acc, manual)
    Hh = H.cpu().numpy()
    for p in (0, P - 1):
        ref = 0
        for d in range(draws):
            b = d * P + p
            p0 = O.move_probe(w.probe, tuple(w.positions[b]))
            _, rdp, _ = O.simulate_fresnel_as(w.potential[w.draw_of_probe[b]], p0, Hh, w.dz, w.energy,
                                              return_wavefronts=False)
            ref = ref + rdp
        assert rel(dp_acc[p].cpu().numpy(), ref) < 1e-5


def test_accumulate_irregular_groups_and_window(wap):
    """Irregular groups (sizes 0..3, one empty pattern index), a detector
    window and the per-pass path (fewer than 8 probes); WPM as well."""
    w = wap.synthetic.batched_scan_class(8, 128, 3, 2, 1)
    H = wap.angular_spectrum_propagation_kernel(128, 128, (w.ps, w.ps), w.dz, w.energy)
    acc = np.array([2, 0, 2, 2])      # pattern 1 gets no probe: zeros
    kw = dict(positions=w.positions, return_wavefronts=False, max_angle=30.0, sampling=(w.ps, w.ps))
    _, dp, _ = wap.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy, **kw)
    _, dpa, _ = wap.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy, accumulate=acc, **kw)
    assert dpa.shape == (3,) + tuple(dp.shape[1:])
    assert torch.equal(dpa[0], dp[1])
    assert torch.equal(dpa[1], torch.zeros_like(dp[0]))
    assert torch.equal(dpa[2], dp[0] + dp[2] + dp[3])
    _, wdp, _ = wap.simulate_wpm(w.potential[0], w.probe, w.dz, w.energy, (w.ps, w.ps), 8, 1.0,
                                 positions=w.positions, return_wavefronts=False)
    _, wdpa, _ = wap.simulate_wpm(w.potential[0], w.probe, w.dz, w.energy, (w.ps, w.ps), 8, 1.0,
                                  positions=w.positions, return_wavefronts=False, accumulate=[0, 0, 1, 1])
    assert torch.equal(wdpa, torch.stack([wdp[0] + wdp[1], wdp[2] + wdp[3]]))


def test_accumulate_rejects_bad_indices(wap):
    w = wap.synthetic.batched_scan_class(8, 128, 2, 2, 1)
    H = wap.angular_spectrum_propagation_kernel(128, 128, (w.ps, w.ps), w.dz, w.energy)
    for bad in ([0, 1, 2], [0, -1, 1, 1], [0.5, 1, 1, 1]):
        with pytest.raises(ValueError):
            wap.simulate_fresnel_as(w.potential[0], w.probe, H, w.dz, w.energy, positions=w.positions,
                                    return_wavefronts=False, accumulate=bad)
