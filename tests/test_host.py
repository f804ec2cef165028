"""Host-side logic that needs no GPU: physics scalars, synthetic inputs,
autotune candidates, detector crop, API guards."""
import numpy as np
import pytest
import torch

import wideanglepropagation_b200 as wap
from wideanglepropagation_b200 import autotune, physics, synthetic
from oracle import propagation_oracle as O


def test_physics_matches_oracle():
    for E in (80e3, 200e3, 300e3):
        assert physics.energy2wavelength(E) == O.energy2wavelength(E)
        for v in (-20.0, 0.0, 1.0, 37.5, 400.0):
            n = O.electron_refractive_index(np.float64(v), E)
            assert physics.refractive_index_minus_one(v, E) == pytest.approx(n - 1, rel=1e-9, abs=1e-15)
    assert physics.energy2wavelength(200e3) == pytest.approx(0.0250793, rel=1e-5)
    assert physics.energy2wavelength(300e3) == pytest.approx(0.0196875, rel=1e-5)
    # sigma(200 kV) ~ 7.29e-4 / (V A)
    assert physics.energy2sigma(200e3) == pytest.approx(7.29e-4, rel=2e-3)


def test_synthetic_shapes_and_determinism():
    w = synthetic.plain_fresnel(0, n_slices=3)
    assert w.potential.shape == (1, 3, 256, 256) and w.potential.dtype == np.float32
    assert np.array_equal(w.potential, synthetic.plain_fresnel(0, n_slices=3).potential)
    assert abs(np.sum(np.abs(w.probe) ** 2) / (256 * 256) - 1) < 1e-5
    # peak projected potential of one atom ~ amp / dz volts
    assert 5 < w.potential.max() < 40
    cls = synthetic.batched_scan(0, small=True)
    assert [c.n_probes for c in cls] == [32, 4]
    assert cls[0].positions.dtype == np.int32 and cls[0].draw_of_probe.max() == 1


def test_gaussian_slice_is_separable_sum():
    ny, nx, ps = 32, 48, 0.1
    c = np.array([[1.0, 2.0], [3.1, 4.4]])
    g = synthetic.gaussian_slice(ny, nx, ps, c, 10.0, 0.3)
    y = np.arange(ny) * ps
    x = np.arange(nx) * ps
    want = np.zeros((ny, nx))
    for cy, cx in c:
        dy = (y - cy + ny * ps / 2) % (ny * ps) - ny * ps / 2
        dx = (x - cx + nx * ps / 2) % (nx * ps) - nx * ps / 2
        want += 10.0 * np.exp(-(dy[:, None] ** 2 + dx[None, :] ** 2) / 0.18)
    assert np.allclose(g, want)


def test_autotune_candidates_are_valid():
    for n in (32, 64, 256, 512, 1024, 2048):
        cands = autotune.candidates(n, n)
        assert cands
        for row_e, col_e, w in cands:
            assert n // row_e <= 256 and w * (n // col_e) <= 512 and w <= n


def test_detector_crop_matches_oracle(golden):
    assert wap.max_angle_gpts((64, 64), (0.1, 0.1), 0.025, 40.0) == O.max_angle_gpts((64, 64), (0.1, 0.1), 0.025, 40.0)
    assert np.array_equal(wap.downsample_to_max_angle(golden["crop_in"], (0.1, 0.1), 0.025, 40.0), golden["crop_odd"])
    t = torch.as_tensor(golden["crop_in"])
    assert np.array_equal(wap.downsample_to_max_angle(t, (0.1, 0.12), 0.025, 50.0, parity="even").numpy(),
                          golden["crop_even"])


@pytest.mark.parametrize("shape,sampling,energy,angle,parity", [
    ((64, 64), (0.1, 0.1), 200e3, 40.0, "odd"),
    ((128, 64), (0.05, 0.08), 300e3, 25.0, "even"),
    ((256, 256), (0.05, 0.05), 300e3, 60.0, "odd"),
    ((32, 32), (0.2, 0.2), 80e3, 1e5, "odd"),
])
def test_detector_window_is_the_oracle_crop(shape, sampling, energy, angle, parity):
    """The fused crop's window selects the same pixels as the oracle's
    downsample_to_max_angle (propagation.py:424-439) of the full pattern."""
    idx = np.arange(shape[0] * shape[1]).reshape(shape)
    ref = O.downsample_to_max_angle(idx, sampling, O.energy2wavelength(energy), angle, parity=parity)
    win = wap.detector_window(shape, sampling, energy, angle, parity)
    if win is None:
        assert ref.shape == shape
        return
    y0, x0, ny, nx = win
    assert np.array_equal(idx[y0:y0 + ny, x0:x0 + nx], ref)


def test_move_probe_matches_golden(golden):
    for pos, want in zip(golden["mp_pos"], golden["mp_out"]):
        assert np.array_equal(wap.move_probe(golden["mp_in"], tuple(pos)).numpy(), want)


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback():
    with pytest.raises(RuntimeError, match="no CPU path"):
        wap.simulate_fresnel_as(np.zeros((1, 64, 64), np.float32), np.ones((64, 64), np.complex64),
                                np.ones((64, 64), np.complex64), 1.0, 2e5)
    with pytest.raises(RuntimeError, match="no CPU path"):
        wap.fresnel_propagation_kernel(64, 64, (0.1, 0.1), 1.0, 2e5)


def test_atom_lists_reproduce_the_host_potentials():
    """The atom lists behind the synthetic workloads give the same potentials
    (the device builder is fed these lists)."""
    w = synthetic.batched_scan_class(3, 64, 5, 2, 2)
    pos, rows = synthetic.batched_scan_class_atoms(3, 64, 5, 2, 2)
    V = np.stack([synthetic.gaussian_slice(64, 64, 0.05, pos[rows == r], 25.0, 0.25) for r in range(10)])
    assert np.allclose(V.reshape(2, 5, 64, 64) / 1.3575, w.potential, rtol=1e-6, atol=1e-6 * np.abs(V).max())


def test_balanced_probe_groups():
    """Probe groups split a batch evenly: 1024 probes at a nominal 111 make 9
    groups of 114, 64 at 28 make 2 of 32; a batch below the size is one group."""
    assert autotune.balanced_group(111, 1024) == 114
    assert autotune.balanced_group(28, 64) == 32
    assert autotune.balanced_group(444, 9) == 9
    assert autotune.balanced_group(0, 100) == 0
    for g in (7, 28, 111):
        for B in (1, 9, 64, 100, 1024):
            G = autotune.balanced_group(g, B)
            ng = -(-B // G)
            assert 1 <= G <= B
            if B >= g:
                assert g / 2 < G < 2 * g
            assert G - ng <= B - (ng - 1) * G <= G   # the last group is within ng of the others
