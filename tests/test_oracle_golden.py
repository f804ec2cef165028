"""Pin the NumPy oracle against fixtures produced by the reference's own code.

tests/golden/make_golden.py executed the reference propagation.py (with NumPy
standing in for jax.numpy); these tests require the restatement in
oracle/propagation_oracle.py to reproduce those outputs.
"""
import numpy as np
import pytest

from oracle import propagation_oracle as O


def close(a, b, tol=1e-12):
    a = np.asarray(a)
    b = np.asarray(b)
    assert a.shape == b.shape
    err = np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300)
    assert err < tol, err


def test_constants(golden):
    for E in (80e3, 200e3, 300e3):
        assert O.energy2wavelength(E) == pytest.approx(float(golden[f"lam_{int(E)}"]), rel=1e-15)
    assert O.electron_rest_energy() == pytest.approx(float(golden["E0"]), rel=1e-15)
    close(O.electron_refractive_index(golden["nref_V"], 200e3), golden["nref_n_200k"], 1e-15)
    # refractive index minus one: stable FP32 form vs FP64 reference
    dn64 = golden["nref_n_200k"] - 1
    dn32 = O.refractive_index_minus_one(golden["nref_V"].astype(np.float32), 200e3, "fp32_stable")
    assert np.max(np.abs(dn32 - dn64) / np.maximum(np.abs(dn64), 1e-12)) < 3e-7


def test_transfer_functions(golden):
    close(O.fresnel_propagation_kernel(48, 64, (0.11, 0.09), 2.0, 200e3), golden["H_fres_48x64"])
    close(O.angular_spectrum_propagation_kernel(48, 64, (0.11, 0.09), 1.5, 300e3), golden["H_as_48x64"])
    close(O.angular_spectrum_propagation_kernel(32, 32, (0.01, 0.01), 0.7, 300e3), golden["H_as_evan_32x32"])


def test_fresnel_multislice(golden):
    ny, nx, ps, N, dz, E = golden["fres_meta"]
    ex, dp, st = O.simulate_fresnel_as(golden["fres_V"], golden["fres_probe"], golden["fres_H"], dz, E)
    close(ex, golden["fres_exit"])
    close(dp, golden["fres_dp"])
    close(st, golden["fres_stack"])


def test_as_multislice_nonsquare(golden):
    ny, nx, ps, N, dz, E = golden["as_meta"]
    ex, dp, st = O.simulate_fresnel_as(golden["as_V"], golden["as_probe"], golden["as_H"], dz, E)
    close(ex, golden["as_exit"])
    close(dp, golden["as_dp"])
    close(st, golden["as_stack"])


def test_fresnel_fp32_reference_mode(golden):
    ex, dp, _ = O.simulate_fresnel_as(golden["fres_V"].astype(np.float32), golden["fres_probe"],
                                      golden["fres_H"], 2.0, 200e3, mode="fp32")
    close(ex, golden["fres32_exit"], 2e-6)
    close(dp, golden["fres32_dp"], 2e-6)


@pytest.mark.parametrize("K,p", [(16, 1.0), (8, 2.0)])
def test_wpm_multislice(golden, K, p):
    ny, nx, ps, N, dz, E = golden["wpm_meta"]
    ex, dp, st = O.simulate_wpm(golden["wpm_V"], golden["wpm_probe"], dz, E, (ps, ps),
                                n_bins=K, power_spacing=p)
    close(ex, golden[f"wpm_K{K}_exit"])
    close(dp, golden[f"wpm_K{K}_dp"])
    close(st, golden[f"wpm_K{K}_stack"])


def test_wpm_step_aux_outputs(golden):
    ny, nx, ps, N, dz, E = golden["wpm_meta"]
    nmap = O.electron_refractive_index(golden["wpm_V"][0], E)
    nw, w, iL, nrefs = O.wpm_step_adaptive(golden["wstep_wave0"], nmap, dz, E, (ps, ps), 12, 2.0)
    close(nw, golden["wstep_out"])
    close(w, golden["wstep_w"])
    assert np.array_equal(iL, golden["wstep_idxL"])
    close(nrefs, golden["wstep_nrefs"], 1e-15)


def test_wpm_constant_slice_denominator_guard(golden):
    ny, nx, ps, N, dz, E = golden["wpm_meta"]
    nconst = O.electron_refractive_index(np.full((int(ny), int(nx)), 7.5), E)
    nw, w, iL, _ = O.wpm_step_adaptive(golden["wstep_wave0"], nconst, dz, E, (ps, ps), 4, 1.0)
    close(nw, golden["wconst_out"])
    assert np.array_equal(iL, golden["wconst_idxL"])
    assert np.all(w == golden["wconst_w"])


def test_move_probe(golden):
    for pos, want in zip(golden["mp_pos"], golden["mp_out"]):
        assert np.array_equal(O.move_probe(golden["mp_in"], tuple(pos)), want)


def test_detector_crop(golden):
    assert np.array_equal(O.downsample_to_max_angle(golden["crop_in"], (0.1, 0.1), 0.025, 40.0), golden["crop_odd"])
    assert np.array_equal(O.downsample_to_max_angle(golden["crop_in"], (0.1, 0.12), 0.025, 50.0, parity="even"),
                          golden["crop_even"])


def test_naive_wpm_step(golden):
    ny, nx, ps, dz, E = golden["naive_meta"]
    out = O.wpm_step(golden["naive_wave"], golden["naive_n"], dz, E, (ps, ps))
    assert O.rel_l2(out, golden["naive_out"]) < 1e-12


def test_1d_helpers(golden):
    n, dx, dy, k0 = golden["l1_meta"]
    kx = O.get_kx_1d(int(n), dx)
    assert np.array_equal(kx, golden["l1_kx"])
    assert O.rel_l2(O.fresnel_kernel_1d(kx ** 2, k0, dy), golden["l1_Hf"]) < 1e-14
    assert O.rel_l2(O.angular_spectrum_kernel_1d(kx ** 2, k0, dy), golden["l1_Ha"]) < 1e-14
    assert O.rel_l2(O.propagate_1d(golden["l1_psi"], golden["l1_Hf"]), golden["l1_prop_f"]) < 1e-13
    assert O.rel_l2(O.propagate_1d(golden["l1_psi"], golden["l1_Ha"]), golden["l1_prop_a"]) < 1e-13
    psik = np.fft.fft(golden["l1_psi"][0])
    assert O.rel_l2(O.wpm_kernel_1d(psik, 1.3, k0, kx ** 2, dy), golden["l1_wpm1"]) < 1e-13
    assert O.rel_l2(O.wpm_kernel_1d_vmap(psik, golden["l1_nvals"], k0, kx ** 2, dy), golden["l1_wpmv"]) < 1e-13


def test_lippmann_schwinger(golden):
    k0, h, n = golden["ls_meta"]
    n = int(n)
    Khat, emb = O.build_lippmann_schwinger_kernel_2d(k0, h, h, n, n)
    assert emb == (2 * n, 2 * n)
    assert O.rel_l2(Khat, golden["ls_Khat"]) < 1e-13
    assert O.rel_l2(O.apply_convolution(golden["ls_src"], Khat, emb, (n, n)), golden["ls_conv"]) < 1e-13
    E, ps, tol = golden["ls_solve_meta"]
    psi = O.solve_scattering_2d_lippmann_schwinger(golden["ls_V"], E, ps, gmres_tol=tol)
    assert O.rel_l2(psi, golden["ls_psi"]) < 1e-10


@pytest.mark.parametrize("case", ["fres", "as"])
def test_torch_gradient_oracle_pinned(golden, case):
    """The complex128 torch restatement behind the gradient tests reproduces
    the reference's own Fresnel and (non-square) angular-spectrum outputs."""
    import torch
    from oracle import torch_oracle as T
    ny, nx, ps, N, dz, E = golden[f"{case}_meta"]
    ex, dp = T.simulate(torch.tensor(golden[f"{case}_V"], dtype=torch.float64), golden[f"{case}_probe"],
                        golden[f"{case}_H"], dz, E)
    close(ex[0].numpy(), golden[f"{case}_exit"])
    close(dp[0].numpy(), golden[f"{case}_dp"])


def test_torch_gradient_oracle_positions():
    """With probe positions the torch restatement matches the NumPy oracle's
    move_probe (pinned to the reference's roll above) probe for probe."""
    import torch
    from oracle import torch_oracle as T
    rng = np.random.default_rng(3)
    n, N, dz, E = 32, 3, 2.0, 300e3
    V = rng.uniform(0, 30, (N, n, n))
    probe = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    H = O.fresnel_propagation_kernel(n, n, (0.1, 0.1), dz, E)
    pos = np.array([[3, 30], [16, 16], [31, 0]])
    ex, dp = T.simulate(torch.tensor(V), probe, H, dz, E, pos)
    for b, p in enumerate(pos):
        rex, rdp, _ = O.simulate_fresnel_as(V, O.move_probe(probe, tuple(p)), H, dz, E, return_wavefronts=False)
        close(ex[b].numpy(), rex)
        close(dp[b].numpy(), rdp)
