"""Generate golden fixtures by executing the reference's own propagation.py.

The reference module (``wide_angle_propagation/propagation.py``) imports jax,
abtem and ase at module level (propagation.py:1-6); none of them is installed
here.  This script installs minimal stand-ins *for this process only*:

* ``jax.numpy``  -> NumPy (every jnp call on the multislice path has the same
  name and semantics in NumPy: fft, meshgrid, sqrt, exp, clip, searchsorted,
  take_along_axis, where, roll, stack, linspace);
* ``jax.jit``    -> identity (static_argnames accepted and ignored);
* ``jax.vmap``   -> a Python loop over the mapped axis + np.stack;
* ``jnp.zeros``  -> NumPy arrays that also offer JAX's functional
  ``.at[idx].set(v)`` (used by the Lippmann-Schwinger convolution);
* ``jax.scipy.sparse.linalg.gmres`` -> SciPy's restarted GMRES with the same
  relative tolerance and restart length (the solve is therefore pinned to
  within that tolerance, the kernel and the convolution exactly);
* ``ase.units``  -> ASE's default CODATA-2014 constants;
* ``abtem.*``    -> empty placeholders (only used by get_abtem_transmit, which
  is not on the path).

It then loads the reference file read-only from the reference checkout, runs
the path functions on small seeded float64/complex128 inputs (the notebooks
run with ``jax_enable_x64``) and on float32/complex64 inputs, and writes
``tests/golden/golden.npz``.  Re-run with
``python tests/golden/make_golden.py path/to/reference`` (the checkout of
WideAnglePropagation), or with the path in the environment variable
``WAP_REFERENCE_ROOT``.
"""
from __future__ import annotations

import importlib.util
import math
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _install_stubs():
    jax = types.ModuleType("jax")

    def jit(fun=None, **kw):
        if fun is None:
            return lambda f: f
        return fun

    def vmap(fun, in_axes=0):
        def mapped(*args):
            axes = in_axes if isinstance(in_axes, (tuple, list)) else [in_axes] * len(args)
            n = None
            for a, ax in zip(args, axes):
                if ax is not None:
                    n = np.shape(a)[ax]
            outs = []
            for i in range(n):
                call = [np.take(a, i, axis=ax) if ax is not None else a
                        for a, ax in zip(args, axes)]
                outs.append(fun(*call))
            return np.stack(outs)
        return mapped

    jax.jit = jit
    jax.vmap = vmap
    jax.config = types.SimpleNamespace(update=lambda *a, **k: None)
    jnp = types.ModuleType("jax.numpy")
    for name in dir(np):
        if not name.startswith("__"):
            setattr(jnp, name, getattr(np, name))
    jnp.fft = np.fft

    class _AtArray(np.ndarray):
        """ndarray with JAX's functional index update, a.at[idx].set(v)."""
        @property
        def at(self):
            arr = self

            class _Idx:
                def __getitem__(self, idx):
                    class _Set:
                        def set(self, v):
                            out = np.array(arr)
                            out[idx] = v
                            return out.view(_AtArray)
                    return _Set()
            return _Idx()

    jnp.zeros = lambda *a, **k: np.zeros(*a, **k).view(_AtArray)
    jax.numpy = jnp
    sys.modules["jax"] = jax
    sys.modules["jax.numpy"] = jnp

    import scipy.sparse.linalg as _sla
    jsp = types.ModuleType("jax.scipy")
    jsp_sparse = types.ModuleType("jax.scipy.sparse")
    jsp_linalg = types.ModuleType("jax.scipy.sparse.linalg")

    def gmres(A, b, x0=None, tol=1e-5, atol=0.0, restart=20, maxiter=None, M=None):
        b = np.asarray(b)
        op = _sla.LinearOperator((b.size, b.size), matvec=lambda v: np.asarray(A(v)), dtype=np.complex128)
        x, info = _sla.gmres(op, b, rtol=tol, atol=atol, restart=restart, maxiter=maxiter)
        return x, info

    jsp_linalg.gmres = gmres
    jsp_sparse.linalg = jsp_linalg
    jsp.sparse = jsp_sparse
    jax.scipy = jsp
    sys.modules["jax.scipy"] = jsp
    sys.modules["jax.scipy.sparse"] = jsp_sparse
    sys.modules["jax.scipy.sparse.linalg"] = jsp_linalg

    abtem = types.ModuleType("abtem")
    ms = types.ModuleType("abtem.multislice")
    ms._generate_potential_configurations = None
    aa = types.ModuleType("abtem.antialias")
    aa.AntialiasAperture = None
    abtem.multislice = ms
    abtem.antialias = aa
    sys.modules["abtem"] = abtem
    sys.modules["abtem.multislice"] = ms
    sys.modules["abtem.antialias"] = aa

    ase = types.ModuleType("ase")
    units = types.ModuleType("ase.units")
    # ASE default CODATA 2014 set (ase/units.py)
    units._c = 299792458.0
    units._hplanck = 6.626070040e-34
    units._e = 1.6021766208e-19
    units._me = 9.10938356e-31
    units._amu = 1.660539040e-27
    units._mu0 = 4.0e-7 * math.pi
    units._eps0 = 1 / units._mu0 / units._c ** 2
    units.Ang = 1.0
    units.eV = 1.0
    units.J = 1 / units._e
    units.C = 1 / units._e
    units.kg = 1 / units._amu
    units.s = 1e10 * math.sqrt(units._e / units._amu)
    ase.units = units
    sys.modules["ase"] = ase
    sys.modules["ase.units"] = units


def load_reference(ref_root: str):
    _install_stubs()
    path = os.path.join(ref_root, "wide_angle_propagation", "propagation.py")
    spec = importlib.util.spec_from_file_location("_ref_propagation", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _gauss_stack(rng, n_slices, ny, nx, ps, n_atoms, amp, sigma):
    """Seeded sum-of-Gaussians projected potential (V*A), periodic wrap."""
    y = np.arange(ny) * ps
    x = np.arange(nx) * ps
    Ly, Lx = ny * ps, nx * ps
    V = np.zeros((n_slices, ny, nx))
    for s in range(n_slices):
        for cy, cx in rng.uniform(0, 1, (n_atoms, 2)) * (Ly, Lx):
            dy = (y - cy + Ly / 2) % Ly - Ly / 2
            dx = (x - cx + Lx / 2) % Lx - Lx / 2
            V[s] += amp * np.exp(-(dy[:, None] ** 2 + dx[None, :] ** 2) / (2 * sigma ** 2))
    return V


def _probe(ny, nx, ps, lam, alpha, rng=None):
    fy = np.fft.fftfreq(ny, ps)
    fx = np.fft.fftfreq(nx, ps)
    k = np.sqrt(fy[:, None] ** 2 + fx[None, :] ** 2)
    aperture = (k * lam < alpha).astype(np.complex128)
    if rng is not None:
        aperture *= np.exp(1j * rng.uniform(-0.3, 0.3, aperture.shape))
    p = np.fft.fftshift(np.fft.ifft2(aperture))
    return p / np.sqrt(np.sum(np.abs(p) ** 2))


def make(ref_root: str, out: str):
    ref = load_reference(ref_root)
    rng = np.random.default_rng(1234)
    g = {}

    # --- constants -------------------------------------------------------
    for E in (80e3, 200e3, 300e3):
        g[f"lam_{int(E)}"] = np.float64(ref.energy2wavelength(E))
    g["E0"] = np.float64(ref.electron_rest_energy())
    vv = np.linspace(-50, 400, 257)
    g["nref_V"] = vv
    g["nref_n_200k"] = np.asarray(ref.electron_refractive_index(vv, 200e3))

    # --- transfer functions (non-square, anisotropic sampling) -----------
    g["H_fres_48x64"] = np.asarray(ref.fresnel_propagation_kernel(48, 64, (0.11, 0.09), 2.0, 200e3))
    g["H_as_48x64"] = np.asarray(ref.angular_spectrum_propagation_kernel(48, 64, (0.11, 0.09), 1.5, 300e3))
    # evanescent components present (coarse lambda relative to sampling)
    g["H_as_evan_32x32"] = np.asarray(ref.angular_spectrum_propagation_kernel(32, 32, (0.01, 0.01), 0.7, 300e3))

    # --- Fresnel multislice, fp64 ----------------------------------------
    ny, nx, ps, N, dz, E = 64, 64, 0.1, 5, 2.0, 200e3
    lam = ref.energy2wavelength(E)
    V = _gauss_stack(rng, N, ny, nx, ps, 6, 20.0, 0.3) / dz
    probe = _probe(ny, nx, ps, lam, 0.02, rng)
    H = np.asarray(ref.fresnel_propagation_kernel(ny, nx, (ps, ps), dz, E))
    ex, dp, st = ref.simulate_fresnel_as(V, probe, H, dz, E)
    g.update(fres_V=V, fres_probe=probe, fres_H=H, fres_exit=np.asarray(ex),
             fres_dp=np.asarray(dp), fres_stack=np.asarray(st),
             fres_meta=np.array([ny, nx, ps, N, dz, E]))

    # --- AS multislice, non-square fp64 -----------------------------------
    ny, nx, ps, N, dz, E = 32, 64, 0.05, 4, 1.3575, 300e3
    lam = ref.energy2wavelength(E)
    V = _gauss_stack(rng, N, ny, nx, ps, 5, 25.0, 0.25) / dz
    probe = _probe(ny, nx, ps, lam, 0.025, rng)
    H = np.asarray(ref.angular_spectrum_propagation_kernel(ny, nx, (ps, ps), dz, E))
    ex, dp, st = ref.simulate_fresnel_as(V, probe, H, dz, E)
    g.update(as_V=V, as_probe=probe, as_H=H, as_exit=np.asarray(ex),
             as_dp=np.asarray(dp), as_stack=np.asarray(st),
             as_meta=np.array([ny, nx, ps, N, dz, E]))

    # --- Fresnel, FP32 inputs (reference evaluated in single precision) ---
    V32 = g["fres_V"].astype(np.float32)
    ex, dp, st = ref.simulate_fresnel_as(V32, g["fres_probe"].astype(np.complex64),
                                         g["fres_H"].astype(np.complex64), 2.0, 200e3)
    g.update(fres32_exit=np.asarray(ex), fres32_dp=np.asarray(dp))

    # --- WPM step + multislice (fp64), both bin spacings -------------------
    ny, nx, ps, N, dz, E = 32, 64, 0.05, 3, 2.04, 300e3
    V = _gauss_stack(rng, N, ny, nx, ps, 5, 80.0, 0.2) / dz
    probe = np.ones((ny, nx), np.complex128)
    for K, p in ((16, 1.0), (8, 2.0)):
        ex, dp, st = ref.simulate_wpm(V, probe, dz, E, (ps, ps), n_bins=K, power_spacing=p)
        g[f"wpm_K{K}_exit"] = np.asarray(ex)
        g[f"wpm_K{K}_dp"] = np.asarray(dp)
        g[f"wpm_K{K}_stack"] = np.asarray(st)
    g.update(wpm_V=V, wpm_probe=probe, wpm_meta=np.array([ny, nx, ps, N, dz, E]))
    # a single adaptive step with a convergent, off-centre probe and its
    # auxiliary outputs (weights, left indices, reference indices)
    wave0 = _probe(ny, nx, ps, ref.energy2wavelength(E), 0.03, rng)
    nmap = ref.electron_refractive_index(V[0], E)
    nw, w, iL, nrefs = ref.wpm_step_adaptive(wave0, nmap, dz, E, (ps, ps), n_bins=12, power_spacing=2.0)
    g.update(wstep_wave0=wave0, wstep_out=np.asarray(nw), wstep_w=np.asarray(w),
             wstep_idxL=np.asarray(iL), wstep_nrefs=np.asarray(nrefs))
    # a slice with constant potential: every pixel hits the denom==0 guard
    nconst = ref.electron_refractive_index(np.full((ny, nx), 7.5), E)
    nw, w, iL, nrefs = ref.wpm_step_adaptive(wave0, nconst, dz, E, (ps, ps), n_bins=4, power_spacing=1.0)
    g.update(wconst_out=np.asarray(nw), wconst_w=np.asarray(w), wconst_idxL=np.asarray(iL))

    # --- move_probe ---------------------------------------------------------
    pr = rng.normal(size=(16, 24)) + 1j * rng.normal(size=(16, 24))
    g["mp_in"] = pr
    g["mp_pos"] = np.array([[3, 20], [15, 0], [8, 12], [0, 23]])
    g["mp_out"] = np.stack([np.asarray(ref.move_probe(pr, tuple(p))) for p in g["mp_pos"]])

    # --- detector crop --------------------------------------------------------
    pat = rng.random((65, 64))
    g["crop_in"] = pat
    g["crop_odd"] = np.asarray(ref.downsample_to_max_angle(pat, (0.1, 0.1), 0.025, 40.0))
    g["crop_even"] = np.asarray(ref.downsample_to_max_angle(pat, (0.1, 0.12), 0.025, 50.0, parity="even"))

    # --- naive per-pixel WPM step (small grid: one propagate per pixel) ------
    ny, nx, ps, dz, E = 16, 24, 0.05, 2.04, 300e3
    Vn = _gauss_stack(rng, 1, ny, nx, ps, 3, 80.0, 0.2)[0] / dz
    wave = _probe(ny, nx, ps, ref.energy2wavelength(E), 0.05, rng)
    nmap = ref.electron_refractive_index(Vn, E)
    g.update(naive_wave=wave, naive_n=np.asarray(nmap), naive_meta=np.array([ny, nx, ps, dz, E]),
             naive_out=np.asarray(ref.wpm_step(wave, nmap, dz, E, (ps, ps))))

    # --- Lippmann-Schwinger 2D: Green's function kernel, one convolution, a solve --
    k0_ls, h_ls, n_ls = 2 * np.pi / 0.4, 0.05, 24
    Khat, emb = ref.build_lippmann_schwinger_kernel_2d(k0_ls, h_ls, h_ls, n_ls, n_ls)
    src = rng.normal(size=(n_ls, n_ls)) + 1j * rng.normal(size=(n_ls, n_ls))
    g.update(ls_meta=np.array([k0_ls, h_ls, n_ls]), ls_Khat=np.asarray(Khat), ls_src=src,
             ls_conv=np.asarray(ref.apply_convolution(src, Khat, emb, (n_ls, n_ls))))
    Vls = _gauss_stack(rng, 1, 16, 16, 0.1, 3, 20.0, 0.3)[0] / 2.0
    psi_ls = ref.solve_scattering_2d_lippmann_schwinger(Vls, 200e3, 0.1, gmres_tol=1e-6, gmres_restart=70)
    g.update(ls_V=Vls, ls_psi=np.asarray(psi_ls), ls_solve_meta=np.array([200e3, 0.1, 1e-6]))

    # --- 1D helpers (k0 small enough that the AS kernel has evanescent parts) --
    n1, dx1, dy1, k01 = 64, 0.35, 1.7, 7.0
    kx = np.asarray(ref.get_kx_1d(n1, dx1))
    psi1 = rng.normal(size=(3, n1)) + 1j * rng.normal(size=(3, n1))
    Hf = np.asarray(ref.fresnel_kernel_1d(kx ** 2, k01, dy1))
    Ha = np.asarray(ref.angular_spectrum_kernel_1d(kx ** 2, k01, dy1))
    psik = np.fft.fft(psi1[0])
    nv = np.array([1.0, 1.2, 1.5, 2.0])
    g.update(l1_meta=np.array([n1, dx1, dy1, k01]), l1_kx=kx, l1_psi=psi1, l1_Hf=Hf, l1_Ha=Ha,
             l1_prop_f=np.stack([np.asarray(ref.propagate_1d(p, Hf)) for p in psi1]),
             l1_prop_a=np.stack([np.asarray(ref.propagate_1d(p, Ha)) for p in psi1]),
             l1_nvals=nv, l1_wpm1=np.asarray(ref.wpm_kernel_1d(psik, 1.3, k01, kx ** 2, dy1)),
             l1_wpmv=np.asarray(ref.wpm_kernel_1d_vmap(psik, nv, k01, kx ** 2, dy1)))

    np.savez_compressed(out, **g)
    print(f"wrote {out} ({os.path.getsize(out)} bytes, {len(g)} arrays)")


if __name__ == "__main__":
    ref_root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WAP_REFERENCE_ROOT")
    if not ref_root:
        sys.exit("usage: make_golden.py path/to/reference (or set WAP_REFERENCE_ROOT)")
    make(ref_root, os.path.join(HERE, "golden.npz"))
