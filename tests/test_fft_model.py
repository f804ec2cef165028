"""NumPy model of the per-thread Stockham schedule in csrc/wap_fft.cuh.

Thread t holds x[t + T e]; stage s (radix R, span L) twiddles slot q + (E/R) j
by W_{LR}^{jk} read from the table of rows j = 1..R-1 at tw_offset(s) + (j-1) L + k, runs a
radix-R DFT and scatters y_m to (b - k) R + k + m L.  The model uses the same
plan arithmetic and table layout and must reproduce numpy.fft exactly (to
rounding) for every size and elements-per-thread the kernels instantiate.
"""
import numpy as np
import pytest


def plan(N, E):
    logN, logE = N.bit_length() - 1, E.bit_length() - 1
    nfull, rem = logN // logE, 1 << (logN % logE)
    return [E] * nfull + ([rem] if rem > 1 else [])


def twiddle_table(N, E):
    radices = plan(N, E)
    tab, offs, L, off = [], [], radices[0], 0
    for s in range(1, len(radices)):
        R = radices[s]
        offs.append(off)
        for j in range(1, R):
            for k in range(L):
                tab.append(np.exp(-2j * np.pi * ((j * k) % (L * R)) / (L * R)))
        off += (R - 1) * L
        L *= R
    return np.array(tab), [None] + offs


def model_fft(x, E, inv=False):
    N = len(x)
    T = N // E
    radices = plan(N, E)
    tab, offs = twiddle_table(N, E)
    if inv:
        tab = tab.conj()
    regs = np.array([[x[t + T * e] for e in range(E)] for t in range(T)], dtype=complex)
    L = 1
    for s, R in enumerate(radices):
        B = E // R
        last = s == len(radices) - 1
        smem = np.full(N, np.nan + 0j)
        jj = np.arange(R)
        D = np.exp((1 if inv else -1) * 2j * np.pi * np.outer(jj, jj) / R)
        for t in range(T):
            for q in range(B):
                b = t + T * q
                k = b & (L - 1)
                a = np.array([regs[t][q + B * j] for j in range(R)])
                if L > 1:
                    a = a * np.array([1] + [tab[offs[s] + (j - 1) * L + k] for j in range(1, R)])
                y = D @ a
                for m in range(R):
                    if last:
                        regs[t][q + B * m] = y[m]
                    else:
                        smem[(b - k) * R + k + m * L] = y[m]
        if not last:
            assert not np.isnan(smem).any()
            regs = np.array([[smem[t + T * e] for e in range(E)] for t in range(T)])
        L *= R
    out = np.empty(N, complex)
    for t in range(T):
        for e in range(E):
            out[t + T * e] = regs[t][e]
    return out


@pytest.mark.parametrize("E", [8, 16])
@pytest.mark.parametrize("N", [16, 32, 64, 128, 256, 512, 1024, 2048])
def test_schedule_matches_numpy(N, E):
    if N < E:
        pytest.skip("N < E")
    rng = np.random.default_rng(N + E)
    x = rng.normal(size=N) + 1j * rng.normal(size=N)
    assert np.allclose(model_fft(x, E), np.fft.fft(x), atol=1e-9 * N)
    assert np.allclose(model_fft(x, E, inv=True), np.fft.ifft(x) * N, atol=1e-9 * N)


def test_row_padding_is_bank_conflict_free():
    """p + (p >> 4) maps the 16 lanes of a half-warp to distinct 8-byte bank
    pairs for the first-stage scatter b R + m (R = 16, 8, 4, 2) and the
    gather t + T e."""
    for R in (16, 8, 4, 2):
        for m in range(R):
            banks = {((R * b + m) + ((R * b + m) >> 4)) % 16 for b in range(16)}
            assert len(banks) == 16, R
    for T in (16, 32, 64):
        for e in range(16):
            banks = {((t + T * e) + ((t + T * e) >> 4)) % 16 for t in range(16)}
            assert len(banks) == 16
