"""Shared-memory layouts of the FFT exchanges, checked exhaustively on the host.

The Stockham stages (csrc/wap_fft.cuh, fft_stage) store output m of butterfly
b at position (b - k) R + k + m L (k = b mod L) and read position t + T e.
The padded column exchange (ColExchangePad) forms the padded row
pad(p) = p + p // 16 from the run-time base and the compile-time offset
separately, pad(base) + pad(offset); that equals pad(base + offset) only if
the low four bits of the two never carry, which must hold for every access
of every E = 16 plan.  The scheduler uses it for 512-point columns (8 per
tile), where it must also leave no two lanes of a half-warp on the same bank
with different addresses (64-bit accesses are served per half-warp).
"""
import pytest


def plan(n, e):
    """(radix, span) of every stage of the n-point plan with e elements per
    thread: radix-e stages, then one smaller remainder radix."""
    logn, loge = n.bit_length() - 1, e.bit_length() - 1
    radices = [e] * (logn // loge)
    if logn % loge:
        radices.append(1 << (logn % loge))
    spans, span = [], 1
    for r in radices:
        spans.append(span)
        span *= r
    return list(zip(radices, spans))


def pad(p):
    return p + (p >> 4)


def stage_accesses(n, e):
    """Every exchange access as (stage, kind, thread, base, offset): the
    stores of all stages but the last and the reads that follow them."""
    t_count = n // e
    stages = plan(n, e)
    for si, (r, span) in enumerate(stages[:-1]):
        per_thread = e // r
        for t in range(t_count):
            for q in range(per_thread):
                b = t + t_count * q
                k = b % span
                for m in range(r):
                    yield si, "st", t, (b - k) * r + k, m * span
        for t in range(t_count):
            for slot in range(e):
                yield si, "ld", t, t, t_count * slot


@pytest.mark.parametrize("n", [128, 256, 512, 1024, 2048])
def test_padded_index_splits_without_carry(n):
    for si, kind, t, base, off in stage_accesses(n, 16):
        assert pad(base) + pad(off) == pad(base + off), (n, si, kind, t, base, off)
        assert base + off < n


def test_padded_512_column_tile_fits_the_exchange_buffer():
    n, w, e = 512, 8, 16
    exch_float2 = (256 * e * 8 + 256 * e * 8 // 16) // 8   # kExchBytesFor(16) / sizeof(float2)
    assert (n + n // 16) * w <= exch_float2
    assert max(pad(p) for p in range(n)) < n + n // 16


def _banks(n, w, padded):
    """For each exchange instruction of the 512-point column tile (W columns,
    thread = (column cc, lane t) with cc = tid % W, t = tid / W): the number of
    distinct addresses that share a bank within a half-warp, worst case."""
    t_count = n // 16
    worst = 1
    accesses = {}
    for si, kind, t, base, off in stage_accesses(n, 16):
        accesses.setdefault((si, kind, off), {}).setdefault(t, base + off)
    for (si, kind, off), pos_of_t in accesses.items():
        for tid0 in range(0, t_count * w, 16):            # half-warps
            banks = {}
            for tid in range(tid0, tid0 + 16):
                cc, t = tid % w, tid // w
                p = pos_of_t[t]
                row = pad(p) if padded else p
                word = 2 * (row * w + cc)                   # float2 = 2 words
                for wd in (word, word + 1):
                    banks.setdefault(wd % 32, set()).add(wd)
            worst = max(worst, max(len(v) for v in banks.values()))
    return worst


def test_padding_removes_the_512_column_scatter_conflict():
    assert _banks(512, 8, padded=False) == 2   # the radix-16 scatter, unpadded: 2-way
    assert _banks(512, 8, padded=True) == 1
