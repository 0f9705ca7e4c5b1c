"""CPU model of the phase-contrast FFT kernels' index arithmetic
(phasecon_b200/csrc/kernels_pc.cu: fpos, twid, dft_regs, stockham_stage,
fft_smem), checked against numpy's FFT.

The kernels keep every sequence in a padded shared-memory layout (element i
of sequence q at q * S + i + i // 16, S = (n + n // 16) | 1) and run radix-16
Stockham stages (radix 8, 4 or 2 for the rest) whose butterfly j reads
x_p = a[j + p n / R], multiplies by w_{RL}^{p (j mod L)}, transforms the R
points and writes them to (j - j mod L) R + j mod L + p L. This model runs
the same formulas for each largest stage radix (the same twiddle table: the half circle exp(-2 pi i m /
nmax), m < nmax / 2) in FP64; it must reproduce the DFT for every power of
two the kernels accept and never address outside its buffers.
"""
import numpy as np
import pytest


def _bitrev(i, bits):
    r = 0
    for b in range(bits):
        if i & (1 << b):
            r |= 1 << (bits - 1 - b)
    return r


def _twid(tw, m, nmax, inv):
    h = nmax // 2
    w = tw[m] if m < h else -tw[m - h]
    return np.conj(w) if inv else w


def _dft_regs(x, tw, nmax, inv):
    R = len(x)
    bits = R.bit_length() - 1
    y = [0j] * R
    for i in range(R):
        y[_bitrev(i, bits)] = x[i]
    ln = 2
    while ln <= R:
        for i in range(0, R, ln):
            for k in range(ln // 2):
                t = _twid(tw, k * (nmax // ln), nmax, inv) * y[i + k + ln // 2]
                y[i + k + ln // 2] = y[i + k] - t
                y[i + k] = y[i + k] + t
        ln *= 2
    return y


def _fpos(q, i, S):
    return q * S + i + (i >> 4)


def fft_model(seqs, nmax, inv, max_radix=16):
    nseq, n = seqs.shape
    S = (n + n // 16) | 1
    size = nseq * S
    tw = np.exp(-2j * np.pi * np.arange(nmax // 2) / nmax)
    a = np.zeros(size, complex)
    b = np.zeros(size, complex)
    for q in range(nseq):
        for i in range(n):
            a[_fpos(q, i, S)] = seqs[q, i]
    L, log2n = 1, n.bit_length() - 1
    while L < n:
        rem = min(n // L, max_radix)
        R = 16 if rem >= 16 else 8 if rem >= 8 else 4 if rem >= 4 else 2
        lr = R.bit_length() - 1
        lm = log2n - lr
        m = 1 << lm
        tscale = nmax // (R * L)
        for idx in range(nseq << lm):
            q, j = idx >> lm, idx & (m - 1)
            k = j & (L - 1)
            src = [_fpos(q, j + p * m, S) for p in range(R)]
            assert max(src) < size
            x = [a[i] for i in src]
            if L > 1:
                for p in range(1, R):
                    assert k * p * tscale < nmax
                    x[p] = _twid(tw, k * p * tscale, nmax, inv) * x[p]
            x = _dft_regs(x, tw, nmax, inv)
            o = ((j - k) << lr) + k
            for p in range(R):
                d = _fpos(q, o + p * L, S)
                assert d < size
                b[d] = x[p]
        a, b = b, a
        L *= R
    return np.array([[a[_fpos(q, i, S)] for i in range(n)] for q in range(nseq)])


@pytest.mark.parametrize("max_radix", [2, 4, 8, 16])
@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024])
def test_stockham_schedule_reproduces_the_dft(n, max_radix):
    rng = np.random.default_rng(n)
    for nmax in sorted({n, 1024}):
        x = rng.normal(size=(2, n)) + 1j * rng.normal(size=(2, n))
        fwd = fft_model(x, nmax, False, max_radix)
        inv = fft_model(x, nmax, True, max_radix)
        assert np.abs(fwd - np.fft.fft(x, axis=1)).max() <= 1e-12 * np.abs(fwd).max()
        assert np.abs(inv - np.fft.ifft(x, axis=1) * n).max() <= 1e-12 * np.abs(inv).max()


def test_padded_layout_spreads_the_transposed_staging_over_the_banks():
    """The column pass stages element (row r, column q) at fpos(q, r, S): the
    16 columns one row's consecutive threads write land on 16 distinct
    two-bank pairs (a float2 is two 4-byte banks) for every power-of-two
    column length."""
    for n in [16, 32, 64, 128, 256, 512, 1024]:
        S = (n + n // 16) | 1
        for r in (0, 5, n - 1):
            banks = {(2 * _fpos(q, r, S)) % 32 for q in range(16)}
            assert len(banks) == 16, (n, r)
