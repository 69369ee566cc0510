"""The row pass's twiddle multipliers held in tensor memory (CPU only).

At 4096 and 2048 wide, k_pass_c keeps per thread the c2r packing's multipliers
W_X^k (k = t + P r, columns 112-127) and, for stages 1 .. n-1 of its
H-point inverse transform (H = X / 2, 8 values per thread), the powers
w^1 .. w^(RS-1) of each of its R / RS butterflies (PassCStageTw: stage s at
columns 64 + 16 (s - 1), butterfly u's power r at float 2 (u (RS - 1) + r - 1)),
and tmfft::fft_pre multiplies by them instead of building powers from a table
lookup.  This test restates that layout, checks that it fits the columns the
kernel gives it, and runs the transform thread by thread with the multipliers
taken from the layout (the kernel's shared-memory addressing, as in
test_pruned_decomposition_cpu) against numpy's inverse FFT.
"""
import numpy as np
import pytest

from tests.test_pruned_decomposition_cpu import _pad16, _plan, _rd_index


def _stage_columns(H, t):
    """PassCStageTw::fill for thread t: {stage: 16 floats}."""
    R, P = 8, H // 8
    seq = _plan(H, R)
    cols = {}
    Ns = seq[0]
    for s in range(1, len(seq)):
        RS = seq[s]
        g = np.zeros(16)
        for u in range(R // RS):
            jm = (t + P * u) % Ns
            for r in range(1, RS):
                w = np.exp(2j * np.pi * ((jm * (H // (Ns * RS)) * r) % H) / H)   # DIR +1
                i = 2 * (u * (RS - 1) + r - 1)
                assert i + 1 < 16
                g[i], g[i + 1] = w.real, w.imag
        cols[s] = g
        Ns *= RS
    return cols


def _fft_pre_inverse(x):
    """tmfft::fft_pre<H, 8, +1> thread by thread with PassCStageTw's multipliers."""
    H = len(x)
    R, P = 8, H // 8
    seq = _plan(H, R)
    cols = [_stage_columns(H, t) for t in range(P)]
    v = [[x[t + P * r] for r in range(R)] for t in range(P)]
    buf = np.full(_pad16(H) + 64, np.nan, complex)
    Ns = 1
    for s, RS in enumerate(seq):
        last = s == len(seq) - 1
        if s > 0:
            for t in range(P):
                v[t] = [buf[_rd_index(P, t, r)] for r in range(R)]
        new_buf = np.full_like(buf, np.nan)
        for t in range(P):
            for u in range(R // RS):
                b = t + P * u
                e = np.array([v[t][u + r * (R // RS)] for r in range(RS)])
                if s > 0:
                    g = cols[t][s]
                    for r in range(1, RS):
                        i = 2 * (u * (RS - 1) + r - 1)
                        e[r] *= g[i] + 1j * g[i + 1]
                y = np.array([np.sum(e * np.exp(2j * np.pi * np.arange(RS) * q / RS)) for q in range(RS)])
                if last:
                    for r in range(RS):
                        v[t][u + r * (R // RS)] = y[r]
                elif RS == R and ((Ns == 1 and 16 % R == 0) or Ns % 16 == 0):
                    base = _pad16(b * R) if Ns == 1 else _pad16((b // Ns) * Ns * R + b % Ns)
                    for r in range(RS):
                        new_buf[base + (r if Ns == 1 else r * (Ns + Ns // 16))] = y[r]
                else:
                    idx = (b // Ns) * Ns * RS + b % Ns
                    for r in range(RS):
                        new_buf[_pad16(idx + r * Ns)] = y[r]
        buf = new_buf
        Ns *= RS
    out = np.zeros(H, complex)
    for t in range(P):
        for r in range(R):
            out[t + P * r] = v[t][r]
    return out


@pytest.mark.parametrize("X", [4096, 2048])
def test_stage_multiplier_layout_fits_its_columns(X):
    H = X // 2
    seq = _plan(H, 8)
    assert len(seq) <= 4                        # stages 1-3 at columns 64-111
    assert 64 + 16 * (len(seq) - 1) <= 112      # the packing's multipliers start at 112
    for s in range(1, len(seq)):
        assert 2 * (8 // seq[s]) * (seq[s] - 1) <= 16


@pytest.mark.parametrize("X", [4096, 2048])
def test_fft_pre_with_tmem_multipliers_is_the_inverse_fft(X):
    H = X // 2
    rng = np.random.default_rng(X)
    x = rng.normal(size=H) + 1j * rng.normal(size=H)
    got = _fft_pre_inverse(x)
    ref = np.fft.ifft(x) * H
    assert not np.isnan(got).any()
    assert np.abs(got - ref).max() < 1e-9 * np.abs(ref).max()
