"""The index algebra the kernels are built on, checked in numpy (CPU only).

* Pruned forward transform (passes A and B): an N-point DFT of a vector whose
  only non-zero entries are its first T samples equals M = N/L twiddled
  L-point DFTs of the zero-padded samples, F[s + M k] = DFT_L(a[n] W_N^(n s))[k],
  for any L >= T that divides N.
* Register Stockham layout: a thread t of P = L/R holding x[t + P r] ends with
  X[t + P r]; thread j = s + M tp of the pruned transform holds F[j + (N/R) r].
* Real inverse transform by even/odd packing (k_row_c2r, pass C): an N-point
  c2r equals an N/2-point complex inverse of Z[k] = E[k] + i W^-k O[k].
* Radix plans of the kernels' transform lengths, and the shared-memory
  addressing of tmfft::fft emulated thread by thread.
"""
import numpy as np
import pytest


def _plan(L, R):
    """radix_seq of tm_fft.cuh: R while it divides (butterflies of at most radix
    24), then the largest divisors of R that divide the rest."""
    seq, m = [], L
    while R <= 24 and m > 1 and m % R == 0:
        seq.append(R)
        m //= R
    while m > 1:
        d = min(R, 24)
        while d > 1 and not (R % d == 0 and m % d == 0):
            d -= 1
        if d <= 1:
            return None
        seq.append(d)
        m //= d
    return seq


def _prune_len(T, N, V):
    for L in range(T, N + 1):
        if N % L == 0 and L % V == 0 and _plan(L, V):
            return L
    return None


@pytest.mark.parametrize("T,N,V", [(256, 4096, 16), (384, 4096, 16), (256, 3888, 18), (256, 5832, 18),
                                   (384, 5832, 18), (32, 288, 18), (48, 288, 18), (48, 256, 16),
                                   (256, 4096, 32), (384, 4096, 32), (64, 4096, 32)])
def test_pruned_forward_equals_full_dft(T, N, V):
    rng = np.random.default_rng(T + N)
    a = rng.normal(size=T) + 1j * rng.normal(size=T)
    full = np.fft.fft(np.concatenate([a, np.zeros(N - T)]))
    L = _prune_len(T, N, V)
    assert L is not None and L >= T and N % L == 0
    M = N // L
    n = np.arange(T)
    got = np.zeros(N, complex)
    for s in range(M):
        sub = np.zeros(L, complex)
        sub[:T] = a * np.exp(-2j * np.pi * n * s / N)
        got[s + M * np.arange(L)] = np.fft.fft(sub)
    assert np.abs(got - full).max() < 1e-9 * np.abs(full).max()
    # the thread layout: P = N/V threads per column, thread j = s + M*tp holds F[j + P*r]
    P, PT = N // V, L // V
    assert M * PT == P
    for j in (0, 1, P // 2, P - 1):
        s, tp = j % M, j // M
        for r in range(V):
            assert s + M * (tp + PT * r) == j + P * r


@pytest.mark.parametrize("L,R,expect", [(4096, 16, [16, 16, 16]), (2048, 8, [8, 8, 8, 4]), (5832, 18, [18, 18, 18]),
                                        (3888, 18, [18, 18, 6, 2]), (324, 18, [18, 18]), (486, 18, [18, 9, 3]),
                                        (384, 24, [24, 8, 2]), (192, 24, [24, 8]), (288, 18, [18, 2, 2, 2, 2]),
                                        (4096, 32, [16, 16, 16]), (256, 32, [16, 16]), (512, 32, [16, 16, 2]),
                                        (64, 32, [16, 4])])
def test_radix_plans(L, R, expect):
    seq = _plan(L, R)
    assert seq == expect
    assert int(np.prod(seq)) == L and all(R % r == 0 for r in seq)


@pytest.mark.parametrize("N", [64, 96, 384, 5832])
def test_even_odd_packed_c2r(N):
    rng = np.random.default_rng(N)
    real = rng.normal(size=N)
    Hs = np.fft.rfft(real)                       # N/2+1 values
    H = N // 2
    k = np.arange(H)
    hk, hm = Hs[k], np.conj(Hs[H - k])
    e = hk + hm
    d = (hk - hm) * np.exp(2j * np.pi * k / N)
    z = np.fft.ifft(e + 1j * d) * H              # unnormalised H-point inverse
    out = np.empty(N)
    out[0::2], out[1::2] = z.real, z.imag
    assert np.abs(out - real * N).max() < 1e-9 * N


# ---------------------------------------------------------------------------
# Emulation of tmfft::fft (csrc/tm_fft.cuh) thread by thread, with the exact
# shared-memory addressing of its fast and generic paths.
def _pad16(i):
    return i + (i >> 4)


def _rd_index(P, t, r):
    if P % 16 == 0:
        return (t + (t >> 4)) + r * (P + P // 16)
    if 16 % P == 0:
        return t + P * r + ((P * r) >> 4)
    return _pad16(t + P * r)


def _kernel_fft(x, R, sign, lmax=None):
    L = len(x)
    P = L // R
    seq = _plan(L, R)
    lmax = lmax or L
    tab = np.exp(-2j * np.pi * np.arange(lmax) / lmax)

    def tw(m):
        mm = m & (L - 1) if (L & (L - 1)) == 0 else m % L
        t = tab[mm * (lmax // L)]
        return t if sign < 0 else np.conj(t)

    v = [[x[t + P * r] for r in range(R)] for t in range(P)]
    buf = np.full(_pad16(L) + 64, np.nan, complex)
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
                    w = tw((b % Ns) * (L // (Ns * RS)))
                    e = e * w ** np.arange(RS)
                y = np.array([np.sum(e * np.exp(sign * 2j * np.pi * np.arange(RS) * q / RS)) for q in range(RS)])
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
    out = np.zeros(L, complex)
    for t in range(P):
        for r in range(R):
            out[t + P * r] = v[t][r]
    return out


@pytest.mark.parametrize("L,R,lmax", [(36, 18, 288), (288, 18, 288), (324, 18, 3888), (3888, 18, 3888),
                                      (5832, 18, 5832), (486, 18, 5832), (48, 24, 48), (24, 24, 48), (384, 24, 384),
                                      (192, 24, 384), (256, 16, 4096), (4096, 16, 4096), (2048, 8, 4096),
                                      (64, 16, 256), (512, 16, 4096), (4096, 32, 4096), (256, 32, 4096),
                                      (512, 32, 4096), (64, 32, 4096)])
def test_kernel_fft_addressing(L, R, lmax):
    rng = np.random.default_rng(L + R)
    x = rng.normal(size=L) + 1j * rng.normal(size=L)
    for sign in (-1, 1):
        got = _kernel_fft(x, R, sign, lmax)
        ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * L
        assert not np.isnan(got).any()
        assert np.abs(got - ref).max() < 1e-9 * np.abs(ref).max()
