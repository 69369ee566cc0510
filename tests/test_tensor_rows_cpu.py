"""CPU emulation of the tensor-core row pass (k_pass_c_tc, csrc/tm_tensor.cuh).

The kernel's index algebra -- the c2r packing, the four-step split of the
X/2-point inverse transform into a 64-point stage and an N1-point stage, the
operands' no-swizzle core-matrix layouts, the lane-pair combination of real
and imaginary products and the pixel ownership of the epilogue -- is replayed
in numpy with the same formulas and compared with numpy's inverse real FFT of
the row.  It also checks that every operand byte address the descriptors can
reach stays inside its shared-memory region and that distinct elements never
share an address.
"""
import numpy as np
import pytest

SBO_A = 144
LBO_A = 16 * SBO_A


def geometry(X):
    H = X // 2
    N1 = H // 64
    R = 64 // N1
    K2 = max(16, N1)
    return H, N1, R, K2


def a_off(m, k):
    return (m % 8) * 2 + (k % 8) * 16 + (m // 8) * SBO_A + (k // 8) * LBO_A


def b_off(n, k, n_total):
    lbo = (n_total // 8) * 128
    return (n % 8) * 16 + (k % 8) * 2 + (n // 8) * 128 + (k // 8) * lbo


def mma_from_layouts(a_bytes, b_bytes, M, N, K):
    """D = A B read through the kernel's descriptors: A MN-major (SBO 144,
    LBO 16*144), B K-major (SBO 128, LBO (N/8)*128), one K = 16 step at a time
    with both start addresses advanced by two K groups."""
    D = np.zeros((M, N))
    for kk in range(K // 16):
        a0, b0 = kk * 2 * LBO_A, kk * 2 * (N // 8) * 128
        for k in range(16):
            A = np.array([a_bytes[(a0 + a_off(m, k)) // 2] for m in range(M)])
            Bk = np.array([b_bytes[(b0 + b_off(n, k, N)) // 2] for n in range(N)])
            D += np.outer(A, Bk)
    return D


@pytest.mark.parametrize("X", [1024, 2048, 4096])
def test_operand_layouts_in_bounds_and_injective(X):
    H, N1, R, K2 = geometry(X)
    a1 = {a_off(m, k) for m in range(128) for k in range(64)}
    assert len(a1) == 128 * 64 and max(a1) + 2 <= 8 * LBO_A
    a2 = {a_off(m, k) for m in range(128) for k in range(K2)}
    assert len(a2) == 128 * K2 and max(a2) + 2 <= (K2 // 8) * LBO_A
    for n_total, k_total in ((128, 64), (2 * N1, K2)):
        b = {b_off(n, k, n_total) for n in range(n_total) for k in range(k_total)}
        assert len(b) == n_total * k_total and max(b) + 2 <= (k_total // 8) * (n_total // 8) * 128
    # the descriptor of the last K step of a stage reaches exactly the end of its region
    last = (K2 // 16 - 1) * 2 * LBO_A + a_off(127, 15)
    assert last < (K2 // 8) * LBO_A


@pytest.mark.parametrize("X", [1024, 4096])
def test_four_step_rows_match_inverse_rfft(X):
    rng = np.random.default_rng(X)
    H, N1, R, K2 = geometry(X)
    # half-complex rows of R real rows
    real_rows = rng.standard_normal((R, X))
    Z = np.fft.rfft(real_rows, axis=1)                  # (R, H+1)
    # the kernel's c2r packing: v[k] = e + i W^{+k} d
    k = np.arange(H)
    hk, hm = Z[:, k].copy(), Z[:, H - k].copy()
    hk[:, 0] = hk[:, 0].real
    hm[:, 0] = hm[:, 0].real
    e = hk + np.conj(hm)
    d = hk - np.conj(hm)
    od = d * np.exp(2j * np.pi * k / X)
    v = e + 1j * od
    # stage-1 A operand A1[(r, k1, p)][k2] in the MN-major core-matrix layout
    a1 = np.zeros(8 * LBO_A // 2)
    for r in range(R):
        for kk in range(H):
            k1, k2 = kk % N1, kk // N1
            m = 2 * (k1 + N1 * r)
            a1[a_off(m, k2) // 2] = v[r, kk].real
            a1[(a_off(m, k2) + 2) // 2] = v[r, kk].imag
    # B1 = [cos | sin] of the 64-point DFT, K = k2 (fill_tc_dft)
    b1 = np.zeros((64 // 8) * (128 // 8) * 128 // 2)
    for k2 in range(64):
        for n in range(64):
            th = 2 * np.pi * ((k2 * n) % 64) / 64
            b1[b_off(n, k2, 128) // 2] = np.cos(th)
            b1[b_off(64 + n, k2, 128) // 2] = np.sin(th)
    D1 = mma_from_layouts(a1, b1, 128, 128, 64)
    # epilogue 1: lane m = (r, k1, p); the pair combines Re and Im, twiddles, writes A2_r[(n2, p)][k1]
    a2 = np.zeros((R, (K2 // 8) * LBO_A // 2))
    for m in range(0, 128, 2):
        k1, r = (m >> 1) % N1, (m >> 1) // N1
        Pre_c, Pre_s = D1[m, :64], D1[m, 64:]
        Pim_c, Pim_s = D1[m + 1, :64], D1[m + 1, 64:]
        Y = (Pre_c - Pim_s) + 1j * (Pre_s + Pim_c)
        n2 = np.arange(64)
        Yt = Y * np.exp(2j * np.pi * k1 * n2 / H)
        for j in range(64):
            a2[r, a_off(2 * j, k1) // 2] = Yt[j].real
            a2[r, (a_off(2 * j, k1) + 2) // 2] = Yt[j].imag
    b2 = np.zeros((K2 // 8) * (2 * N1 // 8) * 128 // 2)
    for k1 in range(N1):
        for n in range(N1):
            th = 2 * np.pi * ((k1 * n) % N1) / N1
            b2[b_off(n, k1, 2 * N1) // 2] = np.cos(th)
            b2[b_off(N1 + n, k1, 2 * N1) // 2] = np.sin(th)
    out = np.zeros((R, X))
    for r in range(R):
        D2 = mma_from_layouts(a2[r], b2, 128, 2 * N1, K2)
        # epilogue 2: lane m = (n2, p); items (r, n1); pixels 2 (n2 + 64 n1) + {0, 1}
        for n2 in range(64):
            Qre_c, Qre_s = D2[2 * n2, :N1], D2[2 * n2, N1:]
            Qim_c, Qim_s = D2[2 * n2 + 1, :N1], D2[2 * n2 + 1, N1:]
            z = (Qre_c - Qim_s) + 1j * (Qre_s + Qim_c)
            n = n2 + 64 * np.arange(N1)
            out[r, 2 * n] = z.real
            out[r, 2 * n + 1] = z.imag
    # the reference's unnormalised c2r (FFTW, image.cpp:5104-5113) is X * numpy's irfft
    ref = np.fft.irfft(Z, n=X, axis=1) * X
    assert np.allclose(out, ref, atol=1e-9 * np.abs(ref).max())


def test_epilogue_pixel_ownership_covers_each_pixel_once():
    for X in (1024, 2048, 4096):
        H, N1, R, K2 = geometry(X)
        seen = np.zeros((R, X), np.int64)
        for t in range(512):
            warp, lane = t >> 5, t & 31
            q, sub = warp & 3, warp >> 2
            m = 32 * q + lane
            n2, p = m >> 1, m & 1
            item0 = 8 * (2 * sub + p)
            for i in range(8):
                it = item0 + i
                r, n1 = it // N1, it % N1
                x = 2 * (n2 + 64 * n1)
                seen[r, x] += 1
                seen[r, x + 1] += 1
        assert np.all(seen == 1)


def _factorized(n, template):
    """The padded size the reference chooses (functions.cpp:529-577 through match_template.cpp:527-575)."""
    from cistem_downstream_bah_b200 import hostprep as H
    return H.factorize_dimension(n, template)


def _radix_plannable(L):
    m = L
    for r in (2, 3, 5, 7, 11, 13):
        while m % r == 0:
            m //= r
    return m == 1


def test_every_padded_size_has_a_transform():
    """Every side length the reference's factorisation produces for sides
    256..8000 has radix plans for the run-time-length kernels (the side, and
    its half when even, with prime factors up to 13); the factorisation's
    "multiple of four" step does not always reach one (e.g. 6556 -> 6561 = 3^8),
    so odd and 2 (mod 4) sides occur and are covered."""
    odd = 0
    for n in range(256, 8001):
        p = _factorized(n, 64)
        assert 64 <= p <= 8192 and _radix_plannable(p), (n, p)
        assert p % 2 or _radix_plannable(p // 2), (n, p)
        odd += p % 2
    assert odd > 0
