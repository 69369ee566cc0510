"""CPU emulation of the tensor-core column pass (k_pass_b_tc, csrc/tm_tensor.cuh).

For one item (4 columns of one orientation) the kernel's algebra is replayed
in numpy with the kernel's formulas and operand layouts: the pruned forward
transform along y of the T non-zero rows split as Y = 64 x 64 (stage H: the
NB = T/64 rows of each residue n1 against the 64 outputs a, one MMA with the
data as B operand; twiddle exp(-2 pi i n1 a / Y); stage F: the 64-point DFT
over n1), the product with the prepared micrograph spectrum, and the inverse
64 x 64 four-step transform (stages 1 and 2, each the forward DFT matrix
applied to the conjugate).  Complex numbers are 2 x 2 real blocks so that a
TMEM lane holds whole complex values.  The result is compared with numpy's
FFTs of the same column, and the operand regions are checked for bounds and
distinct addresses.
"""
import numpy as np
import pytest

Y = 4096


def kmaj_off(m, k, sbo, lbo):
    """K-major operand: core-matrix rows of 8 K elements (16 B)."""
    return (m % 8) * 16 + (k % 8) * 2 + (m // 8) * sbo + (k // 8) * lbo


def mnmaj_off(m, k, sbo, lbo):
    """MN-major operand: core-matrix rows of 8 M (or N) elements (16 B)."""
    return (m % 8) * 2 + (k % 8) * 16 + (m // 8) * sbo + (k // 8) * lbo


# operand layouts of the kernel (bytes)
E_SBO, E_LBO = 128, 16 * 128                  # stage-H A operand (K-major, M = 128, K = 16)
BH_SBO, BH_LBO = 128, 32 * 128                # stage-H B operand (MN-major, N = 256, K = 16)
BF_SBO, BF_LBO = 128, 16 * 128                # DFT B operand (K-major, N = 128, K = 128)
AK_SBO, AK_LBO = 128, 16 * 128                # K-major A operands (A_F, A1): M = 128, K = 128
AM_SBO, AM_LBO = 128, 16 * 128 + 16           # MN-major A operand (A2): K groups skewed by 16 B


def mma(a, b, a_off, b_off, M, N, K):
    D = np.zeros((M, N))
    for k in range(K):
        A = np.array([a[a_off(m, k) // 2] for m in range(M)])
        B = np.array([b[b_off(n, k) // 2] for n in range(N)])
        D += np.outer(A, B)
    return D


def forward_dft_embedding():
    """B[(n1, q)][(b, p)]: out = sum g exp(-2 pi i n1 b / 64) as real 2 x 2 blocks."""
    bf = np.zeros(16 * BF_LBO // 2)
    for n1 in range(64):
        for b in range(64):
            th = 2 * np.pi * ((n1 * b) % 64) / 64
            c, s = np.cos(th), np.sin(th)
            for (q, p, v) in ((0, 0, c), (1, 0, s), (0, 1, -s), (1, 1, c)):
                bf[kmaj_off(2 * b + p, 2 * n1 + q, BF_SBO, BF_LBO) // 2] = v
    return bf


def test_layouts_in_bounds_and_injective():
    for off, M, K, size in ((lambda m, k: kmaj_off(m, k, E_SBO, E_LBO), 128, 16, 2 * E_LBO),
                            (lambda m, k: mnmaj_off(m, k, BH_SBO, BH_LBO), 256, 16, 2 * BH_LBO),
                            (lambda m, k: kmaj_off(m, k, BF_SBO, BF_LBO), 128, 128, 16 * BF_LBO),
                            (lambda m, k: kmaj_off(m, k, AK_SBO, AK_LBO), 128, 128, 16 * AK_LBO),
                            (lambda m, k: mnmaj_off(m, k, AM_SBO, AM_LBO), 128, 128, 16 * AM_LBO)):
        addrs = {off(m, k) for m in range(M) for k in range(K)}
        assert len(addrs) == M * K and max(addrs) + 2 <= size


@pytest.mark.parametrize("T", [64, 256, 384])
def test_column_pass_matches_numpy(T):
    rng = np.random.default_rng(T)
    NB = T // 64
    cols = 4
    A = rng.standard_normal((T, cols)) + 1j * rng.standard_normal((T, cols))   # rows n < T of 4 columns
    Ip = rng.standard_normal((Y, cols)) + 1j * rng.standard_normal((Y, cols))  # prepared micrograph spectrum
    # ---- stage H: D_H[(a, p)][(v, n1)] = sum_(n2, q) E[(a, p)][(n2, q)] BH[(n2, q)][(v, n1)]
    e = np.zeros(2 * E_LBO // 2)
    for a in range(64):
        for n2 in range(NB):
            th = 2 * np.pi * ((n2 * a) % 64) / 64
            c, s = np.cos(th), np.sin(th)
            for (p, q, v) in ((0, 0, c), (0, 1, s), (1, 0, -s), (1, 1, c)):
                e[kmaj_off(2 * a + p, 2 * n2 + q, E_SBO, E_LBO) // 2] = v
    bh = np.zeros(2 * BH_LBO // 2)
    for n in range(T):
        n1, n2 = n % 64, n // 64
        for v in range(cols):
            bh[mnmaj_off(64 * v + n1, 2 * n2, BH_SBO, BH_LBO) // 2] = A[n, v].real
            bh[mnmaj_off(64 * v + n1, 2 * n2 + 1, BH_SBO, BH_LBO) // 2] = A[n, v].imag
    DH = mma(e, bh, lambda m, k: kmaj_off(m, k, E_SBO, E_LBO), lambda n, k: mnmaj_off(n, k, BH_SBO, BH_LBO),
             128, 256, 16)
    # epilogue H: lanes (a, p) pair up; g = h exp(-2 pi i n1 a / Y) -> A_F[(vl, a)][(n1, q)] per tile
    af = np.zeros((2, 16 * AK_LBO // 2))
    for a in range(64):
        for v in range(cols):
            h = DH[2 * a, 64 * v:64 * v + 64] + 1j * DH[2 * a + 1, 64 * v:64 * v + 64]
            g = h * np.exp(-2j * np.pi * np.arange(64) * a / Y)
            for n1 in range(64):
                af[v // 2, kmaj_off(64 * (v % 2) + a, 2 * n1, AK_SBO, AK_LBO) // 2] = g[n1].real
                af[v // 2, kmaj_off(64 * (v % 2) + a, 2 * n1 + 1, AK_SBO, AK_LBO) // 2] = g[n1].imag
    bf = forward_dft_embedding()
    kk = lambda m, k: kmaj_off(m, k, AK_SBO, AK_LBO)
    bfo = lambda n, k: kmaj_off(n, k, BF_SBO, BF_LBO)
    out = np.zeros((Y, cols), complex)
    for t in range(2):
        DF = mma(af[t], bf, kk, bfo, 128, 128, 128)
        # epilogue F: lane (vl, a), columns (b, p): F[a + 64 b]; Z = I' conj(F); A1 gets conj(Z)
        a1 = np.zeros(16 * AK_LBO // 2)
        for vl in range(2):
            v = 2 * t + vl
            for a in range(64):
                F = DF[64 * vl + a, 0::2] + 1j * DF[64 * vl + a, 1::2]
                Z = Ip[a + 64 * np.arange(64), v] * np.conj(F)
                W = np.conj(Z)
                for b in range(64):
                    a1[kk(64 * vl + a, 2 * b) // 2] = W[b].real
                    a1[kk(64 * vl + a, 2 * b + 1) // 2] = W[b].imag
        D1 = mma(a1, bf, kk, bfo, 128, 128, 128)
        # epilogue 1: lane (vl, k1): Y = conj(D1); Y' = Y exp(+2 pi i k1 n2 / Y); A2[(vl, n2)][(k1, q)] = conj(Y')
        a2 = np.zeros(16 * AM_LBO // 2)
        mm = lambda m, k: mnmaj_off(m, k, AM_SBO, AM_LBO)
        for vl in range(2):
            for k1 in range(64):
                Yv = np.conj(D1[64 * vl + k1, 0::2] + 1j * D1[64 * vl + k1, 1::2])
                Yt = np.conj(Yv * np.exp(2j * np.pi * k1 * np.arange(64) / Y))
                for n2 in range(64):
                    a2[mm(64 * vl + n2, 2 * k1) // 2] = Yt[n2].real
                    a2[mm(64 * vl + n2, 2 * k1 + 1) // 2] = Yt[n2].imag
        D2 = mma(a2, bf, mm, bfo, 128, 128, 128)
        # epilogue 2: lane (vl, n2): z[n2 + 64 n1] = conj(D2)
        for vl in range(2):
            for n2 in range(64):
                z = np.conj(D2[64 * vl + n2, 0::2] + 1j * D2[64 * vl + n2, 1::2])
                out[n2 + 64 * np.arange(64), 2 * t + vl] = z
    # numpy: forward FFT along y of the zero-padded column, times I' (conj), unnormalised inverse
    padded = np.zeros((Y, cols), complex)
    padded[:T] = A
    ref = np.fft.ifft(Ip * np.conj(np.fft.fft(padded, axis=0)), axis=0) * Y
    assert np.allclose(out, ref, atol=1e-9 * np.abs(ref).max())
