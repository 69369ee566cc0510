"""CPU replay of the tensor-core GEMM (k_gemm_tc, csrc/tm_gemm.cuh): the
operand layout of a 128 x 32 slice (K-major, no swizzle, K groups 2064 bytes
apart), read back through the descriptors of the four K = 8 MMAs, and the
split-TF32 arithmetic (hi = x with 13 low mantissa bits cleared, lo = x - hi,
hi*hi + hi*lo + lo*hi with lo rounded to TF32 by the tensor core) against an
FP64 product."""
import numpy as np
import pytest

SBO, LBO, BK = 128, 16 * 128 + 16, 32


def off(r, k):
    return (r % 8) * 16 + (k % 4) * 4 + (r // 8) * SBO + (k // 4) * LBO


def test_slice_layout_in_bounds_injective_and_bank_spread():
    addrs = {off(r, k) for r in range(128) for k in range(BK)}
    assert len(addrs) == 128 * BK and max(addrs) + 4 <= (BK // 4) * LBO
    assert all(a % 4 == 0 for a in addrs)
    # A stores: one K index per lane -> 32 different banks for every row
    for r in range(128):
        assert len({(off(r, k) // 4) % 32 for k in range(32)}) == 32
    # B stores: one N index per lane, 16 bytes each -> 512 contiguous bytes per warp
    for q in range(BK // 4):
        for w in range(4):
            starts = sorted(off(32 * w + l, 4 * q) for l in range(32))
            assert starts == list(range(starts[0], starts[0] + 512, 16))


def test_descriptors_read_the_slice_back():
    """MMA kk reads K = 8 kk .. 8 kk + 7: core matrix (i, j) at start + i SBO + j LBO
    with start = base + 2 kk LBO."""
    rng = np.random.default_rng(0)
    a = rng.standard_normal((128, BK))
    mem = np.zeros((BK // 4) * LBO // 4)
    for r in range(128):
        for k in range(BK):
            mem[off(r, k) // 4] = a[r, k]
    for kk in range(BK // 8):
        start = kk * 2 * LBO
        for r in range(128):
            for k in range(8):
                i, j = r // 8, k // 4
                addr = start + i * SBO + j * LBO + (r % 8) * 16 + (k % 4) * 4
                assert mem[addr // 4] == a[r, 8 * kk + k]


def _tf32_trunc(x):
    return (np.asarray(x, np.float32).view(np.uint32) & np.uint32(0xFFFFE000)).view(np.float32)


def _tf32_round(x):
    u = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x1000) & 0xFFFFE000
    return u.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("lo_rounding", [_tf32_trunc, _tf32_round])
def test_split_tf32_error_bound(lo_rounding):
    rng = np.random.default_rng(1)
    M, N, K = 64, 64, 288
    A = (rng.standard_normal((M, K)) * 3).astype(np.float32)
    B = (rng.standard_normal((K, N)) / np.sqrt(K)).astype(np.float32)
    ah = _tf32_trunc(A)
    al = (A - ah).astype(np.float32)
    bh = _tf32_trunc(B)
    bl = (B - bh).astype(np.float32)
    assert np.all(A == ah + al) and np.all(B == bh + bl)     # the split is exact
    al_t, bl_t = lo_rounding(al).astype(np.float64), lo_rounding(bl).astype(np.float64)
    got = ah.astype(np.float64) @ bh + ah.astype(np.float64) @ bl_t + al_t @ bh.astype(np.float64)
    ref = A.astype(np.float64) @ B.astype(np.float64)
    scale = np.abs(A.astype(np.float64)) @ np.abs(B.astype(np.float64))
    assert (np.abs(got - ref) / scale).max() < 3e-6
    # plain TF32 operands for comparison: two orders of magnitude worse
    plain = ah.astype(np.float64) @ bh.astype(np.float64)
    assert (np.abs(plain - ref) / scale).max() > 1e-4
