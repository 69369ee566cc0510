"""The dense-operator GEMM of the pixel-size change (template volume and
refine_template) on the tensor cores: split TF32 (x = hi + lo, three
kind::tf32 MMAs per K step, FP32 accumulation in tensor memory) against an
FP64 product, and the FP32 CUDA-core form beside it.  Sizes cover partial
128 x 128 tiles and partial 32-deep K slices, the subtracted scalar and the
accumulate flag, as the template and refine callers use them."""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import core

pytestmark = pytest.mark.gpu

# error bound relative to the scale sum_k |a_mk| |b_kn| of each output (plain TF32
# operands would leave about 5e-4 of it)
TOL_TENSOR = 1e-5
TOL_CUDA = 1e-5


@pytest.mark.parametrize("M,N,K", [(128, 128, 32), (288, 512, 288), (256, 256, 288), (65, 300, 7), (1, 1, 1),
                                   (384, 384, 768)])
@pytest.mark.parametrize("accumulate", [False, True])
def test_gemm_matches_fp64(M, N, K, accumulate):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    A = rng.standard_normal((M, K)).astype(np.float32) * np.float32(3.0)
    B = (rng.standard_normal((K, N)) / np.sqrt(K)).astype(np.float32)
    C0 = rng.standard_normal((M, N)).astype(np.float32)
    s = 0.37
    ref = (A.astype(np.float64) - np.float64(np.float32(s))) @ B.astype(np.float64)
    if accumulate:
        ref += C0
    scale = np.abs(A.astype(np.float64) - s) @ np.abs(B.astype(np.float64)) + (np.abs(C0) if accumulate else 0)
    for tensor, tol in ((True, TOL_TENSOR), (False, TOL_CUDA)):
        got = core.debug_gemm(A, B, C0 if accumulate else None, s=s, accumulate=accumulate, tensor=tensor)
        err = np.abs(got - ref) / scale
        assert err.max() <= tol, (tensor, float(err.max()))


def test_gemm_small_values_keep_relative_precision():
    """Operands far from 1 (the pixel-size operators divided by P^3, values ~1e-7):
    the split keeps FP32's exponent range, so the relative error does not grow."""
    rng = np.random.default_rng(3)
    A = (rng.standard_normal((256, 256)) * 1e-7).astype(np.float32)
    B = (rng.standard_normal((256, 4096)) * 1e3).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64)
    scale = np.abs(A.astype(np.float64)) @ np.abs(B.astype(np.float64))
    got = core.debug_gemm(A, B, tensor=True)
    assert (np.abs(got - ref) / scale).max() <= TOL_TENSOR
