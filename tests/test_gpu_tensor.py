"""The FP16 tensor-core form of the search (tm_set_precision) on the GPU.

The form stores the correlation spectra in FP16 and runs the row transform as
two DFT-matrix stages on the tensor cores (FP16 operands, FP32 accumulation);
MIP, argmax and the compensated sums stay FP32 (FP64 across batches).  Bars
against the FP64 oracle on the same prepared inputs: MIP within 1e-3 of the MIP
scale (the north-star bound is 1e-2; the expected error is ~1e-4), best
orientation equal wherever the oracle's runner-up is more than 1e-3 of the
scale below its maximum, sums within 1e-3 of their scale, histogram counts
within 1% (+ 0.5% of the total in the two edge bins of a value's bin).
"""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import core
from oracle import oracle as O
from tests.search_cases import make_case

pytestmark = pytest.mark.gpu

TOL = 1e-3


def _search(case, precision, orientation_batch=0):
    with core.SearchCore(case["X"], case["Y"], case["T"], histogram_min_scaled=case["hmin"],
                         histogram_step_scaled=case["hstep"], orientation_batch=orientation_batch) as sc:
        sc.set_precision(precision)
        assert sc.precision() == precision
        sc.set_template(case["tspec"])
        sc.set_image(case["ispec"])
        sc.run_plane(case["filt"], case["angles"])
        return sc.results()


def _errors(got, st):
    scale = np.abs(st.mip).max()
    mip_err = float(np.abs(got["mip"] - st.mip).max() / scale)
    decided = (st.mip - st.second) > TOL * scale
    agree = float(np.mean(got["psi"][decided] == st.psi[decided]) * np.mean(got["theta"][decided] == st.theta[decided]))
    sum_err = float(np.abs(got["sum"] - st.sum).max() / np.abs(st.sum).max())
    sq_err = float(np.abs(got["sumsq"] - st.sumsq).max() / np.abs(st.sumsq).max())
    return mip_err, decided, agree, sum_err, sq_err


@pytest.mark.parametrize("T,X", [(64, 1024), (128, 2048)])
def test_fp16_tensor_form_matches_oracle(T, X):
    case = make_case(T=T, X=X, Y=X, pixel_size=1.5, n_particles=6, snr=0.3, angular_step=30.0, psi_step=30.0)
    got = _search(case, core.PRECISION_FP16_TENSOR)
    st = O.SearchState(X, X)
    O.search(st, case["tspec"], case["ispec"], case["filt"], case["angles"], hist_min_scaled=case["hmin"],
             hist_step_scaled=case["hstep"])
    mip_err, decided, _, sum_err, sq_err = _errors(got, st)
    assert mip_err <= TOL, mip_err
    assert decided.mean() > 0.8        # the comparison covers most pixels
    for k in ("psi", "theta", "phi"):
        assert np.mean(got[k][decided] == getattr(st, k)[decided]) >= 0.999, k
    assert sum_err <= TOL and sq_err <= TOL, (sum_err, sq_err)
    h = st.hist[:512]
    assert abs(int(got["hist"].sum()) - int(h.sum())) <= 1e-3 * h.sum()
    # a value moves at most to a neighbouring bin: compare 3-bin windows
    hw = np.convolve(h, np.ones(3), "same")
    gw = np.convolve(got["hist"], np.ones(3), "same")
    assert np.all(np.abs(gw - hw) <= 0.01 * hw + 0.005 * h.sum() + 2)


def test_fp16_tensor_form_agrees_with_fp32_at_4096():
    """The metric's geometry: 4096^2 with a 256^3 box, FP16 form against the FP32 path."""
    case = make_case(T=256, X=4096, Y=4096, pixel_size=1.0, n_particles=8, snr=0.3, angular_step=60.0,
                     psi_step=45.0, n_orient=96)
    ref = _search(case, core.PRECISION_FP32, orientation_batch=32)
    got = _search(case, core.PRECISION_FP16_TENSOR, orientation_batch=32)
    scale = np.abs(ref["mip"]).max()
    assert np.abs(got["mip"] - ref["mip"]).max() <= TOL * scale
    assert np.abs(got["sum"] - ref["sum"]).max() <= TOL * np.abs(ref["sum"]).max()
    assert np.abs(got["sumsq"] - ref["sumsq"]).max() <= TOL * np.abs(ref["sumsq"]).max()
    # best orientations: FP16 and FP32 resolve near-ties (96 orientations, no margin filter) differently
    assert np.mean(got["psi"] == ref["psi"]) > 0.9


def test_fp16_tensor_form_rejected_where_it_has_no_kernels():
    case = make_case(T=32, X=256, Y=256, angular_step=60.0, psi_step=60.0)
    with core.SearchCore(256, 256, 32, histogram_min_scaled=case["hmin"], histogram_step_scaled=case["hstep"]) as sc:
        with pytest.raises(core.TmError) as e:
            sc.set_precision(core.PRECISION_FP16_TENSOR)
        assert e.value.code == core.TM_ERR_UNSUPPORTED
        assert sc.precision() == core.PRECISION_FP32
