"""The timed CPU baseline (oracle/cpu_port.py: the reference's CPU inner loop in
FP32 with pocketfft transforms) against the FP64 oracle search (CPU only).

The baseline is a timing stand-in for the reference's FFTW build, so it must
compute the same search: MIP within FP32 accuracy of the FP64 search, the same
best orientation wherever the FP64 search's winning margin exceeds that
accuracy, sums and sums of squares within FP32 accuracy of their scale, and the
same histogram up to values on bin edges.
"""
import numpy as np

from oracle import cpu_port
from oracle import oracle as O
from tests.search_cases import make_case


def test_cpu_port_matches_fp64_oracle():
    case = make_case(T=32, X=256, Y=256, angular_step=45.0, psi_step=45.0, n_orient=24)
    X, Y = case["X"], case["Y"]
    got = cpu_port.search(case["tspec"], case["ispec"], case["filt"], case["angles"], X, Y,
                          hist_min_scaled=case["hmin"], hist_step_scaled=case["hstep"], threads=3)
    st = O.SearchState(X, Y)
    O.search(st, case["tspec"], case["ispec"], case["filt"], case["angles"], hist_min_scaled=case["hmin"],
             hist_step_scaled=case["hstep"])
    mip_ref = st.mip.reshape(Y, X)
    scale = np.abs(mip_ref).max()
    assert np.abs(got["mip"] - mip_ref).max() < 1e-4 * scale
    decided = (st.mip - st.second).reshape(Y, X) > 1e-4 * scale
    assert decided.mean() > 0.9
    # the oracle records the best orientation's angles; compare through the angle list
    ang = np.asarray(case["angles"])
    got_psi = ang[got["best"], 2]
    assert np.array_equal(got_psi[decided], st.psi.reshape(Y, X)[decided])
    for k, ref in (("sum", st.sum), ("sumsq", st.sumsq)):
        r = ref.reshape(Y, X)
        assert np.abs(got[k] - r).max() < 1e-5 * np.abs(r).max(), k
    h_ref = np.asarray(st.hist)
    assert got["hist"].sum() == h_ref.sum()
    assert np.abs(got["hist"] - h_ref).max() <= 2
