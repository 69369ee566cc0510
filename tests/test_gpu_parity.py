"""Parity of the CUDA search core with the FP64 oracle (needs a B200).

Tolerances (the search computes in FP32 with its own FFTs; the oracle in
FP64): correlation maps within 2e-5 of max|cc|; MIP within 1e-4 relative
(the north-star bound); best angles identical wherever the oracle's winning
margin exceeds 1e-4 of the MIP scale; sums within 1e-5 of their scale;
histogram counts within 0.1% (+2) per bin (bins differ only for values that
sit on a bin edge to within FP32 rounding).
"""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import core
from oracle import oracle as O
from tests.search_cases import make_case

pytestmark = pytest.mark.gpu


def _core(case, batch=0):
    sc = core.SearchCore(case["X"], case["Y"], case["T"], histogram_min_scaled=case["hmin"],
                         histogram_step_scaled=case["hstep"], orientation_batch=batch)
    sc.set_template(case["tspec"])
    sc.set_image(case["ispec"])
    return sc


@pytest.mark.parametrize("geom", [(32, 256, 256), (32, 512, 256), (32, 256, 512), (64, 1024, 1024)])
def test_single_orientation_correlation_map(geom):
    T, X, Y = geom
    case = make_case(T=T, X=X, Y=Y, n_orient=40)
    with _core(case) as sc:
        for o in (0, 7, 23, 39):
            sc.reset()
            sc.run_plane(case["filt"], case["angles"][o:o + 1])
            got = sc.results()["mip"].reshape(Y, X)
            ref = O.correlate_one(case["tspec"], case["ispec"], case["filt"], case["angles"], o, X, Y)
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < 2e-5, (o, err)


def _compare_search(case, batch=0, planes=((0.0, 0.0),)):
    X, Y = case["X"], case["Y"]
    st = O.SearchState(X, Y)
    with _core(case, batch) as sc:
        for df, px in planes:
            filt = case["filt"] if df == 0.0 else O.projection_filter(
                case["T"], case["curve"], kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=case["defocus"],
                defocus2=case["defocus"], pixel_size=case["pixel_size"], defocus_offset=df)
            sc.run_plane(filt, case["angles"], defocus_offset=df, pixel_size_offset=px)
            O.search(st, case["tspec"], case["ispec"], filt, case["angles"], hist_min_scaled=case["hmin"],
                     hist_step_scaled=case["hstep"], defocus_value=df, pixel_value=px)
        r = sc.results()
        assert sc.correlations_computed() == len(case["angles"]) * len(planes)
    scale = np.abs(st.mip).max()
    mip_err = np.abs(r["mip"] - st.mip) / scale
    assert mip_err.max() < 1e-4, mip_err.max()
    margin = st.mip - st.second
    decided = margin > 1e-4 * scale
    assert decided.mean() > 0.9
    for k in ("psi", "theta", "phi", "defocus", "pixel"):
        ref = getattr(st, k)
        bad = decided & (r[k] != ref)
        assert not bad.any(), (k, int(bad.sum()))
    s_scale = np.abs(st.sum).max()
    assert np.abs(r["sum"] - st.sum).max() / s_scale < 1e-5
    q_scale = np.abs(st.sumsq).max()
    assert np.abs(r["sumsq"] - st.sumsq).max() / q_scale < 1e-5
    ref_h = st.hist[:512]
    assert np.all(np.abs(r["hist"] - ref_h) <= 0.001 * ref_h + 2)
    return r, st


def test_search_plane_parity():
    case = make_case(T=32, X=256, Y=256, angular_step=30.0, psi_step=30.0)
    _compare_search(case)


def test_ragged_batches_and_defocus_planes():
    # 37 orientations with 8 per device pass: the last batch is partial
    case = make_case(T=32, X=256, Y=512, angular_step=40.0, psi_step=40.0, n_orient=37)
    _compare_search(case, batch=8, planes=((-200.0, 0.0), (0.0, 0.0), (200.0, 0.0)))


def test_template_matching_core_mirror():
    case = make_case(T=32, X=256, Y=256, angular_step=45.0, psi_step=45.0)
    grid = O.search_grid(45.0)
    tmc = core.TemplateMatchingCore()
    tmc.Init(case["tspec"], case["ispec"], 0.0, 0.02, case["pixel_size"], 0.0, 100.0, case["defocus"],
             case["defocus"], 360.0, 0.0, 45.0, grid, case["hmin"], case["hstep"], 512, 0, 0, len(grid) - 1,
             image_x=256)
    pos = tmc.RunInnerLoop(case["filt"], 0, 0)
    assert pos == len(grid) * len(O.psi_list(0.0, 45.0, 360.0))
    st = O.SearchState(256, 256)
    O.search(st, case["tspec"], case["ispec"], case["filt"], tmc.orientations, hist_min_scaled=case["hmin"],
             hist_step_scaled=case["hstep"])
    assert np.abs(tmc.d_max_intensity_projection.ravel() - st.mip).max() / np.abs(st.mip).max() < 1e-4


def test_planted_particles_are_found():
    # physical sanity: each planted particle gives a MIP peak near its centre
    case = make_case(T=32, X=256, Y=256, snr=2.0, angular_step=15.0, psi_step=15.0, n_particles=2)
    with _core(case) as sc:
        sc.run_plane(case["filt"], case["angles"])
        mip = sc.results()["mip"].reshape(256, 256)
    z = (mip - mip.mean()) / mip.std()
    for (px, py) in case["truth"]["positions"]:
        y0, x0 = int(round(py)), int(round(px))
        win = z[max(0, y0 - 3):y0 + 4, max(0, x0 - 3):x0 + 4]
        assert win.max() > 4.0, (px, py, win.max())


def test_autotuned_batch_keeps_parity():
    case = make_case(T=32, X=256, Y=256, angular_step=30.0, psi_step=30.0)
    with _core(case, batch=0) as sc:
        b = sc.autotune(case["filt"], case["angles"][:160])
        assert b in (16, 32, 64, 128) and sc.orientation_batch() == b
        assert sc.correlations_computed() == 0   # the tuning runs are cleared
        sc.run_plane(case["filt"], case["angles"])
        r = sc.results()
    st = O.SearchState(256, 256)
    O.search(st, case["tspec"], case["ispec"], case["filt"], case["angles"], hist_min_scaled=case["hmin"],
             hist_step_scaled=case["hstep"])
    assert np.abs(r["mip"] - st.mip).max() / np.abs(st.mip).max() < 1e-4


def test_large_batches_match_small():
    """256 orientations per device pass (the proposal's window searches) give the
    same maps as 32."""
    case = make_case(T=32, X=256, Y=256, angular_step=20.0, psi_step=20.0)
    out = {}
    for b in (32, 256):
        with _core(case, batch=b) as sc:
            sc.run_plane(case["filt"], case["angles"])
            out[b] = sc.results()
    assert len(case["angles"]) > 256
    for k in ("mip", "psi", "theta", "phi"):
        assert np.array_equal(out[32][k], out[256][k]), k
    scale = np.abs(out[32]["sum"]).max()
    assert np.abs(out[32]["sum"] - out[256]["sum"]).max() <= 1e-5 * scale
