"""Whole searches on the reference's benchmark configurations, against the FP64 oracle.

Configuration 1 (the CPU-runnable one): a seeded 1024^2 micrograph (10 copies
of a 64^3 Gaussian-atom template at 1.5 A/px, 3,000 atoms in a 40 A ball,
SNR 0.05, defocus 12,000 A) searched by the match_template program over the
whole C1 grid of 15 deg out-of-plane / 15 deg in-plane steps (4,700
orientations), and the oracle's restatement of the reference CPU path
(preparation, search, statistics, the result-aggregation peak loop) on the
same files.  Configuration 2 (full size): a 4096^2 micrograph with 80
particles of a 256^3 template at 1.0 A/px searched over 256 contiguous
orientations of the 2.5 / 1.5 deg grid through the C ABI, against the oracle
search on the same prepared inputs.

Bars: MIP within 1e-4 of the MIP scale; best psi/theta/phi identical wherever
the oracle's runner-up is more than 1e-4 of the MIP scale below its maximum;
per-pixel sums within 1e-6 of their scale and sums of squares within 3e-6
(each value carries the FP32 transforms' relative error, ~6e-7 at a particle
peak, which squaring doubles); histogram within 0.1% (+2) per bin; the
thresholded peak list identical wherever a peak's z is decided (more than 2e-3
from the threshold): same positions and angles, z within 2e-3.
"""
import subprocess

import numpy as np
import pytest

from cistem_downstream_bah_b200 import core
from cistem_downstream_bah_b200 import hostprep as H
from cistem_downstream_bah_b200 import synthetic
from oracle import oracle as O
from tests.peak_loop import reference_peaks
from tests.search_cases import histogram_scaled

pytestmark = pytest.mark.gpu

MIP_TOL, SUM_TOL, SUMSQ_TOL, Z_TOL = 1e-4, 1e-6, 3e-6, 2e-3


def _program_args(tmp, img, tpl, pixel, defocus, step, psi_step):
    names = ["mip", "psi", "theta", "phi", "defocus", "pixel", "scaled", "avg", "std"]
    f = {n: str(tmp / f"{n}.mrc") for n in names}
    args = [img, tpl, pixel, 300.0, 2.7, 0.07, defocus, defocus, 0.0, 300.0, 2.0 * pixel, step, 20,
            0.0, 0.0, 0.0, 0.0, 1.0, "no", 0.0, 0.0,
            f["mip"], f["psi"], f["theta"], f["phi"], f["defocus"], f["pixel"], f["scaled"], f["avg"], "C1",
            psi_step, str(tmp / "hist.txt"), -1, -1, 0, 0, f["std"], "/dev/null", str(tmp / "result.mrc"), 10.0,
            "yes", 1]
    assert len(args) == 42
    return f, [str(a) for a in args]


def _check_search_state(got, st, X, Y):
    """SearchCore results against an oracle SearchState on the same inputs."""
    scale = np.abs(st.mip).max()
    assert np.abs(got["mip"] - st.mip).max() <= MIP_TOL * scale
    decided = (st.mip - st.second) > MIP_TOL * scale
    assert decided.mean() > 0.9        # the comparison covers most pixels
    for k in ("psi", "theta", "phi"):
        assert np.array_equal(got[k][decided], getattr(st, k)[decided]), k
    s_scale = np.abs(st.sum).max()
    q_scale = np.abs(st.sumsq).max()
    assert np.abs(got["sum"] - st.sum).max() <= SUM_TOL * s_scale, np.abs(got["sum"] - st.sum).max() / s_scale
    assert np.abs(got["sumsq"] - st.sumsq).max() <= SUMSQ_TOL * q_scale, np.abs(got["sumsq"] - st.sumsq).max() / q_scale
    h = st.hist[:512]
    assert np.all(np.abs(got["hist"] - h) <= 1e-3 * h + 2)


def _same_peak_lists(got, ref, thr):
    """The two peak lists (x, y, psi, theta, phi, defocus, pixel, z) agree: every
    reference peak more than Z_TOL above the threshold is in the other list at
    the same position with the same angles and z within Z_TOL, and every peak of
    the other list is in the reference list or within Z_TOL of the threshold."""
    def match(p, q):
        return np.flatnonzero((q[:, 0] == p[0]) & (q[:, 1] == p[1]))
    for p in ref:
        k = match(p, got)
        if p[7] > thr + Z_TOL:
            assert len(k) == 1, ("reference peak missing", p)
        if len(k):
            assert np.array_equal(got[k[0], 2:7], p[2:7]), (got[k[0]], p)
            assert abs(got[k[0], 7] - p[7]) <= Z_TOL
    for p in got:
        assert len(match(p, ref)) == 1 or p[7] <= thr + Z_TOL, ("extra peak", p)


def _check_fp16_form(got, st, n_orient, X, Y):
    """MIP error (relative to the MIP scale) and z-score error of the FP16
    tensor-core form against the FP64 oracle; the north-star bound on the MIP
    error is 1e-2."""
    sq = np.sqrt(float(X * Y))
    mip_ref, z_ref, _, _ = O.finalize(st, n_orient, sq)
    gs = O.SearchState(X, Y)
    gs.mip[:], gs.sum[:], gs.sumsq[:] = got["mip"], got["sum"], got["sumsq"]
    mip_got, z_got, _, _ = O.finalize(gs, n_orient, sq)
    mip_err = float(np.abs(mip_got - mip_ref).max() / np.abs(mip_ref).max())
    z_err = float(np.abs(z_got - z_ref).max())
    print(f"FP16 tensor-core form vs FP64 oracle, {X}x{Y}, {n_orient} orientations: "
          f"MIP max rel err {mip_err:.2e}, z max abs err {z_err:.2e}")
    assert mip_err <= 1e-2
    assert z_err <= 0.05
    return mip_err, z_err


def test_config1_whole_search_program_matches_oracle(tmp_path):
    T, PIXEL, DEFOCUS, STEP = 64, 1.5, 12000.0, 15.0
    vol = synthetic.template_volume(T, PIXEL, 3000, 40.0, seed=20261204)
    img, truth = synthetic.micrograph(1024, 1024, PIXEL, 3000, 40.0, 10, 0.05, DEFOCUS, seed=20261205,
                                      atom_seed=20261204)
    H.write_mrc(tmp_path / "img.mrc", img, PIXEL)
    H.write_mrc(tmp_path / "tpl.mrc", vol, PIXEL)
    files, args = _program_args(tmp_path, str(tmp_path / "img.mrc"), str(tmp_path / "tpl.mrc"), PIXEL, DEFOCUS,
                                STEP, STEP)
    r = subprocess.run([H.CLI_PATH, *args], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]

    # the oracle pipeline: the reference CPU path restated in FP64
    img32 = H.read_mrc(tmp_path / "img.mrc")[0][0]
    vol32 = H.read_mrc(tmp_path / "tpl.mrc")[0]
    X, Y = O.factorize_dimension(1024, T), O.factorize_dimension(1024, T)
    assert (X, Y) == (1024, 1024)
    ispec, curve = O.whiten_image(img32.astype(np.float64))
    tspec = O.prepare_template(vol32.astype(np.float64))
    filt = O.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=DEFOCUS,
                               defocus2=DEFOCUS, pixel_size=PIXEL)
    ang = O.orientation_list(O.search_grid(STEP), O.psi_list(0.0, STEP, 360.0))
    assert len(ang) == 4700
    sq = np.sqrt(float(X * Y))
    hmin, hstep = histogram_scaled(X, Y)
    st = O.SearchState(X, Y)
    O.search(st, tspec, ispec, filt, ang, hist_min_scaled=hmin, hist_step_scaled=hstep)
    mip, z, avg, sd = O.finalize(st, len(ang), sq)
    shape = (Y, X)

    got = {k: H.read_mrc(v)[0][0] for k, v in files.items()}
    mscale = np.abs(mip).max()
    assert np.abs(got["mip"] - mip.reshape(shape)).max() <= MIP_TOL * mscale
    assert np.abs(got["scaled"] - z.reshape(shape)).max() <= Z_TOL
    assert np.abs(got["avg"] - avg.reshape(shape)).max() <= MIP_TOL * np.abs(sd).max()
    assert np.abs(got["std"] - sd.reshape(shape)).max() <= MIP_TOL * np.abs(sd).max()
    decided = ((st.mip - st.second) > MIP_TOL * np.abs(st.mip).max()).reshape(shape)
    assert decided.mean() > 0.9        # the comparison covers most pixels
    for k in ("psi", "theta", "phi"):
        assert np.array_equal(got[k][decided], getattr(st, k).reshape(shape)[decided]), k
    rows = np.array([[float(v) for v in ln.split()] for ln in open(tmp_path / "hist.txt").read().splitlines()[2:]])
    h = rows[:, 1]
    assert np.all(np.abs(h - st.hist[:512]) <= 1e-3 * st.hist[:512] + 2)

    # the thresholded peak list: the reference's loop on the oracle's maps
    thr = float(np.float32(np.sqrt(np.float32(2.0))) * np.float32(O.erfcinv(2.0 / (float(X) * Y * len(ang)))))
    maps = [st.psi.reshape(shape), st.theta.reshape(shape), st.phi.reshape(shape),
            np.zeros(shape, np.float32), np.zeros(shape, np.float32)]
    ref_peaks = reference_peaks(z.reshape(shape), maps, thr, 10, T, PIXEL)
    lines = [ln.split() for ln in open(tmp_path / "result_peaks.txt").read().splitlines() if not ln.startswith("#")]
    peaks = np.array(lines, np.float32).reshape(-1, 8)
    assert len(ref_peaks) >= 1
    _same_peak_lists(peaks, ref_peaks, thr)

    # the per-pixel sums over all 4,700 orientations (compensated FP32 per batch,
    # FP64 across batches) through the C ABI on the oracle's prepared inputs
    with core.SearchCore(X, Y, T, histogram_min_scaled=hmin, histogram_step_scaled=hstep) as sc:
        sc.set_template(tspec)
        sc.set_image(ispec)
        sc.run_plane(filt, ang)
        _check_search_state(sc.results(), st, X, Y)
        # the FP16 tensor-core form of the same search: MIP and z-score error against the oracle
        sc.reset()
        sc.set_precision(core.PRECISION_FP16_TENSOR)
        sc.run_plane(filt, ang)
        _check_fp16_form(sc.results(), st, len(ang), X, Y)


def test_config2_contiguous_orientations_match_oracle():
    T, PIXEL, DEFOCUS = 256, 1.0, 12000.0
    vol = synthetic.template_volume(T, PIXEL, 120000, 110.0, seed=20261206)
    img, _ = synthetic.micrograph(4096, 4096, PIXEL, 120000, 110.0, 80, 0.03, DEFOCUS, seed=20261207,
                                  atom_seed=20261206)
    X = Y = 4096
    ispec, curve = O.whiten_image(img.astype(np.float64))
    tspec = O.prepare_template(vol.astype(np.float64))
    filt = O.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=DEFOCUS,
                               defocus2=DEFOCUS, pixel_size=PIXEL)
    grid = O.search_grid(2.5)
    ang_all = O.orientation_list(grid, O.psi_list(0.0, 1.5, 360.0))
    assert len(ang_all) == 1595420
    ang = ang_all[800000:800256]          # 256 contiguous orientations of the grid, theta near 90 deg
    hmin, hstep = histogram_scaled(X, Y)
    st = O.SearchState(X, Y)
    O.search(st, tspec, ispec, filt, ang, hist_min_scaled=hmin, hist_step_scaled=hstep)
    with core.SearchCore(X, Y, T, histogram_min_scaled=hmin, histogram_step_scaled=hstep,
                         orientation_batch=128) as sc:
        sc.set_template(tspec)
        sc.set_image(ispec)
        sc.run_plane(filt, ang)
        got = sc.results()
    _check_search_state(got, st, X, Y)
    with core.SearchCore(X, Y, T, histogram_min_scaled=hmin, histogram_step_scaled=hstep,
                         orientation_batch=128) as sc:
        sc.set_precision(core.PRECISION_FP16_TENSOR)
        sc.set_template(tspec)
        sc.set_image(ispec)
        sc.run_plane(filt, ang)
        _check_fp16_form(sc.results(), st, len(ang), X, Y)
    # the peak list over these orientations: the reference's loop on both z maps
    sq = np.sqrt(float(X * Y))
    _, z_ref, _, _ = O.finalize(st, len(ang), sq)
    gs = O.SearchState(X, Y)
    gs.mip[:], gs.sum[:], gs.sumsq[:] = got["mip"], got["sum"], got["sumsq"]
    _, z_got, _, _ = O.finalize(gs, len(ang), sq)
    assert np.abs(z_got - z_ref).max() <= Z_TOL
    shape = (Y, X)
    # the reference's expected threshold for these 256 orientations (about one chance peak)
    thr = float(np.float32(np.sqrt(np.float32(2.0))) * np.float32(O.erfcinv(2.0 / (float(X) * Y * len(ang)))))
    maps_ref = [st.psi.reshape(shape), st.theta.reshape(shape), st.phi.reshape(shape),
                np.zeros(shape, np.float32), np.zeros(shape, np.float32)]
    maps_got = [got["psi"].reshape(shape), got["theta"].reshape(shape), got["phi"].reshape(shape),
                np.zeros(shape, np.float32), np.zeros(shape, np.float32)]
    p_ref = reference_peaks(z_ref.reshape(shape), maps_ref, thr, 10, T, PIXEL)
    p_got = reference_peaks(z_got.reshape(shape), maps_got, thr, 10, T, PIXEL)
    _same_peak_lists(p_got, p_ref, thr)
