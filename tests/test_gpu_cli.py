"""The match_template program (C++ host over the C ABI) end to end on the GPU,
against the oracle pipeline: the reference CPU path restated (whitening,
template spectrum, projection filters, the search over three defocus planes,
statistics, resize to the original micrograph, the histogram file)."""
import os
import subprocess

import numpy as np
import pytest

from cistem_downstream_bah_b200 import hostprep as H
from cistem_downstream_bah_b200 import synthetic
from oracle import oracle as O

pytestmark = pytest.mark.gpu

T, PIXEL, DEFOCUS = 32, 2.0, 8000.0
STEP, PSI_STEP, DF_RANGE, DF_STEP = 20.0, 20.0, 200.0, 200.0


def _files(tmp):
    names = ["mip", "psi", "theta", "phi", "defocus", "pixel", "scaled", "avg", "std"]
    return {n: str(tmp / f"{n}.mrc") for n in names}


def _job_args(tmp, img_path, tpl_path, first=-1, last=-1):
    f = _files(tmp)
    args = [img_path, tpl_path, PIXEL, 300.0, 2.7, 0.07, DEFOCUS, DEFOCUS, 0.0, 300.0, 8.0, STEP, 20,
            DF_RANGE, DF_STEP, 0.0, 0.0, 1.0, "no", 0.0, 0.0,
            f["mip"], f["psi"], f["theta"], f["phi"], f["defocus"], f["pixel"], f["scaled"], f["avg"], "C1",
            PSI_STEP, str(tmp / "hist.txt"), first, last, 0, 0, f["std"], "/dev/null", str(tmp / "result.mrc"), 10.0,
            "yes", 1]
    assert len(args) == 42
    return f, [str(a) for a in args]


def _run_cli(tmp, img_path, tpl_path):
    f, args = _job_args(tmp, img_path, tpl_path)
    r = subprocess.run([H.CLI_PATH, *args], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return f, r.stdout


def _inputs(tmp_path):
    vol = synthetic.template_volume(T, PIXEL, n_atoms=600, radius_A=T * PIXEL * 0.3, seed=21)
    img, truth = synthetic.micrograph(250, 256, PIXEL, n_atoms=600, radius_A=T * PIXEL * 0.3, n_particles=3,
                                      snr=2.0, defocus_A=DEFOCUS, seed=22, atom_seed=21)
    H.write_mrc(tmp_path / "img.mrc", img, PIXEL)
    H.write_mrc(tmp_path / "tpl.mrc", vol, PIXEL)
    return vol, img, truth


def _oracle_pipeline(img, vol):
    Y0, X0 = img.shape
    X, Y = O.factorize_dimension(X0, T), O.factorize_dimension(Y0, T)
    padded = O.clip_into_real(img.astype(np.float64), X, Y, float(H.edge_mean(img)))
    ispec, curve = O.whiten_image(padded)
    tspec = O.prepare_template(vol.astype(np.float64))
    ang = O.orientation_list(O.search_grid(STEP), O.psi_list(0.0, PSI_STEP, 360.0))
    sq = np.sqrt(float(X * Y))
    hstep = np.float32((22.5 - (-12.5)) / np.float32(512))
    st = O.SearchState(X, Y)
    n_planes = 0
    for i in (-1, 0, 1):
        filt = O.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=DEFOCUS,
                                   defocus2=DEFOCUS, pixel_size=PIXEL, defocus_offset=i * DF_STEP)
        O.search(st, tspec, ispec, filt, ang, hist_min_scaled=-12.5 / sq, hist_step_scaled=float(hstep) / sq,
                 defocus_value=float(np.float32(i) * np.float32(DF_STEP)), pixel_value=0.0)
        n_planes += 1
    n_total = len(ang) * n_planes
    mip, z, avg, sd = O.finalize(st, n_total, sq)
    shape = (Y, X)

    def back(a, edge):
        a = np.asarray(a, np.float32).reshape(shape)
        return O.clip_into_real(a.astype(np.float64), X0, Y0, float(H.edge_mean(a)) if edge else 0.0).astype(np.float32)

    # the runner-up margin exceeds 1e-4 of the MIP scale (as the search parity tests)
    decided = ((st.mip - st.second) > 1e-4 * np.abs(st.mip).max()).reshape(shape)
    return dict(mip=back(mip, True), scaled=back(z, True), avg=back(avg, True), std=back(sd, True),
                psi=back(st.psi, False), theta=back(st.theta, False), phi=back(st.phi, False),
                defocus=back(st.defocus, False), decided=O.clip_into_real(decided.astype(np.float64), X0, Y0, 0.0) > 0.5,
                hist=st.hist[:512], n_total=n_total, X0=X0, Y0=Y0)


def test_match_template_program_matches_oracle(tmp_path):
    vol, img, truth = _inputs(tmp_path)
    files, stdout = _run_cli(tmp_path, str(tmp_path / "img.mrc"), str(tmp_path / "tpl.mrc"))
    assert "old x, y; new x, y = 256 250 256 256" in stdout
    ref = _oracle_pipeline(img.astype(np.float32), vol.astype(np.float32))
    got = {k: H.read_mrc(v)[0][0] for k, v in files.items()}
    for k in got:
        assert got[k].shape == (250, 256), k
        assert abs(H.read_mrc(files[k])[1] - PIXEL) < 1e-6
    scale = np.abs(ref["mip"]).max()
    assert np.abs(got["mip"] - ref["mip"]).max() <= 1e-4 * scale
    assert np.abs(got["avg"] - ref["avg"]).max() <= 1e-4 * np.abs(ref["std"]).max()
    assert np.abs(got["std"] - ref["std"]).max() <= 1e-4 * np.abs(ref["std"]).max()
    assert np.abs(got["scaled"] - ref["scaled"]).max() <= 2e-3
    d = ref["decided"]
    assert d.mean() > 0.9
    for k in ("psi", "theta", "phi", "defocus"):
        assert np.array_equal(got[k][d], ref[k][d]), k
    assert np.array_equal(got["pixel"], np.zeros_like(got["pixel"]))
    # histogram text file: two comment lines, then 512 rows of 4 columns
    lines = open(tmp_path / "hist.txt").read().splitlines()
    assert lines[0].startswith("# Expected threshold = ")
    assert lines[1] == "# SNR, histogram, survival histogram, random survival histogram"
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[2:]])
    assert rows.shape == (512, 4)
    assert np.allclose(rows[:, 0], -12.5 + 35.0 / 512 * (np.arange(512) + 0.5), atol=1e-4)
    h = rows[:, 1]
    assert abs(h.sum() - ref["hist"].sum()) <= 2 + 1e-4 * ref["hist"].sum()
    assert np.all(np.abs(h - ref["hist"]) <= 2 + 1e-3 * ref["hist"])
    assert np.allclose(rows[:, 2], np.cumsum(h[::-1])[::-1])
    expected_threshold = np.sqrt(2.0) * O.erfcinv(2.0 / (256.0 * 250.0 * ref["n_total"]))
    assert lines[0] == "# Expected threshold = %.2f" % np.float32(expected_threshold)
    # the planted particles are found at their positions
    for (px, py) in truth["positions"]:
        y, x = int(round(py)), int(round(px))
        win = got["scaled"][max(0, y - 3):y + 4, max(0, x - 3):x + 4]
        assert win.max() > 4.0, (px, py, win.max())
    # the peak list next to the result image (argument 38): the reference's peak
    # loop on the written maps, and every planted particle above the threshold
    # and away from the edges is among the peaks
    rows = [ln.split() for ln in open(tmp_path / "result_peaks.txt").read().splitlines() if not ln.startswith("#")]
    peaks = np.array(rows, np.float32).reshape(-1, 8)
    ref_peaks = H.find_peaks(got["scaled"], got["psi"], got["theta"], got["phi"], got["defocus"], got["pixel"],
                             threshold=float(np.float32(np.sqrt(np.float32(2.0))) *
                                             np.float32(O.erfcinv(2.0 / (256.0 * 250.0 * ref["n_total"])))),
                             min_peak_radius=10, template_size=T,
                             pixel_size=PIXEL)
    assert np.allclose(peaks, ref_peaks[:, :8], rtol=1e-5, atol=1e-3)
    thr = float(lines[0].split("=")[1])
    assert len(peaks) >= 1 and np.all(peaks[:, 7] >= thr - 0.01)
    for (px, py) in truth["positions"]:
        y, x = int(round(py)), int(round(px))
        if min(px, py, 256 - px, 250 - py) < T // 4 + 2 or got["scaled"][y - 3:y + 4, x - 3:x + 4].max() < thr + 0.5:
            continue   # near an edge, or not above the threshold
        d = np.hypot(peaks[:, 0] / PIXEL - px, peaks[:, 1] / PIXEL - py)
        assert d.min() < 3.0, (px, py, d.min())
    # the result image: the template's projections at the peaks, positive values only
    montage, px = H.read_mrc(tmp_path / "result.mrc")
    montage = montage[0]
    assert montage.shape == (250, 256) and abs(px - PIXEL) < 1e-6 and montage.min() >= 0.0
    ref_montage = H.projection_montage(vol, [[p[8], p[9], p[2], p[3], p[4]] for p in ref_peaks], 256, 250)
    assert np.allclose(montage, ref_montage, rtol=1e-4, atol=1e-4 * ref_montage.max())
    for p in ref_peaks:
        assert montage[int(p[9]) - 3:int(p[9]) + 4, int(p[8]) - 3:int(p[8]) + 4].max() > 0


def test_worker_jobs_merged_by_the_master_match_the_local_run(tmp_path):
    """The distributed form: two worker jobs over the reference's split of the
    search positions write result arrays; match_template_merge merges them as
    the master does.  The merged maps equal the local run's (MIP and best
    parameters exactly where the local MIP is positive and decided; the float
    sums of the result arrays to 1e-4 of the deviation scale)."""
    _inputs(tmp_path)
    img, tpl = str(tmp_path / "img.mrc"), str(tmp_path / "tpl.mrc")
    (tmp_path / "local").mkdir()
    f_local, _ = _run_cli(tmp_path / "local", img, tpl)
    n_positions = len(H.search_grid(STEP))
    ranges = H.job_search_ranges(n_positions, 2)
    assert ranges[0][0] == 0 and ranges[1][1] == n_positions - 1
    arrays = []
    for j, (first, last) in enumerate(ranges):
        d = tmp_path / f"w{j}"
        d.mkdir()
        _, args = _job_args(d, img, tpl, first, last)
        r = subprocess.run([H.CLI_PATH, *args, str(d / "result.bin")], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
        assert "Result array of" in r.stdout
        assert not os.path.exists(d / "mip.mrc")   # a worker writes only its array
        arrays.append(str(d / "result.bin"))
    (tmp_path / "merged").mkdir()
    f_m, args = _job_args(tmp_path / "merged", img, tpl)
    r = subprocess.run([H.MERGE_CLI_PATH, *args, *arrays], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    local = {k: H.read_mrc(v)[0][0] for k, v in f_local.items()}
    merged = {k: H.read_mrc(v)[0][0] for k, v in f_m.items()}
    pos = local["mip"] > 0
    assert pos.mean() > 0.99
    assert np.array_equal(merged["mip"][pos], local["mip"][pos])
    # decided pixels: the runner-up over the whole search is not within 1e-4
    # of the MIP; the merged argmax then equals the local one
    ref = _oracle_pipeline(H.read_mrc(img)[0][0], H.read_mrc(tpl)[0])
    d = ref["decided"] & pos
    for k in ("psi", "theta", "phi", "defocus"):
        assert np.array_equal(merged[k][d], local[k][d]), k
    scale = np.abs(local["std"]).max()
    assert np.abs(merged["avg"] - local["avg"]).max() <= 1e-4 * scale
    assert np.abs(merged["std"] - local["std"]).max() <= 1e-4 * scale
    # where every correlation was <= 0 the master's MIP keeps its zero start
    # (ZeroFloatArray, match_template.cpp:2025), and so does its z-score
    assert np.abs(merged["scaled"][pos] - local["scaled"][pos]).max() <= 2e-3
    h_local = np.array([[float(v) for v in ln.split()] for ln in open(tmp_path / "local" / "hist.txt").read().splitlines()[2:]])
    lines = open(tmp_path / "merged" / "hist.txt").read().splitlines()
    h_m = np.array([[float(v) for v in ln.split()] for ln in lines[2:]])
    assert np.array_equal(h_m[:, :2], h_local[:, :2])
    assert lines[0] == open(tmp_path / "local" / "hist.txt").readline().rstrip("\n")

