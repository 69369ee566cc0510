"""The distributed form of match_template on the CPU: the split of the search
positions into jobs, the worker's flat result array and the master's merge and
statistics (host/result_array.cpp), each against a numpy restatement of the
reference loops (src/gui/MatchTemplatePanel.cpp:674-784,
src/programs/match_template/match_template.cpp:1373-1530, 1545-1837,
2015-2103), plus the merge program's argument handling."""
import math
import subprocess

import numpy as np
import pytest

from cistem_downstream_bah_b200 import hostprep as H

f32 = np.float32


def _round(a):
    # myroundint(float): a + 0.5 in double
    a = float(np.float32(a))
    return int(a + 0.5) if a > 0 else int(a - 0.5)


def ref_job_ranges(n, jobs):
    per = f32(f32(n) / f32(jobs))
    if per < 1:
        per = f32(1)
    c = f32(0)
    out = []
    for j in range(jobs):
        if c >= n:
            c = f32(n - 1)
        first = _round(c)
        c = f32(c + per)
        if c >= n or j == jobs - 1:
            c = f32(n - 1)
        last = _round(c)
        c = f32(c + f32(1))
        out.append((first, last))
    return out


@pytest.mark.parametrize("n,jobs", [(10, 3), (4700, 7), (53874, 8), (1, 1), (3, 5), (241, 16), (1595, 64)])
def test_job_search_ranges_match_the_panel_loop(n, jobs):
    got = H.job_search_ranges(n, jobs)
    assert got == ref_job_ranges(n, jobs)
    if jobs <= n:
        # the ranges cover the grid in order; where the float counter reaches
        # the end early, the last jobs repeat the last position (as the panel's)
        assert got[0][0] == 0 and got[-1][1] == n - 1
        for (a, b), (c, d) in zip(got, got[1:]):
            assert a <= b and (c == b + 1 or c == d == n - 1)


def ref_average_in_disc(im, radius):
    ny, nx = im.shape
    cx, cy = nx // 2, ny // 2
    r2 = f32(radius) * f32(radius)
    x = (np.arange(nx) - cx).astype(f32) ** 2
    y = (np.arange(ny) - cy).astype(f32) ** 2
    d2 = (y[:, None] + x[None, :]).astype(f32)
    m = d2 <= r2
    return f32(im[m].astype(np.float64).sum() / m.sum())


def ref_clip(im, ox, oy, pad):
    ny, nx = im.shape
    out = np.full((oy, ox), pad, f32)
    for jj in range(oy):
        j = ny // 2 + (jj - oy // 2)
        if 0 <= j < ny:
            for ii in range(ox):
                i = nx // 2 + (ii - ox // 2)
                if 0 <= i < nx:
                    out[jj, ii] = im[j, i]
    return out


def ref_pack(maps, ox, oy, remove, ccs, sq, hist):
    ny, nx = maps["mip"].shape
    trim_x, trim_y = ox - remove, oy - remove
    central = f32(0.35 * (nx + ny - 2 * remove))
    if ox > nx:
        trim_x = nx - remove
    if oy > ny:
        trim_y = ny - remove
    pitch = ox + (2 if ox % 2 == 0 else 1)
    per = pitch * oy
    out = np.zeros(6 + 8 * per + 2 * len(hist), f32)
    out[:6] = [ox, oy, per, len(hist), ccs, sq]
    for k, name in enumerate(H.WORKER_MAPS):
        ca = ref_average_in_disc(maps[name], central)
        im = ref_clip(ref_clip(maps[name], trim_x, trim_y, ca), ox, oy, ca)
        block = np.zeros((oy, pitch), f32)
        block[:, :ox] = im
        out[6 + per * k:6 + per * (k + 1)] = block.ravel()
    out[6 + 8 * per:] = np.asarray(hist, np.int64).view(f32)
    return out


def _maps(rng, nx, ny, scale=1.0):
    m = {k: rng.normal(size=(ny, nx)).astype(f32) * f32(scale) for k in H.WORKER_MAPS}
    m["mip"] = np.abs(m["mip"]) + f32(0.1)
    m["sum"] = m["sum"] * f32(10)
    m["sumsq"] = np.abs(m["sumsq"]) * f32(100) + f32(50)
    for k in ("psi", "theta", "phi"):
        m[k] = rng.integers(0, 360, size=(ny, nx)).astype(f32)
    return m


@pytest.mark.parametrize("box,orig,remove", [((64, 48), (60, 45), 0), ((64, 48), (61, 40), 5), ((50, 50), (64, 50), 3)])
def test_worker_result_array_matches_the_reference_layout(box, orig, remove):
    rng = np.random.default_rng(1)
    nx, ny = box
    maps = _maps(rng, nx, ny)
    hist = rng.integers(0, 1 << 40, size=512)
    got = H.pack_worker_result(maps, orig[0], orig[1], remove, 1234.0, math.sqrt(nx * ny), hist)
    ref = ref_pack(maps, orig[0], orig[1], remove, f32(1234.0), f32(math.sqrt(nx * ny)), hist)
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.int32), ref.view(np.int32))


def ref_merge(arrays, use_gpu):
    a0 = arrays[0]
    per, bins = int(a0[2]), int(a0[3])
    col = np.zeros_like(a0)
    col[[0, 1, 2, 3, 5]] = a0[[0, 1, 2, 3, 5]]
    total = f32(0)
    hist = np.zeros(512, np.int64)
    for a in arrays:
        total = f32(total + a[4])
        src = [a[6 + per * k:6 + per * (k + 1)] for k in range(8)]
        dst = [col[6 + per * k:6 + per * (k + 1)] for k in range(8)]
        upd = src[0] > dst[0]
        for k in range(6):
            dst[k][upd] = src[k][upd]
        dst[6] += src[6]
        dst[7] += src[7]
        hist += a[6 + 8 * per:6 + 8 * per + 2 * bins].view(np.int64)[:512]
    nx, ny = int(col[0]), int(col[1])
    pitch = per // ny
    sq = float(col[5])

    def compact(v):
        return v.reshape(ny, pitch)[:, :nx]

    mip = col[6:6 + per].copy()
    out = {"mip": compact((mip.astype(np.float64) * sq).astype(f32))}
    for k, name in enumerate(("psi", "theta", "phi", "defocus", "pixel"), start=1):
        out[name] = compact(col[6 + per * k:6 + per * (k + 1)])
    sums = col[6 + per * 6:6 + per * 7] / total
    sqs = np.sqrt((col[6 + per * 7:6 + per * 8] / total - sums * sums).astype(f32))
    with np.errstate(invalid="ignore"):
        pos = sqs > 0
    z = np.where(pos, (mip - sums) / np.where(pos, sqs, 1), 0).astype(f32)
    sqs = np.where(pos, sqs, 0).astype(f32)
    out["scaled_mip"] = compact(z)
    out["avg"] = compact((sums.astype(np.float64) * sq).astype(f32))
    out["std"] = compact((sqs.astype(np.float64) * sq).astype(f32))
    step = f32((f32(22.5) - f32(-12.5)) / f32(512))
    t0 = f32(f32(-12.5) + step / f32(2))
    snr = (t0 + step * np.arange(512, dtype=f32)).astype(f32)
    surv = np.cumsum(hist[::-1])[::-1].astype(np.float64)
    area = f32(f32(nx) * f32(ny) * total)
    erfc = np.array([math.erfc(float(v) / float(np.sqrt(f32(2)))) for v in snr])
    expected = (erfc / 2.0) * float(area)
    if use_gpu:
        surv = surv * float(f32(expected.sum() / surv.sum()))
    out["rows"] = np.stack([snr.astype(np.float64), hist.astype(np.float64), surv, expected], 1)
    out["number_of_ccs"] = float(total)
    return out


@pytest.mark.parametrize("use_gpu", [True, False])
def test_master_merge_matches_the_reference_loops(use_gpu):
    rng = np.random.default_rng(2)
    nx, ny, ox, oy = 40, 36, 38, 33
    arrays = []
    for w in range(3):
        maps = _maps(rng, nx, ny)
        hist = rng.integers(0, 1000, size=512)
        arrays.append(H.pack_worker_result(maps, ox, oy, 2, 100.0 + w, math.sqrt(nx * ny), hist))
    got = H.merge_results(arrays, use_gpu=use_gpu)
    ref = ref_merge(arrays, use_gpu)
    assert got["number_of_ccs"] == ref["number_of_ccs"] == 303.0
    for k in ("mip", "psi", "theta", "phi", "defocus", "pixel"):
        assert np.array_equal(got[k], ref[k]), k
    for k in ("scaled_mip", "avg", "std"):
        assert np.allclose(got[k], ref[k], rtol=2e-6, atol=1e-6 * np.abs(ref[k]).max()), k
    assert np.array_equal(got["rows"][:, :2], ref["rows"][:, :2])
    assert np.allclose(got["rows"][:, 2:], ref["rows"][:, 2:], rtol=1e-5)
    thr = math.sqrt(2.0) * float(H.lib().tmh_erfcinv(2.0 / (float(ox) * float(oy) * 303.0)))
    assert abs(got["expected_threshold"] - thr) < 1e-5


def test_merge_is_order_insensitive_except_ties_and_sums_add():
    rng = np.random.default_rng(3)
    nx = ny = 32
    a = [H.pack_worker_result(_maps(rng, nx, ny), nx, ny, 0, 10.0, 32.0, np.arange(512)) for _ in range(2)]
    m1, m2 = H.merge_results(a), H.merge_results(a[::-1])
    assert np.array_equal(m1["mip"], m2["mip"])
    assert np.array_equal(m1["psi"], m2["psi"])
    assert np.array_equal(m1["rows"][:, 1], 2 * np.arange(512, dtype=np.float64))


def test_merge_rejects_mismatching_arrays():
    rng = np.random.default_rng(4)
    a = H.pack_worker_result(_maps(rng, 32, 32), 32, 32, 0, 1.0, 32.0, np.zeros(512))
    b = H.pack_worker_result(_maps(rng, 30, 32), 30, 32, 0, 1.0, 32.0, np.zeros(512))
    with pytest.raises(ValueError):
        H.merge_results([a, b])
    with pytest.raises(ValueError):
        H.merge_results([a[:100]])


def test_merge_program_usage():
    r = subprocess.run([H.MERGE_CLI_PATH], capture_output=True, text=True, timeout=30)
    assert r.returncode == 2 and "RESULT_ARRAY" in r.stderr


def test_merge_program_writes_the_master_outputs(tmp_path):
    rng = np.random.default_rng(5)
    nx, ny = 48, 40
    T = 16
    arrays = []
    for w in range(2):
        maps = _maps(rng, nx, ny)
        maps["mip"][20, 24] = 50.0 + w   # one clear peak
        a = H.pack_worker_result(maps, nx, ny, 0, 500.0, math.sqrt(nx * ny), rng.integers(0, 100, size=512))
        p = tmp_path / f"w{w}.bin"
        a.tofile(p)
        arrays.append(a)
    vol = rng.normal(size=(T, T, T)).astype(f32)
    H.write_mrc(tmp_path / "tpl.mrc", vol, 1.5)
    names = ["mip", "psi", "theta", "phi", "defocus", "pixel", "scaled", "avg", "std"]
    f = {n: str(tmp_path / f"{n}.mrc") for n in names}
    args = ["img.mrc", str(tmp_path / "tpl.mrc"), 1.5, 300, 2.7, 0.07, 1e4, 1e4, 0, 300, 8, 15, 20, 0, 0, 0, 0, 1,
            "no", 0, 0, f["mip"], f["psi"], f["theta"], f["phi"], f["defocus"], f["pixel"], f["scaled"], f["avg"],
            "C1", 15, str(tmp_path / "hist.txt"), 0, 10, 1, 2, f["std"], "/dev/null", str(tmp_path / "res.mrc"), 5,
            "yes", 1]
    assert len(args) == 42
    r = subprocess.run([H.MERGE_CLI_PATH, *map(str, args), str(tmp_path / "w0.bin"), str(tmp_path / "w1.bin")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stdout + r.stderr
    ref = H.merge_results(arrays, use_gpu=True)
    pairs = dict(mip="mip", psi="psi", theta="theta", phi="phi", defocus="defocus", pixel="pixel",
                 scaled="scaled_mip", avg="avg", std="std")
    for n, k in pairs.items():
        data, px = H.read_mrc(f[n])
        assert px == 1.0
        assert np.array_equal(data[0], ref[k]), n
    lines = open(tmp_path / "hist.txt").read().splitlines()
    assert lines[0] == "# Expected threshold = %.2f" % ref["expected_threshold"]
    assert lines[1] == "# histogram, expected histogram, survival histogram, expected survival histogram"
    rows = np.array([[float(v) for v in ln.split()] for ln in lines[2:]])
    assert np.allclose(rows, ref["rows"], rtol=1e-6, atol=1e-6)
    pk = [ln.split() for ln in open(tmp_path / "res_peaks.txt").read().splitlines() if not ln.startswith("#")]
    peaks = np.array(pk, np.float32).reshape(-1, 8)
    z = ref["scaled_mip"]
    ref_pk = H.find_peaks(z, ref["psi"], ref["theta"], ref["phi"], ref["defocus"], ref["pixel"],
                          ref["expected_threshold"], 5, T, 1.5)
    assert len(ref_pk) >= 1
    assert np.allclose(peaks, ref_pk[:, :8], rtol=1e-5, atol=1e-3)
    montage, px = H.read_mrc(tmp_path / "res.mrc")
    assert px == 1.0 and montage.shape[1:] == (ny, nx)
