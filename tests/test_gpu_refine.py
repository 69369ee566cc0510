"""refine_template on the GPU against the oracle's restatement
(oracle/refine.py): the batched TemplateScore (tm_refine_score) candidate by
candidate, with and without the pixel-size change and the padded template,
and the refine_template program end to end on the maps of a match_template
run -- the peaks, the refined parameters and the refined MIP."""
import os
import subprocess

import numpy as np
import pytest

from cistem_downstream_bah_b200 import core
from cistem_downstream_bah_b200 import hostprep as H
from cistem_downstream_bah_b200 import synthetic
from oracle import oracle as O
from oracle import refine as OR

pytestmark = pytest.mark.gpu

PIXEL, DEFOCUS = 2.0, 8000.0


def _particles(T, seed=31, n_particles=3):
    # 256 x 256: a size the search has a kernel variant for with T = 32
    vol = synthetic.template_volume(T, PIXEL, n_atoms=600, radius_A=T * PIXEL * 0.3, seed=seed)
    img, truth = synthetic.micrograph(256, 256, PIXEL, n_atoms=600, radius_A=T * PIXEL * 0.3,
                                      n_particles=n_particles, snr=2.0, defocus_A=DEFOCUS, seed=seed + 1, atom_seed=seed)
    return vol.astype(np.float32), img.astype(np.float32), truth


@pytest.mark.parametrize("T,TP", [(32, 32), (32, 64), (48, 48)])
def test_batched_scores_match_oracle(T, TP):
    vol, img, truth = _particles(T)
    white, curve = OR.refine_whiten(img)
    windows = [OR.window_particle(white, int(x) - 128, int(y) - 128, T) for (x, y) in truth["positions"]]
    pspec = [OR.particle_spectrum(w) for w in windows]
    tspec = H.padded_template_spectrum(vol, TP)
    ref_tspec = tspec.astype(np.complex128)
    filters = [O.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=d, defocus2=d,
                                   pixel_size=PIXEL) for d in (7900.0, 8000.0, 8150.0)]
    factors = [1.0, 1.02, 0.985]
    rc = core.RefineCore(tspec, T, max_batch=16, max_particles=4, max_filters=4, max_operators=4)
    for k, s in enumerate(pspec):
        rc.set_particle(k, s)
    for k, f in enumerate(filters):
        rc.set_filter(k, f)
    op_slot = {}
    for f in factors[1:]:
        info, ar, ai, brt, bit = H.pixel_size_operator(TP, T, f)
        op_slot[f] = len(op_slot)
        rc.set_operator(op_slot[f], ar, ai, brt, bit, info["has_pad_value"])
    rng = np.random.default_rng(T + TP)
    n = 40
    euler = np.stack([rng.uniform(0, 360, n), rng.uniform(0, 180, n), rng.uniform(0, 360, n)], 1).astype(np.float32)
    part = rng.integers(0, len(pspec), n)
    filt = rng.integers(0, len(filters), n)
    fac = [factors[i] for i in rng.integers(0, len(factors), n)]
    ops = [-1 if f == 1.0 else op_slot[f] for f in fac]
    got = rc.score(euler, part, filt, ops)
    rc.close()
    ref = np.array([OR.template_score(ref_tspec, T, *euler[i], filters[filt[i]], pspec[part[i]], fac[i])
                    for i in range(n)])
    scale = np.abs(ref[:, 0]).max()
    assert np.abs(got[:, 0] - ref[:, 0]).max() <= 1e-4 * scale
    same = (got[:, 1] == ref[:, 1]) & (got[:, 2] == ref[:, 2])
    assert same.mean() >= 0.95, np.nonzero(~same)


def _match_template(tmp, img_path, tpl_path, T):
    names = ["mip", "psi", "theta", "phi", "defocus", "pixel", "scaled", "avg", "std"]
    f = {n: str(tmp / f"mt_{n}.mrc") for n in names}
    args = [img_path, tpl_path, PIXEL, 300.0, 2.7, 0.07, DEFOCUS, DEFOCUS, 0.0, 300.0, 8.0, 15.0, 20,
            200.0, 100.0, 0.0, 0.0, 1.0, "no", 0.0, 0.0,
            f["mip"], f["psi"], f["theta"], f["phi"], f["defocus"], f["pixel"], f["scaled"], f["avg"], "C1",
            15.0, str(tmp / "hist.txt"), -1, -1, 0, 0, f["std"], "/dev/null", "/dev/null", 10.0, "yes", 1]
    r = subprocess.run([H.CLI_PATH, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return f


def test_refine_program_matches_oracle(tmp_path):
    T = 32
    vol, img, truth = _particles(T, seed=47, n_particles=4)   # three particles at least 50 px from the edges
    H.write_mrc(tmp_path / "img.mrc", img, PIXEL)
    H.write_mrc(tmp_path / "tpl.mrc", vol, PIXEL)
    mt = _match_template(tmp_path, str(tmp_path / "img.mrc"), str(tmp_path / "tpl.mrc"), T)
    maps = {k: H.read_mrc(mt[n])[0][0] for k, n in (("mip", "mip"), ("scaled_mip", "scaled"), ("psi", "psi"),
                                                      ("theta", "theta"), ("phi", "phi"), ("defocus", "defocus"),
                                                      ("pixel_size", "pixel"))}
    outs = {k: str(tmp_path / f"rf_{k}.mrc") for k in ("psi", "theta", "phi", "defocus", "pixel", "mip", "scaled")}
    radius = 400.0   # compared with the squared distance: peaks 20 px apart
    # the three highest peaks of the coarse search (its z-scores are modest at this grid)
    top = OR.find_peaks(maps["scaled_mip"], -1e30, radius)[:3]
    threshold = float(top[-1][2]) - 1e-3
    prm = dict(pixel_size=PIXEL, defocus1=DEFOCUS, defocus2=DEFOCUS, angular_step=2.0, in_plane_angular_step=2.0,
               defocus_search_range=200.0, defocus_search_step=10.0, pixel_size_search_range=0.0,
               pixel_size_search_step=0.01, xy_change_threshold=10.0, exclude_above_xy_threshold=False)
    args = [str(tmp_path / "img.mrc"), str(tmp_path / "tpl.mrc"), PIXEL, 300.0, 2.7, 0.07, DEFOCUS, DEFOCUS, 0.0,
            300.0, 8.0, 2.0, prm["angular_step"], 20, prm["defocus_search_range"], prm["defocus_search_step"],
            prm["pixel_size_search_range"], prm["pixel_size_search_step"], 1.0, "no", 0.0, 0.0,
            mt["mip"], mt["scaled"], mt["psi"], mt["theta"], mt["phi"], mt["defocus"], mt["pixel"],
            outs["psi"], outs["theta"], outs["phi"], outs["defocus"], outs["pixel"], outs["mip"], outs["scaled"],
            threshold, radius, prm["xy_change_threshold"], "no", "C1", prm["in_plane_angular_step"], -1, -1, 1, 0, 1, 1,
            "/dev/null", 0.0, ""]
    assert len(args) == 51
    r = subprocess.run([H.REFINE_CLI_PATH, *map(str, args)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "Refine Template: Normal termination" in r.stdout
    got = {k: H.read_mrc(v)[0][0] for k, v in outs.items()}
    # the oracle: same peaks, windows, filters and descent, FP64 TemplateScore
    peaks = OR.find_peaks(maps["scaled_mip"], threshold, radius)
    assert len(peaks) == 3
    white, curve = OR.refine_whiten(img)
    pspec = [OR.particle_spectrum(OR.window_particle(white, int(x), int(y), T)) for (x, y, _) in peaks]
    tspec = O.prepare_template(vol.astype(np.float64))
    fcache = {}

    def score(c):
        phi, theta, psi, df1, df2, factor, k = c
        key = (float(df1), float(df2))
        if key not in fcache:
            fcache[key] = O.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07,
                                              defocus1=float(df1), defocus2=float(df2), pixel_size=PIXEL)
        return OR.template_score(tspec, T, float(phi), float(theta), float(psi), fcache[key], pspec[k], float(factor))

    ref_maps, rows = OR.refine(maps, [(x, y) for (x, y, _) in peaks], prm, T, score)
    for k, rk in (("psi", "psi"), ("theta", "theta"), ("phi", "phi"), ("defocus", "defocus"), ("pixel", "pixel_size")):
        assert np.array_equal(got[k], ref_maps[rk]), k
    for k, rk in (("mip", "mip"), ("scaled", "scaled_mip")):
        assert np.array_equal(got[k] != 0, ref_maps[rk] != 0), k
        assert np.abs(got[k] - ref_maps[rk]).max() <= 1e-4 * np.abs(ref_maps[rk]).max(), k
    # refinement raised every peak's score over its start
    assert np.all(rows[:, 15] > -1e-3)
