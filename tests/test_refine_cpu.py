"""refine_template's host side on the CPU against the oracle's restatement
(oracle/refine.py): the pixel-size operator against the literal
ChangePixelSize chain, the particle windows, the peak picking, the whitening,
the padded template spectrum, and the coordinate descent itself -- the
candidates it scores, in order, and every output -- with a synthetic score
shared by both sides."""
import math
import subprocess

import numpy as np
import pytest

from cistem_downstream_bah_b200 import hostprep as H
from cistem_downstream_bah_b200 import synthetic
from oracle import oracle as O
from oracle import refine as OR

f32 = np.float32


@pytest.mark.parametrize("nin,nout,factor", [(32, 32, 1.02), (32, 32, 0.975), (48, 48, 1.013), (64, 32, 1.01),
                                             (64, 32, 0.99)])
def test_pixel_size_operator_matches_the_literal_chain(nin, nout, factor):
    rng = np.random.default_rng(nin + nout)
    P = rng.normal(size=(nin, nin)) + 0.3
    info, ar, ai, brt, bit = H.pixel_size_operator(nin, nout, factor)
    assert not info["identity"] and info["pad"] == 1000 and info["has_pad_value"]
    pv = float(OR.average_in_disc(P, f32(0.45) * f32(nin)))
    U = P - pv
    got = ar.astype(np.float64) @ U @ brt.astype(np.float64) - ai.astype(np.float64) @ U @ bit.astype(np.float64) + pv
    ref = O.irfft2(OR.change_pixel_size_fft(P, nout, factor), nout)
    assert np.abs(got - ref).max() <= 2e-5 * np.abs(ref).max()


def test_pixel_size_operator_identity_within_tolerance():
    info = H.pixel_size_operator(32, 32, 1.0005)[0]
    assert info["identity"]


@pytest.mark.parametrize("shape,peak", [((200, 240), (10, -7)), ((200, 240), (-100, 90)), ((128, 96), (0, 0))])
def test_particle_window_matches_the_flat_shift(shape, peak):
    rng = np.random.default_rng(3)
    img = rng.normal(size=shape).astype(np.float32)
    got = H.window_particle(img, peak[0], peak[1], 32)
    ref = OR.window_particle(img.astype(np.float64), peak[0], peak[1], 32)
    assert np.array_equal(got, ref.astype(np.float32))


def test_refine_peaks_match_the_reference_loop():
    rng = np.random.default_rng(4)
    z = rng.normal(size=(220, 260)).astype(np.float32)
    for (x, y, v) in [(120, 100, 12.0), (60, 160, 9.0), (200, 60, 8.0), (121, 101, 11.5), (30, 30, 20.0)]:
        z[y, x] = v
    got = H.refine_find_peaks(z, 7.5, 10.0)
    ref = OR.find_peaks(z, 7.5, 10.0)
    assert len(got) == len(ref) >= 3
    assert np.array_equal(got, np.array(ref, np.float32))


def test_refine_whitening_matches_oracle():
    img, _ = synthetic.micrograph(96, 128, 2.0, 300, 20.0, 2, 0.5, 8000.0, seed=7)
    got = H.refine_whiten(img.astype(np.float32))
    ref, _ = OR.refine_whiten(img.astype(np.float32))
    assert np.abs(got - ref).max() <= 1e-5 * np.abs(ref).max()


@pytest.mark.parametrize("T,TP", [(16, 16), (16, 32)])
def test_padded_template_spectrum_matches_oracle(T, TP):
    rng = np.random.default_rng(5)
    vol = rng.normal(size=(T, T, T)).astype(np.float32)
    got = H.padded_template_spectrum(vol, TP)
    if TP == T:
        ref = O.prepare_template(vol.astype(np.float64))
    else:
        v = vol.astype(np.float64)
        edge = np.concatenate([v[0].ravel(), v[-1].ravel(), v[1:-1, [0, -1], :].ravel(), v[1:-1, 1:-1, [0, -1]].ravel()])
        big = np.full((TP, TP, TP), float(f32(edge.sum() / f32(edge.size))))
        o = TP // 2 - T // 2
        big[o:o + T, o:o + T, o:o + T] = v
        ref = O.rfft3(big) / TP ** 3
        ref[0, 0, 0] = 0
        ref = O.swap_quadrants(ref, TP)
    assert np.abs(got - ref).max() <= 1e-6 * np.abs(ref).max()


def _score_fn(targets):
    def score(c):
        phi, theta, psi, df1, _, factor, k = c
        t = [float(v) for v in targets[k]]
        a, b, d = (float(phi) - t[0]) / 3.0, (float(theta) - t[1]) / 3.0, (float(psi) - t[2]) / 3.0
        e, f = (float(df1) - t[3]) / 300.0, (float(factor) - t[4]) * 50.0
        v = 10.0 - a * a - b * b - d * d - e * e - f * f
        x = float(int(math.floor(abs(float(phi) - t[0]) * 10.0)) % 3 - 1)
        y = float(int(math.floor(abs(float(psi) - t[2]) * 10.0)) % 3 - 1)
        return float(f32(v)), x, y
    return score


@pytest.mark.parametrize("pixel_range,defocus_range", [(0.0, 200.0), (0.02, 200.0), (0.02, 0.0)])
def test_descent_matches_the_reference_loops(pixel_range, defocus_range):
    """Every candidate the descent scores, its order, and all outputs."""
    rng = np.random.default_rng(6)
    ny, nx = 120, 140
    maps = {k: np.zeros((ny, nx), np.float32) for k in H.REFINE_MAPS}
    maps["mip"][:] = 5.0
    maps["scaled_mip"][:] = 8.0
    maps["psi"][:] = rng.integers(0, 36, size=(ny, nx)) * 10.0
    maps["theta"][:] = rng.integers(0, 18, size=(ny, nx)) * 10.0
    maps["phi"][:] = rng.integers(0, 36, size=(ny, nx)) * 10.0
    maps["defocus"][:] = rng.integers(-2, 3, size=(ny, nx)) * 100.0
    maps["pixel_size"][:] = 0.0
    peaks = [(10.0, -5.0), (-30.0, 20.0), (11.0, -4.0)]
    targets = []
    for (x, y) in peaks:
        yy, xx = int(y + ny // 2), int(x + nx // 2)
        targets.append([maps["phi"][yy, xx] + 1.3, maps["theta"][yy, xx] - 0.7, maps["psi"][yy, xx] + 0.45,
                        8000.0 + maps["defocus"][yy, xx] + 130.0, 1.0 + 0.3 * pixel_range])
    params = dict(pixel_size=1.5, defocus1=8000.0, defocus2=8000.0, angular_step=0.5, in_plane_angular_step=0.25,
                  defocus_search_range=defocus_range, defocus_search_step=10.0, pixel_size_search_range=pixel_range,
                  pixel_size_search_step=0.01, xy_change_threshold=10.0, exclude_above_xy_threshold=False)
    plist = [params[k] for k in ("pixel_size", "defocus1", "defocus2", "angular_step", "in_plane_angular_step",
                                 "defocus_search_range", "defocus_search_step", "pixel_size_search_range",
                                 "pixel_size_search_step", "xy_change_threshold")] + [0.0, 1.0]
    targets = np.array(targets, np.float64)
    got_maps, got_rows, got_log = H.refine_synthetic(maps, np.array(peaks), targets, plist)
    log = []
    ref_maps, ref_rows = OR.refine(maps, peaks, params, 32, _score_fn(targets), log=log)
    ref_log = np.array([[c[0], c[1], c[2], c[3], c[5], c[6]] for c in log], np.float32)
    assert got_log.shape == ref_log.shape and len(ref_log) > 50
    assert np.array_equal(got_log, ref_log)
    assert np.array_equal(got_rows, ref_rows)
    for k in H.REFINE_MAPS:
        assert np.array_equal(got_maps[k], ref_maps[k]), k
    # the descent moved every peak towards its target
    assert np.all(np.abs(ref_rows[:, 4] - np.array(targets)[:, 0]) <= 0.5)


def test_refine_program_usage():
    r = subprocess.run([H.REFINE_CLI_PATH, "only-one-argument"], capture_output=True, text=True, timeout=30)
    assert r.returncode == 2 and "ARG50" in r.stderr


def test_refine_program_interactive_without_peaks(tmp_path):
    """The prompts of DoInteractiveUserInput, scripted; no peak above the
    threshold, so the program only reads, whitens and writes (no GPU)."""
    rng = np.random.default_rng(9)
    ny, nx, T = 120, 128, 16
    H.write_mrc(tmp_path / "img.mrc", rng.normal(size=(ny, nx)).astype(np.float32), 1.5)
    H.write_mrc(tmp_path / "tpl.mrc", rng.normal(size=(T, T, T)).astype(np.float32), 1.5)
    maps = {}
    for k in ("mip", "scaled", "psi", "theta", "phi", "defocus", "pixel"):
        maps[k] = rng.normal(size=(ny, nx)).astype(np.float32) if k != "scaled" else np.zeros((ny, nx), np.float32)
        H.write_mrc(tmp_path / f"in_{k}.mrc", maps[k], 1.5)
    outs = [str(tmp_path / f"out_{k}.mrc") for k in ("mip", "scaled", "psi", "theta", "phi", "defocus", "pixel")]
    answers = [str(tmp_path / "img.mrc"), str(tmp_path / "tpl.mrc")] + \
        [str(tmp_path / f"in_{k}.mrc") for k in ("mip", "scaled", "psi", "theta", "phi", "defocus", "pixel")] + \
        outs + ["7.5", "10", "1.5", "300", "2.7", "0.07", "10000", "10000", "0", "0", "0.2", "0.1", "200", "10",
                "0.1", "0.01", "1.0", "0", "10", "no", "1", "2"]
    r = subprocess.run([H.REFINE_CLI_PATH], input="\n".join(answers) + "\n", capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "Peak threshold" in r.stdout and "Refining 0 positions" in r.stdout
    got = {k: H.read_mrc(o)[0][0] for k, o in zip(("mip", "scaled", "psi", "theta", "phi", "defocus", "pixel"), outs)}
    assert not got["mip"].any() and not got["scaled"].any()
    for k in ("psi", "theta", "phi", "defocus", "pixel"):
        assert np.array_equal(got[k], maps[k]), k
