"""Micrograph sizes without compiled kernels (the run-time-length kernels of
csrc/tm_generic.cuh) against the FP64 oracle.

The reference pads each side to the nearest size with small prime factors
(match_template.cpp:527-575); sizes just above a 2^a 3^b value get a factor 5
(or 7, 11, 13), e.g. 1030 -> 1080 = 2^3 3^3 5.  Bars as the parity tests: MIP
within 1e-4 of the MIP scale, best orientation equal where the oracle's
runner-up is more than 1e-4 of the scale below, sums within 1e-5 of their
scale, histogram within 0.1% (+2).
"""
import subprocess

import numpy as np
import pytest

from cistem_downstream_bah_b200 import core
from cistem_downstream_bah_b200 import hostprep as H
from cistem_downstream_bah_b200 import synthetic
from oracle import oracle as O
from tests.search_cases import histogram_scaled, make_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("T,X,Y", [(64, 1152, 1080), (32, 560, 700), (64, 729, 640)])
def test_generic_size_search_matches_oracle(T, X, Y):
    case = make_case(T=T, X=X, Y=Y, pixel_size=1.5, n_particles=4, snr=0.5, angular_step=30.0, psi_step=30.0)
    with core.SearchCore(X, Y, T, histogram_min_scaled=case["hmin"], histogram_step_scaled=case["hstep"]) as sc:
        sc.set_template(case["tspec"])
        sc.set_image(case["ispec"])
        sc.run_plane(case["filt"], case["angles"])
        got = sc.results()
    st = O.SearchState(X, Y)
    O.search(st, case["tspec"], case["ispec"], case["filt"], case["angles"], hist_min_scaled=case["hmin"],
             hist_step_scaled=case["hstep"])
    scale = np.abs(st.mip).max()
    assert np.abs(got["mip"] - st.mip).max() <= 1e-4 * scale
    decided = (st.mip - st.second) > 1e-4 * scale
    assert decided.mean() > 0.85       # the comparison covers most pixels
    for k in ("psi", "theta", "phi"):
        assert np.array_equal(got[k][decided], getattr(st, k)[decided]), k
    assert np.abs(got["sum"] - st.sum).max() <= 1e-5 * np.abs(st.sum).max()
    assert np.abs(got["sumsq"] - st.sumsq).max() <= 1e-5 * np.abs(st.sumsq).max()
    assert np.all(np.abs(got["hist"] - st.hist[:512]) <= 1e-3 * st.hist[:512] + 2)


def test_generic_whitening_matches_oracle():
    rng = np.random.default_rng(5)
    img = rng.standard_normal((1080, 1152)).astype(np.float32)
    spec, curve = core.whiten_micrograph(img)
    ref, ref_curve = O.whiten_image(img.astype(np.float64))
    assert np.abs(spec - ref).max() <= 2e-5 * np.abs(ref).max()
    assert np.abs(np.asarray(curve) - ref_curve).max() <= 1e-5 * np.abs(ref_curve).max()


def test_program_on_a_size_without_compiled_kernels(tmp_path):
    """A 1100 x 1030 micrograph pads to 1152 x 1080 (2^7 3^2 and 2^3 3^3 5): the
    match_template program runs it end to end and matches the oracle pipeline."""
    T, PIXEL, DEFOCUS, STEP = 32, 2.0, 8000.0, 30.0
    vol = synthetic.template_volume(T, PIXEL, n_atoms=600, radius_A=T * PIXEL * 0.3, seed=31)
    img, _ = synthetic.micrograph(1030, 1100, PIXEL, n_atoms=600, radius_A=T * PIXEL * 0.3, n_particles=4, snr=1.0,
                                  defocus_A=DEFOCUS, seed=32, atom_seed=31)
    H.write_mrc(tmp_path / "img.mrc", img, PIXEL)
    H.write_mrc(tmp_path / "tpl.mrc", vol, PIXEL)
    names = ["mip", "psi", "theta", "phi", "defocus", "pixel", "scaled", "avg", "std"]
    f = {n: str(tmp_path / f"{n}.mrc") for n in names}
    args = [str(tmp_path / "img.mrc"), str(tmp_path / "tpl.mrc"), PIXEL, 300.0, 2.7, 0.07, DEFOCUS, DEFOCUS, 0.0,
            300.0, 2.0 * PIXEL, STEP, 20, 0.0, 0.0, 0.0, 0.0, 1.0, "no", 0.0, 0.0,
            f["mip"], f["psi"], f["theta"], f["phi"], f["defocus"], f["pixel"], f["scaled"], f["avg"], "C1",
            STEP, str(tmp_path / "hist.txt"), -1, -1, 0, 0, f["std"], "/dev/null", "/dev/null", 10.0, "yes", 1]
    r = subprocess.run([H.CLI_PATH, *[str(a) for a in args]], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    assert "old x, y; new x, y = 1100 1030 1152 1080" in r.stdout
    X0, Y0 = 1100, 1030
    X, Y = O.factorize_dimension(X0, T), O.factorize_dimension(Y0, T)
    assert (X, Y) == (1152, 1080)
    padded = O.clip_into_real(img.astype(np.float64), X, Y, float(H.edge_mean(img)))
    ispec, curve = O.whiten_image(padded)
    tspec = O.prepare_template(vol.astype(np.float64))
    filt = O.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=DEFOCUS,
                               defocus2=DEFOCUS, pixel_size=PIXEL)
    ang = O.orientation_list(O.search_grid(STEP), O.psi_list(0.0, STEP, 360.0))
    hmin, hstep = histogram_scaled(X, Y)
    st = O.SearchState(X, Y)
    O.search(st, tspec, ispec, filt, ang, hist_min_scaled=hmin, hist_step_scaled=hstep)
    mip, z, avg, sd = O.finalize(st, len(ang), np.sqrt(float(X * Y)))
    back = lambda a: O.clip_into_real(np.asarray(a, np.float64).reshape(Y, X), X0, Y0, 0.0)
    got = {k: H.read_mrc(v)[0][0] for k, v in f.items()}
    inner = (slice(2, Y0 - 2), slice(2, X0 - 2))
    scale = np.abs(mip).max()
    assert np.abs(got["mip"][inner] - back(mip)[inner]).max() <= 1e-4 * scale
    assert np.abs(got["scaled"][inner] - back(z)[inner]).max() <= 2e-3
    decided = back(((st.mip - st.second) > 1e-4 * np.abs(st.mip).max()).astype(np.float64)) > 0.5
    for k in ("psi", "theta", "phi"):
        assert np.array_equal(got[k][decided], back(getattr(st, k))[decided].astype(np.float32)), k
