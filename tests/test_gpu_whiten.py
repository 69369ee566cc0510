"""Micrograph whitening on the GPU (tm_whiten_micrograph, tm_set_micrograph)
against the host restatement of match_template.cpp:699-724 (host/prep.cpp,
itself checked against the oracle in test_host_cpu.py): the whitened
spectrum, the whitening curve, and a search plane run from either."""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import core, prep
from cistem_downstream_bah_b200 import hostprep as H
from cistem_downstream_bah_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ny,nx", [(256, 256), (288, 256), (1024, 1024), (2048, 2048)])
def test_device_whitening_matches_host(ny, nx):
    img, _ = synthetic.micrograph(ny, nx, 1.5, 800, 30.0, 6, 0.1, 9000.0, seed=ny + nx)
    img = img.astype(np.float32)
    img[10, 12] = 50.0   # an outlier the 5-sigma replacement removes
    spec, curve = core.whiten_micrograph(img)
    ref_spec, ref_curve = H.whiten(img)
    assert curve.shape == ref_curve.shape
    assert np.abs(curve - ref_curve).max() <= 1e-5 * np.abs(ref_curve).max()
    assert np.abs(spec - ref_spec).max() <= 2e-5 * np.abs(ref_spec).max()
    assert abs(np.linalg.norm(spec) - np.linalg.norm(ref_spec)) <= 1e-5 * np.linalg.norm(ref_spec)


def test_search_from_device_whitening_matches_host_whitening():
    T, X, Y = 32, 256, 256
    vol = synthetic.template_volume(T, 2.0, n_atoms=600, radius_A=20.0, seed=3)
    img, _ = synthetic.micrograph(Y, X, 2.0, 600, 20.0, 3, 1.0, 8000.0, seed=4, atom_seed=3)
    img = img.astype(np.float32)
    tspec = prep.template_spectrum(vol)
    angles = core.orientation_list(prep.search_grid(30.0), 0.0, 30.0, 360.0)[:64]
    results = []
    for use_device in (False, True):
        sc = core.SearchCore(X, Y, T, histogram_min_scaled=-12.5 / 256.0, histogram_step_scaled=35.0 / 512 / 256.0)
        sc.set_template(tspec)
        if use_device:
            curve = sc.set_micrograph(img)
        else:
            spec, curve = H.whiten(img)
            sc.set_image(spec)
        filt = prep.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=8000.0,
                                      defocus2=8000.0, pixel_size=2.0)
        sc.run_plane(filt, angles)
        results.append(sc.results())
        sc.close()
    a, b = results
    scale = np.abs(a["mip"]).max()
    assert np.abs(a["mip"] - b["mip"]).max() <= 1e-4 * scale
    agree = (a["psi"] == b["psi"]) & (a["theta"] == b["theta"]) & (a["phi"] == b["phi"])
    assert agree.mean() > 0.99
