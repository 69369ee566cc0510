"""Template spectrum prepared on the GPU (tm_template_spectrum,
tm_set_template_volume) against the host restatement of
match_template.cpp:842-845 (host/prep.cpp, template_spectrum(), checked
against the oracle in test_host_cpu.py), with and without the pixel-size
change, and a search plane run from either."""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import core, prep
from cistem_downstream_bah_b200 import hostprep as H
from cistem_downstream_bah_b200 import synthetic

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("T,factor", [(32, 1.0), (32, 1.02), (48, 0.97), (64, 1.0), (64, 1.013), (128, 0.99)])
def test_device_template_spectrum_matches_host(T, factor):
    vol = synthetic.template_volume(T, 1.5, n_atoms=400, radius_A=T * 1.5 * 0.3, seed=T).astype(np.float32)
    got = core.template_spectrum_device(vol, factor)
    ref = H.template_spectrum(vol, factor)
    assert np.abs(got - ref).max() <= 2e-5 * np.abs(ref).max()


def test_search_from_device_template_matches_host_template():
    T, X, Y = 32, 256, 256
    vol = synthetic.template_volume(T, 2.0, n_atoms=600, radius_A=20.0, seed=5).astype(np.float32)
    img, _ = synthetic.micrograph(Y, X, 2.0, 600, 20.0, 3, 1.0, 8000.0, seed=6, atom_seed=5)
    spec, curve = H.whiten(img.astype(np.float32))
    filt = prep.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=8000.0,
                                  defocus2=8000.0, pixel_size=2.0)
    angles = core.orientation_list(prep.search_grid(30.0), 0.0, 30.0, 360.0)[:64]
    out = []
    for device in (False, True):
        sc = core.SearchCore(X, Y, T, histogram_min_scaled=-12.5 / 256.0, histogram_step_scaled=35.0 / 512 / 256.0)
        if device:
            sc.set_template_volume(vol, 1.02)
        else:
            sc.set_template(H.template_spectrum(vol, 1.02))
        sc.set_image(spec)
        sc.run_plane(filt, angles)
        out.append(sc.results())
        sc.close()
    a, b = out
    assert np.abs(a["mip"] - b["mip"]).max() <= 1e-4 * np.abs(a["mip"]).max()
    assert ((a["psi"] == b["psi"]) & (a["theta"] == b["theta"]) & (a["phi"] == b["phi"])).mean() > 0.99
