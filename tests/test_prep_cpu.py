"""The numpy host preparation agrees with the oracle's restatement of the
reference preparation (CPU only)."""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import prep, synthetic
from oracle import oracle as O


@pytest.mark.parametrize("shape", [(128, 128), (96, 160)])
def test_whitening_matches_oracle(shape):
    ny, nx = shape
    img, _ = synthetic.micrograph(ny, nx, 2.0, 300, 20.0, 2, 0.5, 8000.0, seed=3)
    s_ref, c_ref = O.whiten_image(img.astype(np.float64))
    s, c = prep.whiten(img)
    assert np.abs(c - c_ref).max() / np.abs(c_ref).max() < 1e-5
    assert np.abs(s - s_ref).max() / np.abs(s_ref).max() < 2e-5


def test_template_spectrum_matches_oracle():
    vol = synthetic.template_volume(32, 2.0, 400, 20.0, seed=2)
    ref = O.prepare_template(vol.astype(np.float64))
    got = prep.template_spectrum(vol)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-5


def test_projection_filter_matches_oracle():
    img, _ = synthetic.micrograph(128, 128, 2.0, 300, 20.0, 2, 0.5, 8000.0, seed=3)
    _, curve = O.whiten_image(img.astype(np.float64))
    kw = dict(kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=9000.0, defocus2=8500.0,
              astigmatism_angle=30.0, pixel_size=1.5, defocus_offset=200.0)
    ref = O.projection_filter(32, curve, **kw)
    got = prep.projection_filter(32, curve, **kw)
    assert np.abs(got - ref).max() < 1e-5


def test_search_grid_and_factorisation_match_oracle():
    for step in (15.0, 7.5, 3.0, 2.5):
        assert np.array_equal(prep.search_grid(step), O.search_grid(step))
    for sym in ("C2", "D3", "O", "I", "T"):
        assert np.array_equal(prep.search_grid(10.0, sym), O.search_grid(10.0, sym))
    for n in (1024, 3838, 3710, 5760, 4092, 4096, 2048, 1000, 777):
        assert prep.factorize_dimension(n, 256) == O.factorize_dimension(n, 256)


def test_finalize_matches_oracle():
    rng = np.random.default_rng(1)
    n = 1000
    st = O.SearchState(40, 25)
    st.mip[:] = rng.random(n).astype(np.float32)
    st.sum[:] = rng.standard_normal(n) * 3
    st.sumsq[:] = rng.random(n) * 50 + st.sum ** 2 / 40
    m_ref, z_ref, a_ref, s_ref = O.finalize(st, 40, np.sqrt(1000.0))
    m, z, a, s = prep.finalize(st.mip, st.sum, st.sumsq, 40, 40, 25)
    assert np.allclose(m, m_ref, rtol=1e-6) and np.allclose(a, a_ref, rtol=1e-6)
    assert np.allclose(s, s_ref, rtol=1e-5) and np.allclose(z, z_ref, rtol=1e-4, atol=1e-5)
