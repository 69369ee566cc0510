"""Parity of the search core on micrograph heights with factors of 3 and on
templates whose box is not a power of two (needs a B200).

The micrograph factorisation of the reference (match_template.cpp:527-596)
pads 3710-pixel sides to 3888 = 2^4 3^5 and 5760-pixel sides to 5832 = 2^3 3^6
(the latter then becomes the height through the 90-degree rotation), and
templates such as 384^3 = 2^7 3 boxes occur.  The small geometries exercise the
same kernel paths as the full-size ones: 288 = 2^5 3^2 heights (radix-18 column
transforms with a pruned forward of length 36), 48-pixel templates (radix-24
slice transforms, zero-padded pruned row and column transforms of length 64).
Tolerances as in test_gpu_parity.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.search_cases import make_case
from tests.test_gpu_parity import _compare_search, _core

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("geom", [(32, 256, 288), (48, 256, 256), (48, 256, 288)])
def test_small_geometry_correlation_maps(geom):
    T, X, Y = geom
    case = make_case(T=T, X=X, Y=Y, n_orient=40)
    with _core(case) as sc:
        for o in (0, 11, 39):
            sc.reset()
            sc.run_plane(case["filt"], case["angles"][o:o + 1])
            got = sc.results()["mip"].reshape(Y, X)
            ref = O.correlate_one(case["tspec"], case["ispec"], case["filt"], case["angles"], o, X, Y)
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < 2e-5, (geom, o, err)


@pytest.mark.parametrize("geom", [(32, 256, 288), (48, 256, 288)])
def test_small_geometry_search_parity(geom):
    T, X, Y = geom
    case = make_case(T=T, X=X, Y=Y, angular_step=30.0, psi_step=30.0)
    _compare_search(case, batch=16, planes=((0.0, 0.0), (200.0, 0.0)))


@pytest.mark.parametrize("geom", [(256, 4096, 3888), (256, 4096, 5832), (384, 4096, 5832), (384, 4096, 4096),
                                  (256, 4096, 4096), (64, 4096, 4096), (256, 2048, 2916), (128, 2048, 2916),
                                  (256, 2048, 1944), (256, 2048, 2592), (256, 4096, 5184)])
def test_full_size_geometry_correlation_maps(geom):
    T, X, Y = geom
    case = make_case(T=T, X=X, Y=Y, pixel_size=1.0, n_particles=4, n_orient=40)
    with _core(case) as sc:
        for o in (5, 30):
            sc.reset()
            sc.run_plane(case["filt"], case["angles"][o:o + 1])
            got = sc.results()["mip"].reshape(Y, X)
            ref = O.correlate_one(case["tspec"], case["ispec"], case["filt"], case["angles"], o, X, Y)
            err = np.abs(got - ref).max() / np.abs(ref).max()
            assert err < 2e-5, (geom, o, err)


@pytest.mark.parametrize("geom", [(128, 2048, 2048), (128, 2048, 2916)])
def test_2048_wide_search_parity(geom):
    """Whole-search parity (MIP, angles, sums, histogram) on 2048-wide micrographs, whose
    row pass keeps its twiddles and compensated sums in tensor memory as at 4096,
    over more orientations than one launch holds (ragged last batch)."""
    T, X, Y = geom
    case = make_case(T=T, X=X, Y=Y, angular_step=30.0, psi_step=30.0, n_orient=40)
    _compare_search(case, batch=16)
