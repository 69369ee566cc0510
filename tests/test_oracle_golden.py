"""Pins the CPU oracle against the reference's own known answers.

Every expected number below is quoted from the reference's unit-test program
src/programs/console_test/console_test.cpp (line numbers given per test) and is
evaluated on the MRC fixtures that program embeds (extracted byte-for-byte by
tests/golden/make_console_fixtures.py).  The reference compares with
|a-b| < 1e-6 on FP32 results (core/functions.h:506-509); the oracle computes
in FP64, so the tolerance here is 2e-6.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O

TOL = 2e-6


def _mrc(golden_dir, name):
    return O.read_mrc(os.path.join(golden_dir, name)).astype(np.float64)


def fwd(img):
    """Image::ForwardFFT (scaled by 1/N)."""
    return O.rfft2(img) / img.size


def bwd(spec, nx):
    """Image::BackwardFFT (unscaled)."""
    return O.irfft2(spec, nx)


def test_mrc_read(golden_dir):
    # console_test.cpp:932-964
    stack = _mrc(golden_dir, "hiv_images_shift_noise_80x80x10.mrc")
    assert stack.shape == (10, 80, 80)
    assert abs(stack[0, 0, 0] - -0.340068) < TOL
    assert abs(stack[0, 79, 79] - 0.637069) < TOL


def test_add_image(golden_dir):
    # console_test.cpp:522-538
    stack = _mrc(golden_dir, "hiv_images_shift_noise_80x80x10.mrc")
    s = stack[0] + stack[1]
    for (x, y), v in [((0, 0), -1.313164), ((40, 40), 3.457573), ((79, 79), 0.318875)]:
        assert abs(s[y, x] - v) < TOL


def test_forward_fft_constant_and_sine(golden_dir):
    # console_test.cpp:967-1013
    ones = np.ones((64, 64))
    f = fwd(ones)
    assert abs(f[0, 0] - 1) < TOL
    f[0, 0] = 0
    assert np.abs(f).max() < TOL
    sine = _mrc(golden_dir, "sine_wave_128x128x1.mrc")[0]
    f = fwd(sine)
    assert abs(f[0, 20].real) < TOL and abs(f[0, 20].imag - -5.0) < TOL
    f[0, 20] = 0
    assert f.real.max() < 1e-6 and f.imag.max() < 1e-6


def test_backward_fft_dc(golden_dir):
    # console_test.cpp:1017-1032
    spec = np.zeros((64, 33), complex)
    spec[0, 0] = 1.0
    out = bwd(spec, 64)
    assert np.abs(out - 1.0).max() < TOL


def test_phase_shift(golden_dir):
    # console_test.cpp:645-655: PhaseShift(20, 20, 0) of slice 1
    img = _mrc(golden_dir, "hiv_images_shift_noise_80x80x10.mrc")[0]
    spec = O.phase_shift(fwd(img), 80, 20, 20, 0)
    out = bwd(spec, 80)
    for (x, y), v in [((0, 0), -1.010296), ((40, 40), -2.280109), ((79, 79), 0.239702)]:
        assert abs(out[y, x] - v) < TOL


def _cross_correlation(a, b):
    """Image::CalculateCrossCorrelationImageWith (image.cpp:9826-9866) for
    images read from file (object centred in the box)."""
    fa, fb = fwd(a), fwd(b)
    fa = fa * np.conj(fb)
    fa = O.swap_quadrants(fa, a.shape[1], centred=False)
    return bwd(fa, a.shape[1])


def test_cross_correlation(golden_dir):
    # console_test.cpp:657-668
    a = _mrc(golden_dir, "hiv_images_shift_noise_80x80x10.mrc")[0]
    b = _mrc(golden_dir, "hiv_image_80x80x1.mrc")[0]
    cc = _cross_correlation(a, b)
    for (x, y), v in [((0, 0), 0.004323), ((40, 40), 0.543692), ((79, 79), 0.006927)]:
        assert abs(cc[y, x] - v) < TOL


def test_find_peak_integer(golden_dir):
    # console_test.cpp:672-686: shift by (7, 10), correlate, integer peak
    ref = _mrc(golden_dir, "hiv_image_80x80x1.mrc")[0]
    shifted = bwd(O.phase_shift(fwd(ref), 80, 7, 10, 0), 80)
    cc = _cross_correlation(shifted, ref)
    x, y, v = O.find_peak_integer(cc)
    assert (x, y) == (7.0, 10.0)
    assert abs(v - 1.0) < TOL


@pytest.mark.parametrize("size,checks", [
    (160, [((40, 40), -0.340068), ((80, 80), 1.819805), ((119, 119), 0.637069)]),
    (50, [((0, 0), -2.287762), ((25, 25), 1.819805), ((49, 49), -1.773780)]),
    (49, [((0, 0), -0.391899), ((25, 25), 1.689942), ((48, 48), -1.773780)]),
])
def test_clip_into_real(golden_dir, size, checks):
    # console_test.cpp:785-816 and 839-848 (Resize shares the path, :873-893)
    img = _mrc(golden_dir, "hiv_images_shift_noise_80x80x10.mrc")[0]
    out = O.clip_into_real(img, size, size, 0.0)
    for (x, y), v in checks:
        assert abs(out[y, x] - v) < TOL


def _logical(spec, x, y, oob):
    ny, hc = spec.shape
    lby, uby = -(ny // 2), ny // 2 - 1
    if x < 0 or x > hc - 1 or y < lby or y > uby:
        return oob
    return spec[y if y >= 0 else ny + y, x]


@pytest.mark.parametrize("size", [160, 50, 49])
def test_clip_into_fourier(golden_dir, size):
    # console_test.cpp:818-837, 850-860; Resize: 895-922
    img = _mrc(golden_dir, "hiv_images_shift_noise_80x80x10.mrc")[0]
    out = O.clip_into_fourier(fwd(img), 80, size, size, 0.0)
    if size == 160:
        assert _logical(out, -90, -90, -100.0) == -100.0
    dc = _logical(out, 0, 0, -100.0)
    assert abs(dc.real - -0.010919) < TOL and abs(dc.imag) < TOL
    v = _logical(out, 5, 5, -100.0)
    assert abs(v.real - 0.075896) < TOL and abs(v.imag - 0.045677) < TOL


def test_fft_matches_numpy_mixed_radix():
    rng = np.random.default_rng(3)
    for nx, ny in [(54, 36), (60, 26), (128, 96)]:
        img = rng.standard_normal((ny, nx))
        assert np.abs(O.rfft2(img) - np.fft.rfft2(img)).max() < 1e-10
        spec = np.fft.rfft2(img)
        assert np.abs(O.irfft2(spec, nx) - np.fft.irfft2(spec, s=(ny, nx)) * nx * ny).max() < 1e-9


def test_search_grid_counts():
    # EulerSearch grids used by the search configurations (euler_search.cpp:180-260)
    for step, psi_step, n in [(15.0, 15.0, 4700), (2.5, 1.5, 1595420), (3.0, 2.0, 833686), (7.5, 5.0, 53874)]:
        assert len(O.search_grid(step)) * len(O.psi_list(0.0, psi_step, 360.0)) == n
    g = O.search_grid(15.0)
    assert tuple(g[0]) == (0.0, 0.0) and g[-1][1] == 180.0


def test_factorization_of_configured_sizes():
    # match_template.cpp:527-596; the reference accepts the first prime whose
    # upper factorised size grows the image by < 10%
    assert O.factorize_dimension(1024, 64) == 1024
    assert O.factorize_dimension(4096, 256) == 4096
    assert O.factorize_dimension(2048, 256) == 2048
    assert O.factorize_dimension(5760, 384) == 5832
    assert O.factorize_dimension(4092, 384) == 4096
    assert O.factorize_dimension(3838, 256) == 4096
    assert O.factorize_dimension(3710, 256) == 3888
    assert not O.is_power_of_two(5832) and O.is_power_of_two(4096)


def test_erfcinv_closed_form():
    from scipy.special import erfcinv
    for x in [1e-3, 1e-9, 2.0 / (1024 * 1024 * 4700)]:
        assert abs(O.erfcinv(x) - erfcinv(x)) / erfcinv(x) < 5e-3


def test_euler_matrix_orthonormal():
    m = O.euler_matrix(30.0, 60.0, 90.0).astype(np.float64)
    assert np.abs(m @ m.T - np.eye(3)).max() < 1e-6
