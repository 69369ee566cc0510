"""The C++ host preparation (libtm_host.so, linked into the match_template
program) against the oracle's restatement of the reference preparation, and
the program's argument handling (CPU only)."""
import os
import subprocess

import numpy as np
import pytest

from cistem_downstream_bah_b200 import hostprep as H
from cistem_downstream_bah_b200 import synthetic
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_library_exports_every_binding():
    L = H.lib()
    for name in H.EXPORTED:
        assert hasattr(L, name), name


@pytest.mark.parametrize("shape", [(128, 128), (96, 160), (80, 72)])
def test_whitening_matches_oracle(shape):
    ny, nx = shape
    img, _ = synthetic.micrograph(ny, nx, 2.0, 300, 20.0, 2, 0.5, 8000.0, seed=5)
    img = img.astype(np.float32)
    s_ref, c_ref = O.whiten_image(img.astype(np.float64))
    s, c = H.whiten(img)
    assert c.shape == c_ref.shape
    assert np.abs(c - c_ref).max() / np.abs(c_ref).max() < 1e-9
    assert np.abs(s - s_ref).max() / np.abs(s_ref).max() < 1e-6


def test_whitening_replaces_outliers():
    rng = np.random.default_rng(0)
    img = rng.normal(size=(64, 64)).astype(np.float32)
    img[10, 10] = 1e4
    s_ref, _ = O.whiten_image(img.astype(np.float64))
    s, _ = H.whiten(img)
    assert np.abs(s - s_ref).max() / np.abs(s_ref).max() < 1e-6


@pytest.mark.parametrize("T", [16, 32])
def test_template_spectrum_matches_oracle(T):
    vol = synthetic.template_volume(T, 2.0, 300, T * 0.6, seed=T).astype(np.float32)
    ref = O.prepare_template(vol.astype(np.float64))
    got = H.template_spectrum(vol, 1.0)
    assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-6


def _profile_sigma(vol):
    """Width of a centred Gaussian blob from its central line, A exp(-d^2/2s^2) + B."""
    from scipy.optimize import curve_fit
    T = vol.shape[0]
    d = np.arange(T) - T // 2
    line = vol[T // 2, T // 2, :]
    (a, s, b), _ = curve_fit(lambda d, a, s, b: a * np.exp(-d * d / (2 * s * s)) + b, d, line, p0=(1.0, 3.0, 0.0))
    return abs(s)


@pytest.mark.parametrize("factor", [1.0, 1.04, 0.96])
def test_template_pixel_size_change_rescales(factor):
    """ChangePixelSize (image.cpp:8705-8822): a Gaussian of sigma s voxels
    becomes sigma s/factor on the new pixel grid, with the same box."""
    T = 32
    c = np.arange(T) - T // 2
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    s = 3.0
    vol = np.exp(-(x * x + y * y + z * z) / (2 * s * s)).astype(np.float32)
    spec = H.template_spectrum(vol, factor)
    # undo the quadrant swap (object centred: a phase (-1)^(kx+ky+kz) for even T) and transform back
    k = np.fft.fftfreq(T) * T
    kx = np.arange(T // 2 + 1)
    sign = (-1.0) ** (k[:, None, None] + k[None, :, None] + kx[None, None, :])
    real = np.fft.irfftn(spec * sign, s=(T, T, T), axes=(0, 1, 2)) * T ** 3
    assert np.unravel_index(real.argmax(), real.shape) == (T // 2, T // 2, T // 2)
    # the padding value and the zeroed central pixel add a constant around the blob
    got = _profile_sigma(real)
    assert abs(got - s / factor) < 0.01 * s


def test_projection_filter_matches_oracle():
    img, _ = synthetic.micrograph(128, 128, 2.0, 300, 20.0, 2, 0.5, 8000.0, seed=3)
    _, curve = O.whiten_image(img.astype(np.float64))
    for kw in (dict(kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=9000.0, defocus2=8500.0,
                    astigmatism_angle=30.0, pixel_size=1.5, defocus_offset=200.0),
               dict(kv=200.0, cs_mm=0.01, amplitude_contrast=0.1, defocus1=0.0, defocus2=0.0,
                    pixel_size=1.0, phase_shift_deg=90.0),
               dict(kv=300.0, cs_mm=2.7, amplitude_contrast=1.0, defocus1=12000.0, defocus2=12000.0,
                    pixel_size=1.0, defocus_offset=-1200.0)):
        ref = O.projection_filter(32, curve, **kw)
        got = H.projection_filter(32, curve, **kw)
        assert np.abs(got - ref).max() < 1e-6, kw


def test_search_grid_psi_and_factorisation_match_oracle():
    for step in (15.0, 7.5, 3.0, 2.5):
        assert np.array_equal(H.search_grid(step), O.search_grid(step))
    for sym in ("C2", "C7", "D3", "O", "I", "T"):
        assert np.array_equal(H.search_grid(5.0, sym), O.search_grid(5.0, sym))
    with pytest.raises(ValueError):
        H.search_grid(5.0, "X9")
    for a in ((0.0, 15.0, 360.0), (0.0, 1.5, 360.0), (0.0, 2.0, 360.0), (0.0, 0.7, 360.0)):
        assert np.array_equal(H.psi_list(*a), O.psi_list(*a))
    for n in (1024, 2048, 4096, 3838, 3710, 5760, 4092, 1000, 777, 4100):
        assert H.factorize_dimension(n, 256) == O.factorize_dimension(n, 256), n
    assert H.factorize_dimension(5760, 256) == 5832
    assert H.factorize_dimension(3838, 256) == 4096
    assert H.factorize_dimension(3710, 256) == 3888   # 2^4 3^5
    for n in (1, 2, 3, 4, 96, 128, 5832):
        assert bool(H.lib().tmh_is_power_of_two(n)) == bool(O.is_power_of_two(n))
    assert H.lib().tmh_angular_step(8.0, 200.0) == np.float32(O.angular_step(8.0, 200.0))
    for x in (1e-3, 1e-9, 2.0 / (4096.0 * 4096.0 * 1.6e6)):
        assert H.lib().tmh_erfcinv(x) == O.erfcinv(x)


def test_real_space_helpers_match_oracle():
    rng = np.random.default_rng(1)
    img = rng.normal(size=(37, 50)).astype(np.float32)
    assert np.isclose(H.edge_mean(img), np.float32(np.concatenate(
        [img[0], img[1:-1, 0], img[1:-1, -1], img[-1]]).astype(np.float64).mean()), rtol=1e-6)
    for ox, oy in ((64, 48), (30, 20), (50, 37)):
        got = H.clip_into(img, ox, oy, 0.25)
        ref = O.clip_into_real(img.astype(np.float64), ox, oy, 0.25)
        assert np.array_equal(got, ref.astype(np.float32))
    for pos in (True, False):
        assert np.array_equal(H.rotate90(img, pos), O.rotate90(img.astype(np.float64), pos).astype(np.float32))
    assert np.array_equal(H.rotate90(H.rotate90(img, True), False), img)


def test_mrc_reader_matches_golden_fixtures(tmp_path):
    for name in ("hiv_image_80x80x1.mrc", "hiv_images_shift_noise_80x80x10.mrc", "sine_wave_128x128x1.mrc"):
        got, _ = H.read_mrc(os.path.join(GOLDEN, name))
        ref = O.read_mrc(os.path.join(GOLDEN, name))
        assert np.array_equal(got, ref), name


def test_mrc_write_read_round_trip(tmp_path):
    rng = np.random.default_rng(2)
    vol = rng.normal(size=(3, 20, 30)).astype(np.float32)
    p = tmp_path / "v.mrc"
    H.write_mrc(p, vol, pixel_size=1.25)
    got, px = H.read_mrc(p)
    assert np.array_equal(got, vol)
    assert abs(px - 1.25) < 1e-6
    assert np.array_equal(O.read_mrc(str(p)), vol)
    with open(p, "rb") as f:
        hdr = f.read(1024)
    assert hdr[208:212] == b"MAP "
    assert os.path.getsize(p) == 1024 + vol.nbytes


def test_cli_usage_and_scripted_prompts(tmp_path):
    """The program's argument forms.  Without a GPU the search itself stops at
    the device set-up with an error status, after the prompts and the
    micrograph preparation have run."""
    cli = H.CLI_PATH
    assert os.path.exists(cli)
    r = subprocess.run([cli, "a", "b"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "usage" in r.stderr
    img, _ = synthetic.micrograph(250, 256, 2.0, 300, 20.0, 2, 0.5, 8000.0, seed=3)
    vol = synthetic.template_volume(32, 2.0, 300, 20.0, seed=2)
    H.write_mrc(tmp_path / "img.mrc", img, 2.0)
    H.write_mrc(tmp_path / "tpl.mrc", vol, 2.0)
    answers = [str(tmp_path / "img.mrc"), str(tmp_path / "tpl.mrc")] + \
        [str(tmp_path / f"out{k}.mrc") for k in range(9)] + [str(tmp_path / "hist.txt")] + \
        ["2.0", "300", "2.7", "0.07", "8000", "8000", "0", "0", "8", "15", "15", "0", "0", "0", "0",
         "1.0", "0", "C1", "yes", "1"]
    r = subprocess.run([cli], input="\n".join(answers) + "\n", capture_output=True, text=True, timeout=120)
    out = r.stdout
    assert "Input images to be searched" in out and "Template symmetry" in out
    assert "old x, y; new x, y = 256 250 256 256" in out
    if r.returncode != 0:
        assert "Error" in r.stderr   # no GPU here: tm_create reports it


def test_cli_rejects_blank_scripted_answer(tmp_path):
    r = subprocess.run([H.CLI_PATH], input="\n", capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    assert "Blank answer in scripted mode" in r.stdout


from tests.peak_loop import reference_peaks as _reference_peaks  # noqa: E402


def test_peak_list_matches_the_reference_loop():
    rng = np.random.default_rng(7)
    ny, nx, T = 120, 150, 32
    z = rng.normal(size=(ny, nx)).astype(np.float32)
    for (y, x, h) in ((30, 40, 12.0), (31, 44, 11.0), (90, 100, 9.0), (60, 10, 15.0), (5, 75, 20.0)):
        z[y, x] = h
    maps = [rng.uniform(0, 360, size=(ny, nx)).astype(np.float32) for _ in range(3)] + \
        [rng.choice([-200.0, 0.0, 200.0], size=(ny, nx)).astype(np.float32), np.zeros((ny, nx), np.float32)]
    ref = _reference_peaks(z, maps, 8.0, 10, T, 1.5)
    got = H.find_peaks(z, *maps, threshold=8.0, min_peak_radius=10, template_size=T, pixel_size=1.5)
    # (5, 75) lies within T/4+1 of an edge; (31, 44) is blanked by (30, 40)
    assert [tuple(int(v) for v in p) for p in got[:, 8:]] == [(10, 60), (40, 30), (100, 90)]
    assert np.array_equal(got[:, :8], ref)


def test_projection_montage_is_the_projection_at_zero_angles():
    """At (psi, theta, phi) = 0 the Fourier slice samples the grid exactly, so
    the montage tile is the z-projection of the normalised template,
    scaled by sqrt(T*T*sqrt(T)) * T * T^2 / T^3 = T^1.25, less its edge mean,
    kept where positive."""
    T = 32
    c = np.arange(T) - T // 2
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    vol = (np.exp(-((x - 2) ** 2 + y ** 2 + (z + 1) ** 2) / 18.0) +
           0.5 * np.exp(-((x + 5) ** 2 + (y - 4) ** 2 + z ** 2) / 8.0)).astype(np.float32)
    planes = np.concatenate([vol[T // 2].ravel(), vol[:, T // 2].ravel(), vol[:, :, T // 2].ravel()])
    # voxels on the central planes, each once: the union of the three planes
    mask = np.zeros(vol.shape, bool)
    mask[T // 2] = mask[:, T // 2] = mask[:, :, T // 2] = True
    m = np.sort(vol[mask])[-100:].astype(np.float64).mean()
    proj = (vol / np.float32(m)).astype(np.float64).sum(axis=0)
    # the DC term is zeroed: subtract the volume mean along the projection
    proj = proj - proj.mean()
    proj = proj * T ** 1.25
    edge = np.concatenate([proj[0], proj[1:-1, 0], proj[1:-1, -1], proj[-1]]).mean()
    expect = np.clip(proj - edge, 0, None)
    nx, ny = 100, 90
    got = H.projection_montage(vol, [[50, 40, 0.0, 0.0, 0.0]], nx, ny)
    tile = got[40 - T // 2:40 + T // 2, 50 - T // 2:50 + T // 2]
    assert np.abs(tile - expect).max() < 1e-3 * expect.max()
    assert np.count_nonzero(got) == np.count_nonzero(tile)
    assert planes.size == 3 * T * T
