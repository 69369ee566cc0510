"""Learned proposal on the CPU: the FP64 network oracle pinned by central
differences, BF16 rounding, and the host logic (angular bins, tile features
and labels, window spectra) that needs no GPU."""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import proposal as PR
from oracle import proposal as OP


def _params(cin, seed):
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in OP.layout(cin):
        n = int(np.prod(shape))
        scale = np.sqrt(2.0 / np.prod(shape[1:])) if name.startswith("w") else 0.1
        parts.append(rng.standard_normal(n) * scale)
    return np.concatenate(parts)


def test_layout_matches_host():
    assert [(n, tuple(s)) for n, s in OP.layout(7)] == [(n, tuple(s)) for n, s in PR.param_layout(7)]
    assert OP.param_count(7) == len(PR.init_params(7))
    assert OP.param_count(7) == 242500


@pytest.mark.parametrize("pos_weight,dir_weight", [(1.0, 1.0), (3.0, 0.25)])
def test_oracle_gradients_central_differences(pos_weight, dir_weight):
    cin = 3
    p = _params(cin, 1)
    rng = np.random.default_rng(2)
    x = rng.standard_normal((3, cin, 16, 16))
    lab = np.array([[1, 0.6, 0.8, 0.0], [0, 0, 0, 0], [1, 0.0, 0.0, 1.0]])
    loss, g = OP.gradients(p, x, lab, cin, pos_weight, dir_weight, bf16=False)
    assert np.isclose(loss, OP.loss_only(p, x, lab, cin, pos_weight, dir_weight))
    idx = np.concatenate([rng.choice(len(p), 30, replace=False), np.arange(len(p) - 516, len(p))[::37]])
    h = 1e-6
    for i in idx:
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (OP.loss_only(pp, x, lab, cin, pos_weight, dir_weight) -
              OP.loss_only(pm, x, lab, cin, pos_weight, dir_weight)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, g[i])


def test_bf16_rounding():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, 1.0 + 2 ** -9, -2.5, 3.0e-3], np.float32)
    r = OP.bf16_round(v)
    assert r[0] == 1.0
    assert r[1] == 1.0 + 2 ** -7 or r[1] == 1.0    # representable neighbours
    assert r[3] == 1.0                              # tie to even
    assert r[2] == 1.0 + 2 ** -7                    # above the tie rounds up
    assert r[4] == -2.5
    assert abs(r[5] - 3.0e-3) <= 3.0e-3 * 2 ** -8


def test_angular_bins_partition_fine_grid():
    ab = PR.AngularBins(15.0, 7.5, 10.0)
    fd = PR.directions(ab.fine_grid[:, 0], ab.fine_grid[:, 1])
    # every fine position's bin is a nearest coarse centre
    s = fd @ ab.centers.T
    assert np.all(s[np.arange(len(fd)), ab.bin_of_position] >= s.max(axis=1) - 1e-12)
    rows = ab.orientations(range(ab.n_bins))
    assert np.array_equal(rows, np.arange(len(ab.fine_angles)))
    b = ab.nearest(ab.centers[5], 4)
    assert b[0] == 5 and len(set(b)) == 4
    rows = ab.orientations([b[1], b[0]])
    assert np.all(np.diff(rows) > 0)
    pos = np.unique(rows // ab.n_psi)
    assert set(ab.bin_of_position[pos]) <= {b[0], b[1]}


def test_tile_features_and_labels():
    rng = np.random.default_rng(3)
    z = rng.standard_normal((128, 192)).astype(np.float32)
    th = rng.uniform(0, 180, z.shape).astype(np.float32)
    ph = rng.uniform(0, 360, z.shape).astype(np.float32)
    z[70, 100] = 9.0
    f = PR.tile_features(z, th, ph)
    assert f.shape == (6, PR.FEATURES, 64, 64)
    t = 1 * 3 + 1   # tile row 1, column 1
    assert np.isclose(f[t, 0, 70 - 64, 100 - 64], 9.0 / 4.0)
    d = PR.directions(ph[70, 100], th[70, 100])
    # directions in the tile's frame: the coarse best direction at the maximum reads +z
    frames = PR.tile_frames(z, th, ph)
    assert np.allclose(frames[t] @ d, [0.0, 0.0, 1.0], atol=1e-12)
    assert np.allclose(f[t, 4:7, 6, 36], [0.0, 0.0, 1.0], atol=1e-6)
    assert np.allclose(f[t, 1:4, 6, 36], [0.0, 0.0, 2.0], atol=1e-6)
    d2 = PR.directions(ph[70, 101], th[70, 101])
    assert np.allclose(f[t, 4:7, 6, 37], frames[t] @ d2, atol=1e-6)
    peaks = np.array([[100, 70, 9.0, 30.0, 40.0, 0.0], [101, 71, 8.0, 0.0, 0.0, 0.0], [10, 10, 7.5, 0.0, 90.0, 0.0]])
    lab = PR.tile_labels(peaks, 192, 128)
    assert lab[:, 0].tolist() == [1, 0, 0, 0, 1, 0]
    assert np.allclose(lab[4, 1:], PR.directions(30.0, 40.0))
    loc = PR.to_frames(lab, frames)
    assert np.allclose(loc[:, 0], lab[:, 0])
    out = np.concatenate([np.zeros((6, 1)), loc[:, 1:4] * 3.0], axis=1)
    assert np.allclose(PR.network_directions(out, frames)[4], 3.0 * lab[4, 1:], atol=1e-9)
    for k in range(8):
        a = PR.dihedral(f, k)
        assert a.shape == f.shape
        assert np.isclose(a[:, 0].max(), f[:, 0].max())


def test_window_spectrum_reproduces_correlations():
    """With the search context's conventions (image spectrum divided by its own
    pixel count, DC term dropped), the window's spectrum gives the full
    image's correlation with a T-support kernel at the window's interior
    positions (shifted by the window origin), also for windows that wrap
    around the image edge."""
    rng = np.random.default_rng(4)
    X = Y = 96
    T, W = 16, 48
    lo, hi = 4, 44
    img = rng.standard_normal((Y, X))
    spec = np.fft.rfft2(img) / (X * Y)
    spec[0, 0] = 0
    ky = np.arange(Y)[:, None]
    kx = np.arange(X // 2 + 1)[None, :]
    spec = spec * np.where(((ky + kx) & 1) == 1, -1.0, 1.0)
    s = PR.whitened_real(spec.astype(np.complex64), X, Y)
    assert np.allclose(s, img - img.mean(), atol=1e-4)
    ker = rng.standard_normal((T, T))

    def context_corr(spec_swapped, n, n_pixels):
        kyy = np.arange(n)[:, None]
        kxx = np.arange(n // 2 + 1)[None, :]
        ip = spec_swapped * np.where(((kyy + kxx) & 1) == 1, -1.0, 1.0) / n_pixels
        ip[0, 0] = 0
        kp = np.zeros((n, n))
        kp[:T, :T] = ker
        return np.fft.irfft2(ip * np.conj(np.fft.rfft2(kp)), s=(n, n)) * n * n

    full = context_corr(spec, X, X * Y)
    for x0, y0 in [(10, 20), (-8, -8), (70, 80)]:
        ws = PR.window_spectrum(s, x0, y0, W, X * Y, (lo, hi))
        cw = context_corr(ws, W, W * W)
        for r in [(lo, lo), (lo + 5, lo + 7), (hi - T, hi - T), (lo, hi - T)]:
            ref = full[(y0 + r[0]) % Y, (x0 + r[1]) % X]
            assert np.isclose(cw[r], ref, rtol=1e-5, atol=1e-9), (x0, y0, r, cw[r], ref)
    # a window over the whole image with nothing outside its used square is refused
    with pytest.raises(AssertionError):
        PR.window_spectrum(s, 0, 0, X, X * Y, (0, X))


def test_window_geometry():
    for T in (64, 128, 256):
        W, C = PR.window_size(T), PR.window_core(T)
        assert C % PR.TILE == 0 and C >= PR.TILE
        m = (W - C - T) // 2
        assert m >= 8 and 2 * m + C + T == W


def test_tiles_for_recall():
    # peaks in tiles 3, 7, 7, 1; the second one cannot be recovered by its bins
    ranking = np.array([7, 3, 0, 1, 2, 4, 5, 6])
    need = PR.tiles_for_recall([3, 7, 7, 1], np.array([True, False, True, True]), ranking, levels=(0.5, 0.75, 1.0))
    assert need == {"0.5": 2, "0.75": 4, "1.0": None}
    assert PR.tiles_for_recall([], np.zeros(0, bool), ranking) == {"0.9": 0, "0.95": 0, "0.99": 0, "1.0": 0}


def test_window_variants_are_compiled():
    """Every template box the proposal trains and evaluates on (64, 128, 256) has a
    search kernel for its window geometry and for the 1024^2 training micrographs."""
    import os
    import re
    src = open(os.path.join(os.path.dirname(PR.__file__), "csrc", "tm_capi.cu")).read()
    variants = {tuple(int(v) for v in m) for m in re.findall(r"TM_VARIANT(?:_TC)?\((\d+),\s*(\d+),\s*(\d+)\)", src)}
    for T in (64, 128, 256):
        W = PR.window_size(T)
        assert (T, W, W) in variants, (T, W)
    for T in (64, 128):
        assert (T, 1024, 1024) in variants
    assert (256, 4096, 4096) in variants


def test_threshold_and_bins_helpers():
    from cistem_downstream_bah_b200 import proposal_train as PT
    scores = np.array([5.0, -1.0, 3.0, 0.5, 2.0])
    lab = np.zeros((5, 4))
    lab[[0, 2, 4], 0] = 1.0
    assert PT.threshold_for(scores, lab, margin=0.5) == 2.0 - 0.5           # keeps every positive
    assert PT.threshold_for(scores, lab, margin=0.0, keep=0.5) == 3.0       # keeps the upper half
    assert PT.threshold_for(scores, np.zeros((5, 4)), margin=0.0) == float("inf")
    ab = PR.AngularBins(15.0, 7.5, 10.0)
    d = ab.centers[7]
    assert PT.bins_hit(ab, ab.nearest(d, 1), d)
    far = -d
    assert not PT.bins_hit(ab, ab.nearest(d, 4), far)


def test_case_parameters_follow_the_training_distribution():
    from cistem_downstream_bah_b200 import proposal_train as PT
    for seed in range(1000, 1100, 7):
        c = PT.case_params(seed)
        assert c["T"] in (64, 128)
        assert 0.02 <= c["snr"] <= 0.08 and 5000.0 <= c["defocus"] <= 25000.0
        assert c["radius_A"] <= 0.45 * c["T"] * c["pixel_size"]
        assert c == PT.case_params(seed)    # seeded


class _RecordingContext:
    """Stands in for the window-geometry search context: records the calls and
    returns, per window, a MIP that encodes (window, pixel) and angles that
    encode the number of bins the window was searched with."""

    def __init__(self, W):
        self.W = W
        self.calls = []

    def set_template(self, tspec):
        pass

    def set_normalization_pixels(self, n):
        self.norm = n

    def set_image_set(self, spectra):
        self.n = len(spectra)
        self.runs = [0] * self.n
        self.orient = [0] * self.n

    def run_plane_images(self, filt, angles, images):
        self.calls.append((len(angles), list(images)))
        for k in images:
            self.runs[k] += 1
            self.orient[k] += len(angles)

    def image_results(self, k):
        W = self.W
        mip = (1000.0 * k + np.arange(W * W)).astype(np.float32)
        return {"mip": mip, "psi": np.full(W * W, self.runs[k], np.float32),
                "theta": np.full(W * W, self.orient[k], np.float32), "phi": np.zeros(W * W, np.float32)}


def test_window_search_host_logic():
    X = Y = 1024
    T = 64
    spec = np.zeros((Y, X // 2 + 1), np.complex64)
    ab = PR.AngularBins(15.0, 7.5, 30.0)
    ctx = _RecordingContext(PR.window_size(T))
    ws = PR.WindowSearch(spec, X, Y, T, None, np.zeros((T, T // 2 + 1), np.float32), ab, 0.0, 1.0, context=ctx)
    assert ctx.norm == X * Y
    gx = X // PR.TILE
    C = PR.window_core(T)
    tiles = [0, 1, 5, gx + 1, gx * gx - 1]
    bins = [[0, 1], [1, 2], [3], [2], [4, 0]]
    res = ws.run(PR.Proposal(tiles, bins, None))
    # tiles 0, 1 and gx+1 share the first window (core C = 128 px = 2 tiles)
    assert res["windows"] == 3
    per_bin = {b: len(ab.orientations([b])) for b in range(5)}
    # windows in (core row, core column) order: 0 = tiles 0, 1, gx+1; 1 = tile 5; 2 = the last tile;
    # one call per bin, over the windows that need it, bins in increasing order
    assert ctx.calls == [(per_bin[0], [0, 2]), (per_bin[1], [0]), (per_bin[2], [0]), (per_bin[3], [1]),
                         (per_bin[4], [2])]
    # each window's orientations: the union of its tiles' bins, each bin once
    want = [sum(per_bin[b] for b in {0, 1, 2}), sum(per_bin[b] for b in {3}), sum(per_bin[b] for b in {0, 4})]
    assert ctx.orient == want
    assert res["points"] == float(sum(want)) * ctx.W * ctx.W
    # placement: tile (ty, tx) of window k holds that window's pixels at (y - y0, x - x0)
    m = PR.window_size(T) - C - T
    for t, k in zip(tiles, [0, 0, 1, 0, 2]):
        ty, tx = divmod(t, gx)
        cy, cx = ty // (C // PR.TILE), tx // (C // PR.TILE)
        x0, y0 = cx * C - T // 2 - m // 2, cy * C - T // 2 - m // 2
        y, x = ty * PR.TILE + 5, tx * PR.TILE + 7
        assert res["mip"][y, x] == 1000.0 * k + (y - y0) * ctx.W + (x - x0)
        assert res["theta"][y, x] == want[k]
    untouched = np.ones((Y, X), bool)
    for t in tiles:
        ty, tx = divmod(t, gx)
        untouched[ty * 64:ty * 64 + 64, tx * 64:tx * 64 + 64] = False
    assert np.all(np.isneginf(res["mip"][untouched]))


def test_partial_tiles_are_covered():
    """Micrographs whose sides are not multiples of the tile (4096 x 3888, 5832 x 4096
    in the uneven configurations) keep their last, partial tile row and column."""
    rng = np.random.default_rng(6)
    ny, nx = 100, 150
    z = rng.standard_normal((ny, nx)).astype(np.float32)
    th = rng.uniform(0, 180, z.shape).astype(np.float32)
    ph = rng.uniform(0, 360, z.shape).astype(np.float32)
    z[90, 140] = 11.0                                   # in the partial tile (1, 2)
    assert PR.tile_grid(nx, ny) == (2, 3)
    f = PR.tile_features(z, th, ph)
    assert f.shape == (6, PR.FEATURES, 64, 64)
    zmax, arg = PR.tile_max(z)
    assert zmax[5] == 11.0 and divmod(int(arg[5]), 64) == (90 - 64, 140 - 128)
    assert zmax[3] == z[64:, :64].max()
    assert np.isclose(f[5, 0, 26, 12], 11.0 / 4.0)
    assert np.all(f[5, 0, 36:, :] == -1.0) and np.all(f[5, 1:4, 36:, :] == 0.0)   # padding
    lab = PR.tile_labels(np.array([[140, 90, 11.0, 20.0, 30.0, 0.0]]), nx, ny)
    assert lab[5, 0] == 1.0
    frames = PR.tile_frames(z, th, ph)
    assert np.allclose(frames[5] @ PR.directions(ph[90, 140], th[90, 140]), [0, 0, 1], atol=1e-12)


def test_window_search_partial_tiles():
    X, Y = 1000, 900
    T = 64
    spec = np.zeros((Y, X // 2 + 1), np.complex64)
    ab = PR.AngularBins(15.0, 7.5, 30.0)
    ctx = _RecordingContext(PR.window_size(T))
    ws = PR.WindowSearch(spec, X, Y, T, None, np.zeros((T, T // 2 + 1), np.float32), ab, 0.0, 1.0, context=ctx)
    gy, gx = PR.tile_grid(X, Y)
    last = gy * gx - 1                                   # the bottom-right partial tile
    res = ws.run(PR.Proposal([last], [[0]], None))
    ty, tx = divmod(last, gx)
    h, w = Y - ty * 64, X - tx * 64
    assert 0 < h < 64 and 0 < w < 64
    assert np.all(np.isfinite(res["mip"][ty * 64:, tx * 64:]))
    assert res["mip"].shape == (Y, X)
    assert np.isneginf(res["mip"][:ty * 64, :]).all()
