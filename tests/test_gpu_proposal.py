"""Learned proposal on the GPU: the network kernels (tm_pnet_*) against the
FP64 oracle's outputs and gradients, a training run that lowers the loss,
and the window search of proposed tiles against the full-size search over
the same orientations."""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import core, hostprep, prep
from cistem_downstream_bah_b200 import proposal as PR
from cistem_downstream_bah_b200 import synthetic
from oracle import proposal as OP

pytestmark = pytest.mark.gpu


def _labels(n, rng):
    lab = np.zeros((n, 4), np.float32)
    lab[::2, 0] = 1
    d = rng.standard_normal((n, 3))
    lab[:, 1:] = d / np.linalg.norm(d, axis=1, keepdims=True)
    lab[1::2, 1:] = 0
    return lab


def _layer_slices(cin):
    out, o = {}, 0
    for name, shape in OP.layout(cin):
        n = int(np.prod(shape))
        out[name] = slice(o, o + n)
        o += n
    return out


@pytest.mark.parametrize("tile,n", [(16, 5), (64, 3)])
def test_network_matches_oracle(tile, n):
    rng = np.random.default_rng(tile + n)
    cin = PR.FEATURES
    params = PR.init_params(cin, seed=tile)
    params[_layer_slices(cin)["b1"]] = 0.05
    x = rng.standard_normal((n, cin, tile, tile)).astype(np.float32)
    lab = _labels(n, rng)
    net = PR.ProposalNet(cin, tile, max_batch=8)
    try:
        net.set_params(params)
        assert np.array_equal(net.get_params(), params)
        out = net.forward(x)
        ref, _ = OP.forward(params.astype(np.float64), x, cin, bf16=True)
        assert np.abs(out - ref).max() <= 1e-4 * max(1.0, np.abs(ref).max())
        loss, g = net.gradients(x, lab, pos_weight=2.0, dir_weight=0.5)
        rloss, rg = OP.gradients(params.astype(np.float64), x, lab, cin, 2.0, 0.5, bf16=True)
        assert abs(loss - rloss) <= 1e-4 * abs(rloss)
        for name, sl in _layer_slices(cin).items():
            a, b = g[sl].astype(np.float64), rg[sl]
            # relative L2 error per tensor (a max-pool near-tie may route one
            # pixel differently in FP32 than in FP64)
            assert np.linalg.norm(a - b) <= 2e-3 * np.linalg.norm(b) + 1e-7, name
    finally:
        net.close()


def test_training_lowers_loss():
    """Tiles with a bright blob are positive; the target direction is the
    direction channels' value at the blob."""
    rng = np.random.default_rng(7)
    n, tile = 64, 16
    x = (0.3 * rng.standard_normal((n, PR.FEATURES, tile, tile))).astype(np.float32)
    lab = np.zeros((n, 4), np.float32)
    for i in range(0, n, 2):
        y0, x0 = rng.integers(2, tile - 2, 2)
        d = rng.standard_normal(3)
        d /= np.linalg.norm(d)
        x[i, 0, y0, x0] += 3.0
        x[i, 1:4, y0, x0] = 2.0 * d
        x[i, 4:7, y0, x0] = d
        lab[i] = [1.0, *d]
    net = PR.ProposalNet(PR.FEATURES, tile, max_batch=n)
    try:
        net.set_params(PR.init_params(seed=1))
        first = net.train_step(x, lab, lr=1e-3)
        for _ in range(300):
            last = net.train_step(x, lab, lr=1e-3)
        assert last < 0.3 * first, (first, last)
        out = net.forward(x)
        assert np.all((out[::2, 0] > 0)) and np.all(out[1::2, 0] < 0)
        cos = (out[::2, 1:] * lab[::2, 1:]).sum(1) / np.linalg.norm(out[::2, 1:], axis=1)
        assert np.median(cos) > 0.9
    finally:
        net.close()


@pytest.mark.parametrize("T,N,px,atoms,radius", [(64, 1024, 1.5, 3000, 40.0), (256, 4096, 1.0, 20000, 110.0)])
def test_window_search_matches_full_search(T, N, px, atoms, radius):
    vol = synthetic.template_volume(T, px, atoms, radius, seed=T)
    mic, _ = synthetic.micrograph(N, N, px, atoms, radius, 6, 0.05, 12000.0, seed=T + 1, atom_seed=T)
    ispec, curve = hostprep.whiten(mic)
    tspec = hostprep.template_spectrum(vol)
    filt = hostprep.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=12000.0,
                                      defocus2=12000.0, pixel_size=px)
    hmin, hstep = prep.histogram_scaled(N, N)
    ab = PR.AngularBins(7.5, 2.5, 6.0)
    bins = ab.nearest(PR.directions(40.0, 70.0), 2)
    angles = ab.fine_angles[ab.orientations(bins)]
    sc = core.SearchCore(N, N, T, histogram_min_scaled=hmin, histogram_step_scaled=hstep)
    try:
        sc.set_image(ispec)
        sc.set_template(tspec)
        sc.reset()
        sc.run_plane(filt, angles)
        full = sc.results()
    finally:
        sc.close()
    gx = N // PR.TILE
    tiles = [0, 5, 3 * gx + 7, gx * gx - 1, (gx // 2) * gx + gx // 2 + 1]
    ws = PR.WindowSearch(ispec, N, N, T, tspec, filt, ab, hmin, hstep)
    try:
        res = ws.run(PR.Proposal(tiles, [bins] * len(tiles), None))
    finally:
        ws.close()
    assert res["points"] == float(len(angles)) * ws.W * ws.W * res["windows"]
    fm = full["mip"].reshape(N, N)
    scale = np.abs(fm).max()
    same = 0
    total = 0
    for t in tiles:
        ty, tx = divmod(t, gx)
        ys, xs = slice(ty * 64, ty * 64 + 64), slice(tx * 64, tx * 64 + 64)
        assert np.abs(res["mip"][ys, xs] - fm[ys, xs]).max() <= 2e-5 * scale, t
        for k in ("psi", "theta", "phi"):
            same += int((res[k][ys, xs] == full[k].reshape(N, N)[ys, xs]).sum())
            total += 64 * 64
    assert same >= 0.99 * total
    untouched = np.ones((N, N), bool)
    for t in tiles:
        ty, tx = divmod(t, gx)
        untouched[ty * 64:ty * 64 + 64, tx * 64:tx * 64 + 64] = False
    assert np.all(np.isneginf(res["mip"][untouched]))


def test_trained_network_gains_over_the_method_without_it():
    """On a case outside the training set (1024^2, 128^3 template), with the
    committed weights: at a budget of 3 tiles per strong peak, the trained
    network's proposals recover every exhaustive peak above the reference's
    expected threshold, an untrained network's do not, and the coarse-z
    ranking (the method without the network) is reported beside them."""
    import os
    from cistem_downstream_bah_b200 import proposal_train as PT
    path = os.path.join(os.path.dirname(PR.__file__), "data", "proposal_net.npz")
    w = np.load(path)
    angular = PR.AngularBins(7.5, 2.5, 1.5)
    coarse_angles = core.orientation_list(hostprep.search_grid(7.5), 0.0, 5.0, 360.0)
    c = dict(T=128, pixel_size=1.5, radius_A=70.0, n_atoms=16000, particles=10, snr=0.05, defocus=14000.0, seed=5003)
    cs = PT.search_case(c, angular, coarse_angles, keep_maps=True)
    n_orient = len(angular.fine_angles)
    thr = float(np.sqrt(2.0) * hostprep.lib().tmh_erfcinv(2.0 / (1024.0 * 1024.0 * n_orient)))
    strong = cs["peaks"][cs["peaks"][:, 2] >= thr]
    assert len(strong) >= 5, len(strong)
    budget = 3 * len(strong)
    coarse_dirs = PT.coarse_directions(cs["coarse"])
    gx = 1024 // PR.TILE

    def recall(scores, dirs):
        take = set(np.argsort(-scores, kind="stable")[:budget].tolist())
        hit = 0
        for x, y, _, ph, th, _ in strong:
            t = (int(y) // PR.TILE) * gx + int(x) // PR.TILE
            hit += t in take and PT.bins_hit(angular, angular.nearest(dirs[t]), PR.directions(ph, th))
        return hit / len(strong)

    trained = PT.network_scores(w["params"], cs["feats"])
    untrained = PT.network_scores(PR.init_params(seed=3), cs["feats"])
    r_trained = recall(trained[:, 0], PR.network_directions(trained, cs["frames"]))
    r_untrained = recall(untrained[:, 0], PR.network_directions(untrained, cs["frames"]))
    r_coarse = recall(cs["coarse_tile_max"], coarse_dirs)
    print(f"strong peaks {len(strong)}, budget {budget} of {gx * gx} tiles: trained {r_trained:.3f}, "
          f"untrained {r_untrained:.3f}, coarse z {r_coarse:.3f}")
    assert r_trained == 1.0
    assert r_untrained < r_trained


def test_normalization_pixels_argument():
    sc = core.SearchCore(256, 256, 64, histogram_min_scaled=-0.05, histogram_step_scaled=0.001)
    try:
        with pytest.raises(core.TmError):
            sc.set_normalization_pixels(-1)
        sc.set_normalization_pixels(1024 * 1024)
        sc.set_normalization_pixels(0)
    finally:
        sc.close()


def test_image_set_matches_single_images():
    """Three windows in one image set, bins run over different subsets of them,
    give the maps of the same windows searched one at a time."""
    T, N, W = 64, 1024, 256
    vol = synthetic.template_volume(T, 1.5, 3000, 40.0, seed=9)
    mic, _ = synthetic.micrograph(N, N, 1.5, 3000, 40.0, 6, 0.05, 12000.0, seed=10, atom_seed=9)
    ispec, curve = hostprep.whiten(mic)
    tspec = hostprep.template_spectrum(vol)
    filt = hostprep.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=12000.0,
                                      defocus2=12000.0, pixel_size=1.5)
    s = PR.whitened_real(ispec, N, N)
    spectra = np.stack([PR.window_spectrum(s, x0, y0, W, N * N, (30, W - 30)) for x0, y0 in
                        [(0, 0), (300, 500), (-100, 900)]])
    ab = PR.AngularBins(7.5, 2.5, 6.0)
    ba, bb = ab.nearest(PR.directions(10.0, 50.0), 2)
    ang = {b: ab.fine_angles[ab.orientations([b])] for b in (ba, bb)}
    plan = [[ba], [ba, bb], [bb]]
    hmin, hstep = prep.histogram_scaled(N, N)
    sc = core.SearchCore(W, W, T, histogram_min_scaled=hmin, histogram_step_scaled=hstep, orientation_batch=64)
    try:
        sc.set_template(tspec)
        sc.set_normalization_pixels(N * N)
        sc.set_image_set(spectra)
        sc.run_plane_images(filt, ang[ba], [0, 1])
        sc.run_plane_images(filt, ang[bb], [1, 2])
        got = [sc.image_results(k) for k in range(3)]
        for k, bins in enumerate(plan):
            sc.set_image(spectra[k])
            sc.reset()
            for b in bins:
                sc.run_plane(filt, ang[b])
            ref = sc.results()
            for key in ("mip", "psi", "theta", "phi"):
                assert np.array_equal(got[k][key], ref[key]), (k, key)
        with pytest.raises(core.TmError):
            sc.run_plane_images(filt, ang[ba], [3])
    finally:
        sc.close()
