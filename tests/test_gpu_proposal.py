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
