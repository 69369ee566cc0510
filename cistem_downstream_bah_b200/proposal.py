"""Learned proposal for the fine search (no counterpart in the reference).

A coarse search over every orientation of a coarse angular grid gives, per
pixel, the z-score (MIP normalised by the per-pixel mean and standard
deviation over all its orientations) and the best orientation.  The network
(tm_pnet_* in csrc/tm_proposal.cu) reads TILE x TILE tiles of these maps and
returns, per tile, an objectness logit and a direction.  Tiles whose
objectness passes a threshold get the fine search, but only over the fine
orientations whose out-of-plane direction falls in the K angular bins nearest
to the predicted direction (the bins are the coarse grid's search positions;
every psi of the fine step is searched).  The fine search of a tile runs on a
window of the whitened micrograph around it (``WindowSearch``); with the
projection variance formed over the whole micrograph's pixel count, the
window's correlation values are the full-size search's at the window's
interior positions, so a proposed tile reports the exhaustive search's own
MIP wherever its best orientation was proposed.  z-scores of the proposal path
are normalised with the coarse search's per-pixel statistics (a search over
all orientations of the coarse grid).

Training data are exhaustive fine searches that this package runs on seeded
synthetic micrographs (``training_set``): a tile is positive when it holds a
peak of the exhaustive z-score map at or above the threshold, and its target
direction is the fine best orientation's at that peak.
"""
from __future__ import annotations

import ctypes
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import core, hostprep, prep

FEATURES = 7
TILE = 64
BINS_PER_TILE = 16

_BOUND = False


def _lib():
    global _BOUND
    L = core.load()
    if not _BOUND:
        vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
        dp = ctypes.POINTER(ctypes.c_double)
        L.tm_pnet_create.argtypes = [ip, ip, ip, ip, ctypes.POINTER(vp)]
        L.tm_pnet_param_count.argtypes = [vp]
        L.tm_pnet_param_count.restype = ctypes.c_longlong
        L.tm_pnet_set_params.argtypes = [vp, vp]
        L.tm_pnet_get_params.argtypes = [vp, vp]
        L.tm_pnet_forward.argtypes = [vp, vp, ip, vp]
        L.tm_pnet_gradients.argtypes = [vp, vp, vp, ip, fp, fp, dp, vp]
        L.tm_pnet_train_step.argtypes = [vp, vp, vp, ip, fp, fp, fp, dp]
        L.tm_pnet_last_error.argtypes = [vp]
        L.tm_pnet_last_error.restype = ctypes.c_char_p
        L.tm_pnet_destroy.argtypes = [vp]
        _BOUND = True
    return L


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class ProposalNet:
    """The proposal CNN on one GPU (tm_pnet_create ... tm_pnet_destroy)."""

    def __init__(self, in_channels=FEATURES, tile=TILE, max_batch=256, device=0):
        self.L = _lib()
        self.cin, self.tile, self.max_batch = in_channels, tile, max_batch
        h = ctypes.c_void_p()
        rc = self.L.tm_pnet_create(device, in_channels, tile, max_batch, ctypes.byref(h))
        if rc != core.TM_OK:
            raise core.TmError(rc, "tm_pnet_create failed")
        self.h = h
        self.n_params = int(self.L.tm_pnet_param_count(h))

    def _check(self, rc):
        if rc != core.TM_OK:
            raise core.TmError(rc, self.L.tm_pnet_last_error(self.h).decode())

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        assert p.shape == (self.n_params,), p.shape
        self._check(self.L.tm_pnet_set_params(self.h, _ptr(p)))

    def get_params(self):
        p = np.zeros(self.n_params, np.float32)
        self._check(self.L.tm_pnet_get_params(self.h, _ptr(p)))
        return p

    def _tiles(self, tiles):
        t = np.ascontiguousarray(tiles, np.float32)
        assert t.ndim == 4 and t.shape[1:] == (self.cin, self.tile, self.tile), t.shape
        return t

    def forward(self, tiles):
        t = self._tiles(tiles)
        out = np.zeros((len(t), 4), np.float32)
        for i in range(0, len(t), self.max_batch):
            chunk = np.ascontiguousarray(t[i:i + self.max_batch])
            o = np.zeros((len(chunk), 4), np.float32)
            self._check(self.L.tm_pnet_forward(self.h, _ptr(chunk), len(chunk), _ptr(o)))
            out[i:i + len(chunk)] = o
        return out

    def gradients(self, tiles, labels, pos_weight=1.0, dir_weight=1.0):
        t = self._tiles(tiles)
        lab = np.ascontiguousarray(labels, np.float32)
        g = np.zeros(self.n_params, np.float32)
        loss = ctypes.c_double()
        self._check(self.L.tm_pnet_gradients(self.h, _ptr(t), _ptr(lab), len(t), pos_weight, dir_weight,
                                             ctypes.byref(loss), _ptr(g)))
        return loss.value, g

    def train_step(self, tiles, labels, lr, pos_weight=1.0, dir_weight=1.0):
        t = self._tiles(tiles)
        lab = np.ascontiguousarray(labels, np.float32)
        loss = ctypes.c_double()
        self._check(self.L.tm_pnet_train_step(self.h, _ptr(t), _ptr(lab), len(t), pos_weight, dir_weight, lr,
                                              ctypes.byref(loss)))
        return loss.value

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            self.L.tm_pnet_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def param_layout(cin=FEATURES):
    """[(name, shape)] in the network's flat parameter order."""
    chans = (cin, 32, 64, 128, 128)
    out = []
    for i in range(4):
        out += [(f"w{i + 1}", (chans[i + 1], chans[i], 3, 3)), (f"b{i + 1}", (chans[i + 1],))]
    return out + [("w5", (4, 128)), ("b5", (4,))]


def init_params(cin=FEATURES, seed=0):
    """He-normal weights, zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for name, shape in param_layout(cin):
        n = int(np.prod(shape))
        if name.startswith("w"):
            parts.append(rng.standard_normal(n) * np.sqrt(2.0 / np.prod(shape[1:])))
        else:
            parts.append(np.zeros(n))
    return np.concatenate(parts).astype(np.float32)


# ---------------------------------------------------------------------------------------------
def directions(phi_deg, theta_deg):
    """Unit viewing directions of (phi, theta) search positions."""
    ph = np.radians(np.asarray(phi_deg, np.float64))
    th = np.radians(np.asarray(theta_deg, np.float64))
    return np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=-1)


class AngularBins:
    """Angular neighbourhoods: the search positions of the coarse grid, each
    owning the fine search positions nearest to it."""

    def __init__(self, coarse_step, fine_step, fine_psi_step, symmetry="C1"):
        cg = hostprep.search_grid(coarse_step, symmetry)
        self.centers = directions(cg[:, 0], cg[:, 1])
        self.fine_grid = hostprep.search_grid(fine_step, symmetry)
        fd = directions(self.fine_grid[:, 0], self.fine_grid[:, 1])
        self.bin_of_position = np.argmax(fd @ self.centers.T, axis=1)
        self.fine_angles = core.orientation_list(self.fine_grid, 0.0, fine_psi_step, 360.0)
        self.n_psi = len(self.fine_angles) // len(self.fine_grid)

    @property
    def n_bins(self):
        return len(self.centers)

    def nearest(self, d, k=BINS_PER_TILE):
        """The k bins whose centres are nearest to direction d (any length)."""
        s = self.centers @ np.asarray(d, np.float64)
        return np.argsort(-s, kind="stable")[:k]

    def orientations(self, bins):
        """Rows of fine_angles (in search order) whose position lies in the bins."""
        pos = np.flatnonzero(np.isin(self.bin_of_position, np.asarray(list(bins))))
        return (pos[:, None] * self.n_psi + np.arange(self.n_psi)[None, :]).ravel()


# ---------------------------------------------------------------------------------------------
def search_maps(sc, filt, angles, X, Y):
    """A full search of one context over the given orientations: the raw maps
    plus the finalised scaled MIP, z-score, mean and standard deviation
    (match_template.cpp:1221-1310)."""
    sc.reset()
    t0 = time.perf_counter()
    sc.run_plane(filt, angles)
    r = sc.results()
    secs = time.perf_counter() - t0
    m, z, avg, sd = prep.finalize(r["mip"], r["sum"], r["sumsq"], len(angles), X, Y)
    out = {k: r[k].reshape(Y, X) for k in ("mip", "psi", "theta", "phi")}
    out.update(scaled_mip=m.reshape(Y, X), z=z.reshape(Y, X), avg=avg.reshape(Y, X), sd=sd.reshape(Y, X),
               seconds=secs, points=float(len(angles)) * X * Y)
    return out


def tile_grid(nx, ny, tile=TILE):
    """Tile rows and columns; the last ones may be partial."""
    return -(-ny // tile), -(-nx // tile)


def pad_to_tiles(a, fill, tile=TILE):
    """A map padded (bottom and right, with fill) to whole tiles."""
    gy, gx = tile_grid(a.shape[1], a.shape[0], tile)
    out = np.full((gy * tile, gx * tile), fill, np.float32)
    out[:a.shape[0], :a.shape[1]] = a
    return out


def frame(d):
    """Rotation taking the unit vector d to +z (Rodrigues' formula; the turn
    about x for d = -z)."""
    d = np.asarray(d, np.float64)
    d = d / np.linalg.norm(d)
    z = np.array([0.0, 0.0, 1.0])
    v = np.cross(d, z)
    c = float(d @ z)
    if c < -1.0 + 1e-12:
        return np.diag([1.0, -1.0, -1.0])
    k = np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])
    return np.eye(3) + k + k @ k / (1.0 + c)


def tile_frames(z, theta, phi, tile=TILE):
    """(n_tiles, 3, 3): per tile, the rotation taking the coarse best direction
    at the tile's z-score maximum to +z."""
    ny, nx = z.shape
    gy, gx = tile_grid(nx, ny, tile)
    _, arg = tile_max(z, tile)
    out = np.zeros((gy * gx, 3, 3))
    for i in range(gy * gx):
        ty, tx = divmod(i, gx)
        y = ty * tile + arg[i] // tile
        x = tx * tile + arg[i] % tile
        out[i] = frame(directions(phi[y, x], theta[y, x]))
    return out


def tile_features(z, theta, phi, tile=TILE, frames=None):
    """(n_tiles, FEATURES, tile, tile) float32 from coarse maps: clipped z / 4,
    the best direction weighted by clip(z - 3, 0, 9) / 3, and the direction,
    both directions in the tile's frame (tile_frames), so that the coarse best
    direction at the tile's maximum reads (0, 0, 1)."""
    ny, nx = z.shape
    gy, gx = tile_grid(nx, ny, tile)
    if frames is None:
        frames = tile_frames(z, theta, phi, tile)
    n, P = gy * gx, tile * tile

    def tiles(a):   # (gy*tile, gx*tile, ...) -> (n, P, ...)
        return a.reshape(gy, tile, gx, tile, *a.shape[2:]).swapaxes(1, 2).reshape(n, P, *a.shape[2:])

    # partial tiles: padding reads as z at the clip floor, weight 0, direction +z
    zc = np.clip(pad_to_tiles(z, -4.0, tile), -4.0, 12.0)
    th = np.radians(pad_to_tiles(theta, 0.0, tile))
    ph = np.radians(pad_to_tiles(phi, 0.0, tile))
    st = np.sin(th)
    d = tiles(np.stack([st * np.cos(ph), st * np.sin(ph), np.cos(th)], axis=-1))          # (n, P, 3)
    d = np.matmul(d, np.asarray(frames, np.float32).transpose(0, 2, 1))                    # rows R d
    zt = tiles(zc)
    w = np.clip(zt - 3.0, 0.0, 9.0) / 3.0
    out = np.empty((n, FEATURES, P), np.float32)
    out[:, 0] = zt / 4.0
    dt = d.transpose(0, 2, 1)
    out[:, 1:4] = dt * w[:, None, :]
    out[:, 4:7] = dt
    return out.reshape(n, FEATURES, tile, tile)


def to_frames(labels, frames):
    """Labels with their target directions in the tiles' frames."""
    out = np.array(labels, np.float32, copy=True)
    out[:, 1:4] = np.einsum("nij,nj->ni", frames, labels[:, 1:4])
    return out


def find_peaks(maps, threshold, T, pixel_size=1.0, min_peak_radius=None):
    """Peaks (x, y, z, phi, theta, psi) of a z-score map at or above the
    threshold, as the result aggregation finds them (iterative maximum with an
    exclusion radius, match_template.cpp:1838-1975)."""
    z = maps["z"]
    ny, nx = z.shape
    r = int(min_peak_radius if min_peak_radius is not None else max(10, T // 8))
    zeros = np.zeros_like(z)
    rec = hostprep.find_peaks(z, maps["psi"], maps["theta"], maps["phi"], zeros, zeros, threshold, r, T, pixel_size,
                              max_peaks=100000)
    if len(rec) == 0:
        return np.zeros((0, 6))
    x = np.rint(rec[:, 8]).astype(np.int64)
    y = np.rint(rec[:, 9]).astype(np.int64)
    return np.stack([x, y, z[y, x], maps["phi"][y, x], maps["theta"][y, x], maps["psi"][y, x]], axis=1)


def tile_labels(peaks, nx, ny, tile=TILE):
    """(n_tiles, 4): objectness and the unit direction of the tile's highest peak."""
    gy, gx = tile_grid(nx, ny, tile)
    lab = np.zeros((gy * gx, 4), np.float32)
    best = np.full(gy * gx, -np.inf)
    for x, y, zz, ph, th, _ in peaks:
        ty, tx = int(y) // tile, int(x) // tile
        if ty >= gy or tx >= gx:
            continue
        i = ty * gx + tx
        if zz > best[i]:
            best[i] = zz
            lab[i, 0] = 1.0
            lab[i, 1:] = directions(ph, th)
    return lab


def dihedral(tiles, k):
    """The k-th of the 8 rotations/flips of square tiles (labels unchanged:
    in-plane rotations and mirrors of the maps keep the viewing direction
    channels' values)."""
    t = np.rot90(tiles, k % 4, axes=(2, 3))
    if k >= 4:
        t = t[:, :, :, ::-1]
    return np.ascontiguousarray(t)


# ---------------------------------------------------------------------------------------------
class Proposal:
    """Selected tiles and their angular bins."""

    def __init__(self, tiles, bins, scores):
        self.tiles = np.asarray(tiles, np.int64)
        self.bins = bins
        self.scores = scores


def network_directions(out, frames):
    """The network's directions rotated back out of the tiles' frames."""
    return np.einsum("nji,nj->ni", frames, out[:, 1:4].astype(np.float64))


def propose_network(net, feats, frames, logit_threshold, angular, k=BINS_PER_TILE, out=None):
    """Tiles whose objectness logit reaches the threshold, with the k bins
    nearest to the network's direction."""
    if out is None:
        out = net.forward(feats)
    d = network_directions(out, frames)
    sel = np.flatnonzero(out[:, 0] >= logit_threshold)
    return Proposal(sel, [angular.nearest(d[i], k) for i in sel], out[:, 0])


def tiles_for_recall(peak_tiles, recoverable, ranking, levels=(0.9, 0.95, 0.99, 1.0)):
    """Tiles taken in ranking order until a share of the peaks is recovered
    (a peak counts once its tile is taken, if its bin is among that tile's);
    None where the share cannot be reached."""
    pos = np.empty(len(ranking), np.int64)
    pos[np.asarray(ranking)] = np.arange(len(ranking))
    need = np.sort(np.where(recoverable, pos[np.asarray(peak_tiles, np.int64)] + 1, np.iinfo(np.int64).max))
    out = {}
    for q in levels:
        if len(need) == 0:
            out[str(q)] = 0
            continue
        k = int(np.ceil(q * len(need))) - 1
        out[str(q)] = None if need[k] == np.iinfo(np.int64).max else int(need[k])
    return out


def tile_max(z, tile=TILE):
    ny, nx = z.shape
    gy, gx = tile_grid(nx, ny, tile)
    zt = pad_to_tiles(z, -np.inf, tile).reshape(gy, tile, gx, tile).transpose(0, 2, 1, 3).reshape(gy * gx, tile * tile)
    return zt.max(axis=1), zt.argmax(axis=1)


def propose_heuristic(coarse, threshold, angular, k=BINS_PER_TILE, tile=TILE):
    """The method without the network: tiles whose coarse z-score maximum
    reaches the threshold, bins nearest to the coarse best direction there."""
    z = coarse["z"]
    ny, nx = z.shape
    gy, gx = tile_grid(nx, ny, tile)
    zmax, arg = tile_max(z, tile)
    sel = np.flatnonzero(zmax >= threshold)
    bins = []
    for i in sel:
        ty, tx = divmod(int(i), gx)
        y = ty * tile + arg[i] // tile
        x = tx * tile + arg[i] % tile
        bins.append(angular.nearest(directions(coarse["phi"][y, x], coarse["theta"][y, x]), k))
    return Proposal(sel, bins, zmax)


# ---------------------------------------------------------------------------------------------
def whitened_real(ispec, X, Y):
    """Real-space micrograph of a whitened, quadrant-swapped half spectrum
    (inverse of the forward transform with its 1/N; the swap is a sign pattern
    for even sizes)."""
    ky = np.arange(Y)[:, None]
    kx = np.arange(X // 2 + 1)[None, :]
    sign = np.where(((ky + kx) & 1) == 1, -1.0, 1.0)
    return np.fft.irfft2(ispec.astype(np.complex128) * sign, s=(Y, X)) * (X * Y)


def window_spectrum(s, x0, y0, W, n_full, used):
    """Half spectrum of the W x W window at (x0, y0) of the periodic image s, as
    the search context takes it for a window cut from a micrograph of n_full
    pixels.  The context divides its image spectrum by its own pixel count and
    drops the DC term (tm_set_image); so the forward transform is divided by
    n_full, and the pixels outside the window's used square [used[0],
    used[1])^2 -- pixels no interior correlation reads -- are set to the
    constant that makes the window's mean zero, which leaves nothing for the
    dropped DC term to remove.  The quadrant swap is that of the window size."""
    Y, X = s.shape
    win = s[np.ix_((y0 + np.arange(W)) % Y, (x0 + np.arange(W)) % X)].copy()
    lo, hi = used
    inside = np.zeros((W, W), bool)
    inside[lo:hi, lo:hi] = True
    n_out = W * W - (hi - lo) ** 2
    assert n_out > 0, "the window needs pixels outside its used square"
    win[~inside] = -win[inside].sum() / n_out
    spec = np.fft.rfft2(win) / n_full
    ky = np.arange(W)[:, None]
    kx = np.arange(W // 2 + 1)[None, :]
    return (spec * np.where(((ky + kx) & 1) == 1, -1.0, 1.0)).astype(np.complex64)


def window_size(T):
    """Window edge for a template box: 2T, at least 256."""
    return max(2 * T, 256)


def window_core(T):
    """Edge of the window's interior (whole tiles): the window less the template
    box and a band of one tile that no interior correlation reads."""
    return window_size(T) - T - TILE


class WindowSearch:
    """Fine search of proposed tiles on windows of the whitened micrograph.
    The windows form an image set of one search context; the fine orientations
    are run one angular bin at a time over the windows that need that bin, so
    the per-orientation slice and projection work is shared between them.
    Within a window the bins go in increasing order (a tie between
    orientations of different bins keeps the lower bin's)."""

    def __init__(self, ispec, X, Y, T, tspec, filt, angular, hmin, hstep, device=0, context=None):
        """context: a search context of the window geometry to use instead of a new one."""
        self.X, self.Y, self.T = X, Y, T
        self.W = window_size(T)
        self.core = window_core(T)
        assert self.core % TILE == 0 and self.core >= TILE
        self.margin = (self.W - self.core - T) // 2   # unread pixels on each side of the used square
        self.s = whitened_real(ispec, X, Y)
        self.filt = filt
        self.angular = angular
        self.max_set = 128   # windows per image set (about 8 MB of device state each at 512^2)
        self._slots = 0      # images in the context's current set
        # 256 orientations per device pass: at these small boxes the per-pass costs weigh (1.4x over 32)
        self.sc = context if context is not None else core.SearchCore(
            self.W, self.W, T, histogram_min_scaled=hmin, histogram_step_scaled=hstep, orientation_batch=256,
            device=device)
        self.sc.set_template(tspec)
        self.sc.set_normalization_pixels(X * Y)

    def run(self, proposal):
        """MIP / best angles over the proposed tiles (-inf elsewhere), with the
        number of correlation points and the device-side wall time."""
        X, Y, T, W, C = self.X, self.Y, self.T, self.W, self.core
        gx = tile_grid(X, Y)[1]
        per_core = C // TILE
        mip = np.full((Y, X), -np.inf, np.float32)
        ang = {k: np.zeros((Y, X), np.float32) for k in ("phi", "theta", "psi")}
        groups = {}
        for t, b in zip(proposal.tiles, proposal.bins):
            ty, tx = divmod(int(t), gx)
            groups.setdefault((ty // per_core, tx // per_core), []).append((ty, tx, b))
        m = self.margin

        def prepare(entry):
            """Bins and spectrum of one window (host work)."""
            (cy, cx), items = entry
            bins = set()
            for _, _, b in items:
                bins.update(int(v) for v in b)
            x0, y0 = cx * C - T // 2 - m, cy * C - T // 2 - m
            # the used square keeps two pixels beyond the interior's reach on each side
            spec = window_spectrum(self.s, x0, y0, W, X * Y, (m - 2, W - m + 2))
            return items, bins, spec, x0, y0

        points = 0.0
        launches = 0
        B = self.sc.orientation_batch() if hasattr(self.sc, "orientation_batch") else 256
        t0 = time.perf_counter()
        entries = sorted(groups.items())
        with ThreadPoolExecutor(max_workers=4) as pool:
            for c0 in range(0, len(entries), self.max_set):
                chunk = list(pool.map(prepare, entries[c0:c0 + self.max_set]))
                # one image set per chunk of windows; each angular bin's orientations are
                # sliced and projected once and correlated with every window that needs the bin
                self.sc.set_image_set(np.stack([e[2] for e in chunk]))
                # the results reset (main state and the previous set), then per image: prepare, reset
                launches += 1 + self._slots + 2 * len(chunk)
                self._slots = len(chunk)
                by_bin = {}
                for wi, (_, bins, _, _, _) in enumerate(chunk):
                    for b in bins:
                        by_bin.setdefault(b, []).append(wi)
                for b in sorted(by_bin):
                    angles = self.angular.fine_angles[self.angular.orientations([b])]
                    self.sc.run_plane_images(self.filt, angles, by_bin[b])
                    points += float(len(angles)) * W * W * len(by_bin[b])
                    # per orientation batch: slice, rows, normalisation, pass A; passes B and C per window
                    launches += -(-len(angles) // B) * (4 + 2 * len(by_bin[b]))
                for wi, (items, _, _, x0, y0) in enumerate(chunk):
                    r = self.sc.image_results(wi)
                    wm = r["mip"].reshape(W, W)
                    for ty, tx, _ in items:
                        # a partial last tile keeps its pixels inside the micrograph
                        h = min(TILE, Y - ty * TILE)
                        w = min(TILE, X - tx * TILE)
                        ys = slice(ty * TILE, ty * TILE + h)
                        xs = slice(tx * TILE, tx * TILE + w)
                        wy = slice(ty * TILE - y0, ty * TILE - y0 + h)
                        wx = slice(tx * TILE - x0, tx * TILE - x0 + w)
                        mip[ys, xs] = wm[wy, wx]
                        for k in ang:
                            ang[k][ys, xs] = r[k].reshape(W, W)[wy, wx]
        return {"mip": mip, **ang, "points": points, "seconds": time.perf_counter() - t0, "windows": len(groups),
                "launches": launches}

    def close(self):
        self.sc.close()


def proposal_z(window_result, coarse, X, Y):
    """z-score of the proposal path: fine MIP x sqrt(N), normalised with the
    coarse search's per-pixel mean and standard deviation."""
    m = window_result["mip"].astype(np.float64) * np.float32(np.sqrt(float(X * Y)))
    sd = coarse["sd"].astype(np.float64)
    return np.where(np.isfinite(m) & (sd > 0), (m - coarse["avg"]) / np.where(sd > 0, sd, 1.0), -np.inf)


def recall(peaks, exhaustive, window_result, z_prop, threshold, radius=1, rel_tol=1e-4):
    """Fraction of exhaustive peaks the proposal path recovers: (a) its MIP
    reaches the exhaustive MIP within rel_tol at the peak (within radius px);
    (b) its z-score reaches the threshold there."""
    if len(peaks) == 0:
        return 1.0, 1.0
    Y, X = z_prop.shape
    hit_m = hit_z = 0
    for x, y, *_ in peaks:
        x, y = int(x), int(y)
        ys = slice(max(0, y - radius), min(Y, y + radius + 1))
        xs = slice(max(0, x - radius), min(X, x + radius + 1))
        ref = float(exhaustive["mip"][y, x])
        got = float(np.max(window_result["mip"][ys, xs]))
        hit_m += got >= ref - rel_tol * abs(ref)
        hit_z += float(np.max(z_prop[ys, xs])) >= threshold
    return hit_m / len(peaks), hit_z / len(peaks)


def propose_top_tiles(coarse, n_tiles, angular, k=BINS_PER_TILE, tile=TILE):
    """The method without the network at a given tile budget: the n_tiles tiles
    with the highest coarse z-score maximum, bins nearest to the coarse best
    direction there."""
    zmax, _ = tile_max(coarse["z"], tile)
    order = np.argsort(-zmax, kind="stable")[:n_tiles]
    thr = float(zmax[order[-1]]) if len(order) else np.inf
    p = propose_heuristic(coarse, thr, angular, k, tile)
    keep = np.isin(p.tiles, order)
    return Proposal(p.tiles[keep], [b for b, kk in zip(p.bins, keep) if kk], zmax)


def peak_diagnostics(peaks, exhaustive, coarse, proposals, angular, tile=TILE):
    """Per exhaustive peak: its z, the distance to the nearest higher peak, the
    angular bin of its best orientation, and for each proposal whether its tile
    was selected, the rank of that bin among the tile's proposed bins (-1: not
    proposed) and whether the proposal recovers the peak (tile selected, bin
    proposed: the window search then evaluates the exhaustive search's own best
    orientation there).  Also the rank of the bin around the coarse best
    direction at the peak pixel itself."""
    Y, X = coarse["z"].shape
    gx = tile_grid(X, Y, tile)[1]
    n = len(peaks)
    out = {"z": np.array([p[2] for p in peaks]), "x": np.array([p[0] for p in peaks]),
           "y": np.array([p[1] for p in peaks])}
    d_near = np.full(n, np.inf)
    for i in range(n):
        for j in range(n):
            if peaks[j][2] > peaks[i][2]:
                d_near[i] = min(d_near[i], float(np.hypot(peaks[i][0] - peaks[j][0], peaks[i][1] - peaks[j][1])))
    out["dist_to_higher_peak"] = d_near
    bins = np.array([int(np.argmax(angular.centers @ directions(p[3], p[4]))) for p in peaks], np.int64)
    out["bin"] = bins
    rank_here = []
    for p, b in zip(peaks, bins):
        x, y = int(p[0]), int(p[1])
        order = angular.nearest(directions(coarse["phi"][y, x], coarse["theta"][y, x]), angular.n_bins)
        rank_here.append(int(np.flatnonzero(order == b)[0]))
    out["bin_rank_at_peak_coarse_direction"] = np.array(rank_here)
    for name, prop in proposals.items():
        where = {int(t): i for i, t in enumerate(prop.tiles)}
        sel = np.zeros(n, bool)
        rank = np.full(n, -1)
        for i, (p, b) in enumerate(zip(peaks, bins)):
            t = (int(p[1]) // tile) * gx + int(p[0]) // tile
            if t in where:
                sel[i] = True
                pb = np.asarray(prop.bins[where[t]])
                hit = np.flatnonzero(pb == b)
                rank[i] = int(hit[0]) if len(hit) else -1
        out[name + "_selected"] = sel
        out[name + "_bin_rank"] = rank
        out[name + "_recovered"] = sel & (rank >= 0)
    return out
