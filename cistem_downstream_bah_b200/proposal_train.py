"""Training of the proposal network on exhaustive searches of synthetic micrographs.

    python -m cistem_downstream_bah_b200.proposal_train --micrographs 24 --out net.npz

Each seeded case is a 1024 x 1024 micrograph of ten copies of a random
Gaussian-atom template (box 64 or 128, defocus 5,000-25,000 A, per-particle SNR
0.02-0.08).  Per case the search runs twice on the GPU: the coarse grid
(7.5 / 5 degrees), whose z-score and best-orientation maps are the network's
input, and the exhaustive fine grid (2.5 / 1.5 degrees), whose z >= 7 peaks are
its labels.  Cases are split into training, validation and held-out sets; the network is
trained with Adam on balanced batches (positives drawn with replacement under
the 8 rotations/flips of the tile); the objectness threshold keeps a set
share of the training and validation positives (less a margin), and the held-out cases
measure recall and searched points against the exhaustive search, beside the
method without the network (tiles by coarse z -- at its own threshold and at
the network's tile count -- with bins around the coarse best direction).
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import core, hostprep, prep, synthetic
from . import proposal as PR

FINE = (2.5, 1.5)
COARSE = (7.5, 5.0)
Z_THRESHOLD = 7.0
N = 1024


def case_params(seed):
    rng = np.random.default_rng(seed)
    T = int(rng.choice([64, 128]))
    px = 1.5
    radius = float(rng.uniform(0.30, 0.42) * T * px)
    atoms = int(3000 * (radius / 40.0) ** 3)
    return dict(T=T, pixel_size=px, radius_A=radius, n_atoms=atoms, particles=10, snr=float(rng.uniform(0.02, 0.08)),
                defocus=float(rng.uniform(5000.0, 25000.0)), seed=seed)


def search_case(c, angular, coarse_angles, device=0, keep_maps=False):
    """Coarse and exhaustive fine search of one synthetic case."""
    T, px = c["T"], c["pixel_size"]
    vol = synthetic.template_volume(T, px, c["n_atoms"], c["radius_A"], seed=c["seed"])
    mic, _ = synthetic.micrograph(N, N, px, c["n_atoms"], c["radius_A"], c["particles"], c["snr"], c["defocus"],
                                  seed=c["seed"] + 1, atom_seed=c["seed"])
    ispec, curve = hostprep.whiten(mic)
    tspec = hostprep.template_spectrum(vol)
    filt = hostprep.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=c["defocus"],
                                      defocus2=c["defocus"], pixel_size=px)
    hmin, hstep = prep.histogram_scaled(N, N)
    sc = core.SearchCore(N, N, T, histogram_min_scaled=hmin, histogram_step_scaled=hstep, device=device)
    try:
        sc.set_image(ispec)
        sc.set_template(tspec)
        coarse = PR.search_maps(sc, filt, coarse_angles, N, N)
        fine = PR.search_maps(sc, filt, angular.fine_angles, N, N)
    finally:
        sc.close()
    peaks = PR.find_peaks(fine, Z_THRESHOLD, T, px)
    frames = PR.tile_frames(coarse["z"], coarse["theta"], coarse["phi"])
    labels = PR.tile_labels(peaks, N, N)
    out = dict(case=c, feats=PR.tile_features(coarse["z"], coarse["theta"], coarse["phi"], frames=frames),
               frames=frames, labels=labels, labels_local=PR.to_frames(labels, frames), peaks=peaks,
               coarse_tile_max=PR.tile_max(coarse["z"])[0], seconds=(coarse["seconds"], fine["seconds"]))
    if keep_maps:
        out.update(coarse=coarse, fine=fine, ispec=ispec, tspec=tspec, filt=filt, hmin=hmin, hstep=hstep)
    return out


def train(feats, labels, steps=1500, batch=128, lr=1e-3, seed=0, dir_weight=1.0, device=0, log=None):
    """Adam on balanced batches; returns the trained parameters and the loss curve."""
    rng = np.random.default_rng(seed)
    pos = np.flatnonzero(labels[:, 0] > 0.5)
    neg = np.flatnonzero(labels[:, 0] <= 0.5)
    net = PR.ProposalNet(PR.FEATURES, PR.TILE, max_batch=batch, device=device)
    curve = []
    try:
        net.set_params(PR.init_params(seed=seed))
        n_pos = batch // 4 if len(pos) else 0
        for s in range(steps):
            idx = np.concatenate([rng.choice(pos, n_pos) if n_pos else np.zeros(0, np.int64),
                                  rng.choice(neg, batch - n_pos)])
            k = int(rng.integers(8))
            x = PR.dihedral(feats[idx], k)
            rate = lr * (0.1 if s >= int(0.8 * steps) else 1.0)
            loss = net.train_step(x, labels[idx], rate, pos_weight=1.0, dir_weight=dir_weight)
            curve.append(loss)
            if log and (s % 100 == 0 or s == steps - 1):
                log(f"step {s} loss {np.mean(curve[-100:]):.4f}")
        params = net.get_params()
    finally:
        net.close()
    return params, np.array(curve)


def threshold_for(scores, labels, margin, keep=1.0):
    """Threshold that keeps the share `keep` of the positives, lowered by the margin."""
    pos = np.sort(scores[labels[:, 0] > 0.5])
    if not len(pos):
        return float("inf")
    return float(pos[int(np.floor((1.0 - keep) * (len(pos) - 1)))] - margin)


def network_scores(params, feats, device=0):
    net = PR.ProposalNet(PR.FEATURES, PR.TILE, max_batch=256, device=device)
    try:
        net.set_params(params)
        out = net.forward(feats)
    finally:
        net.close()
    return out


def bins_hit(angular, bins, label_dir):
    """Whether the label direction's bin is among the proposed bins."""
    target = int(np.argmax(angular.centers @ label_dir))
    return target in set(int(b) for b in bins)


def evaluate(cases, params, net_logit_threshold, heur_threshold, angular, device=0):
    """Recall of labelled tiles (tile selected and the label's bin proposed)
    and the fine-search points each method asks for, over the given cases."""
    res = {k: dict(tiles=0, hit=0, points=0.0, missed_not_selected=0, missed_bin=0)
           for k in ("network", "heuristic", "top_tiles")}
    res["positives"] = 0
    per_bin = len(angular.fine_angles) / angular.n_bins
    rank_net, rank_top, peak_tiles, rec_net, rec_top = [], [], [], [], []
    offset = 0
    for cs in cases:
        out = network_scores(params, cs["feats"], device)
        ndir = PR.network_directions(out, cs["frames"])
        lab = cs["labels"]
        posi = np.flatnonzero(lab[:, 0] > 0.5)
        res["positives"] += len(posi)
        net_mask = out[:, 0] >= net_logit_threshold
        top_mask = np.zeros(len(lab), bool)
        top_mask[np.argsort(-cs["coarse_tile_max"], kind="stable")[:int(net_mask.sum())]] = True
        for name, sel_mask, dirs in (
                ("network", net_mask, ndir),
                ("heuristic", cs["coarse_tile_max"] >= heur_threshold, cs.get("coarse_dirs")),
                ("top_tiles", top_mask, cs.get("coarse_dirs"))):
            sel = np.flatnonzero(sel_mask)
            r = res[name]
            r["tiles"] += len(sel)
            W = PR.window_size(cs["case"]["T"])
            r["points"] += len(sel) * PR.BINS_PER_TILE * per_bin * W * W
            for i in posi:
                if not sel_mask[i]:
                    r["missed_not_selected"] += 1
                    continue
                h = bins_hit(angular, angular.nearest(dirs[i]), lab[i, 1:4])
                r["hit"] += h
                r["missed_bin"] += 1 - h
        # recall against tiles taken in each method's order, all cases pooled
        rank_net.append(out[:, 0])
        rank_top.append(cs["coarse_tile_max"])
        for i in posi:
            peak_tiles.append(offset + i)
            rec_net.append(bins_hit(angular, angular.nearest(ndir[i]), lab[i, 1:4]))
            rec_top.append(bins_hit(angular, angular.nearest(cs["coarse_dirs"][i]), lab[i, 1:4]))
        offset += len(lab)
    if peak_tiles:
        res["tiles_for_recall"] = {
            "network": PR.tiles_for_recall(peak_tiles, np.array(rec_net, bool),
                                           np.argsort(-np.concatenate(rank_net), kind="stable")),
            "coarse_z": PR.tiles_for_recall(peak_tiles, np.array(rec_top, bool),
                                            np.argsort(-np.concatenate(rank_top), kind="stable")),
            "tiles": offset}
    return res


def coarse_directions(coarse):
    """Direction at each tile's coarse z maximum (the heuristic's bin centre)."""
    z = coarse["z"]
    gy, gx = PR.tile_grid(z.shape[1], z.shape[0])
    _, arg = PR.tile_max(z)
    out = np.zeros((gy * gx, 3))
    for i in range(gy * gx):
        ty, tx = divmod(i, gx)
        y = ty * PR.TILE + arg[i] // PR.TILE
        x = tx * PR.TILE + arg[i] % PR.TILE
        out[i] = PR.directions(coarse["phi"][y, x], coarse["theta"][y, x])
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--micrographs", type=int, default=24)
    ap.add_argument("--validation", type=int, default=6, help="cases that set the objectness threshold")
    ap.add_argument("--held-out", type=int, default=6, help="cases that only measure")
    ap.add_argument("--steps", type=int, default=1500)
    ap.add_argument("--keep", type=float, default=0.95,
                    help="share of training and validation positives the objectness threshold keeps")
    ap.add_argument("--seed", type=int, default=1000)
    ap.add_argument("--out", required=True)
    ap.add_argument("--summary", default=None)
    ap.add_argument("--device", type=int, default=0)
    args = ap.parse_args(argv)
    log = lambda m: print(m, flush=True)   # noqa: E731
    angular = PR.AngularBins(COARSE[0], *FINE)
    coarse_angles = core.orientation_list(hostprep.search_grid(COARSE[0]), 0.0, COARSE[1], 360.0)
    cases = []
    t0 = time.perf_counter()
    for i in range(args.micrographs):
        c = case_params(args.seed + 7 * i)
        cs = search_case(c, angular, coarse_angles, args.device, keep_maps=True)
        cs["coarse_dirs"] = coarse_directions(cs["coarse"])
        for k in ("coarse", "fine", "ispec", "tspec", "filt"):
            cs.pop(k)
        cases.append(cs)
        log(f"case {i}: T={c['T']} snr={c['snr']:.3f} df={c['defocus']:.0f} peaks={len(cs['peaks'])} "
            f"positive tiles={int(cs['labels'][:, 0].sum())} search s={cs['seconds'][0]:.2f}+{cs['seconds'][1]:.2f}")
    gen_s = time.perf_counter() - t0
    nv, nh = args.validation, args.held_out
    train_cases, val, held = cases[:-(nv + nh)], cases[-(nv + nh):-nh], cases[-nh:]
    feats = np.concatenate([c["feats"] for c in train_cases])
    labels = np.concatenate([c["labels_local"] for c in train_cases])
    log(f"training tiles {len(feats)}, positives {int(labels[:, 0].sum())}")
    t0 = time.perf_counter()
    params, curve = train(feats, labels, steps=args.steps, seed=args.seed, device=args.device, log=log)
    train_s = time.perf_counter() - t0
    # thresholds: every training and validation positive kept, less a margin
    fit = train_cases + val
    fit_labels = np.concatenate([c["labels"] for c in fit])
    out = np.concatenate([network_scores(params, c["feats"], args.device) for c in fit])
    net_thr = threshold_for(out[:, 0], fit_labels, margin=0.5, keep=args.keep)
    heur_thr = threshold_for(np.concatenate([c["coarse_tile_max"] for c in fit]), fit_labels, margin=0.25,
                             keep=args.keep)
    ev_train = evaluate(train_cases, params, net_thr, heur_thr, angular, args.device)
    ev_val = evaluate(val, params, net_thr, heur_thr, angular, args.device)
    ev_held = evaluate(held, params, net_thr, heur_thr, angular, args.device)
    summary = dict(cases=[c["case"] for c in cases], generation_s=gen_s, training_s=train_s, steps=args.steps,
                   loss_first=float(np.mean(curve[:50])), loss_last=float(np.mean(curve[-50:])),
                   network_logit_threshold=net_thr, heuristic_z_threshold=heur_thr, train=ev_train, validation=ev_val,
                   held_out=ev_held,
                   n_params=int(len(params)))
    np.savez(args.out, params=params, network_logit_threshold=net_thr, heuristic_z_threshold=heur_thr,
             loss_curve=curve.astype(np.float32))
    text = json.dumps(summary, indent=1, default=float)
    if args.summary:
        with open(args.summary, "w") as f:
            f.write(text)
    print(text)


if __name__ == "__main__":
    main()
