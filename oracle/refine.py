"""CPU restatement of refine_template (test infrastructure only).

Restates src/programs/refine_template/refine_template.cpp on the oracle's FP64
primitives (oracle.py): TemplateScore (:24-80) with Image::ChangePixelSize
(src/core/image.cpp:8705-8822) written out as its literal chain of
transforms, the whitening (:612-630), the peak picking (:503-553), the
particle windows (:717-724, RealSpaceIntegerShift image.cpp:9064-9110) and
the coordinate descent (:636-1130) as plain Python loops.  Only the tests
import this module; the product never does.
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as O

f32 = np.float32
FLT_MAX = float(np.finfo(np.float32).max)


def fourier_sum_of_squares(spec, nx):
    """Image::ReturnSumOfSquares in Fourier space, 2-D (image.cpp:300-313)."""
    ny = spec.shape[0]
    p = np.abs(spec.astype(np.complex128)) ** 2
    w = np.ones(p.shape)
    x_even = nx % 2 == 0
    ub_x = nx // 2
    lb_y = -(ny // 2) if ny % 2 == 0 else -((ny - 1) // 2)
    for j in range(ny):
        jj = j if j < (ny // 2 + (ny % 2)) else j - ny
        for i in (0, ub_x):
            if not (i == 0 or (i == ub_x and x_even)):
                continue
            if jj == 0 or (jj == lb_y and x_even):
                w[j, i] = 0.5
            elif jj < 0:
                w[j, i] = 0.0
    return 2.0 * float((p * w).sum())


def average_in_disc(img, radius):
    ny, nx = img.shape
    r2 = f32(radius) * f32(radius) if radius > 0 else None
    if r2 is None:
        return f32(img.astype(np.float64).mean())
    x = (np.arange(nx) - nx // 2).astype(f32) ** 2
    y = (np.arange(ny) - ny // 2).astype(f32) ** 2
    m = (y[:, None] + x[None, :]).astype(f32) <= r2
    return f32(img[m].astype(np.float64).sum() / m.sum())


def change_pixel_size_fft(img, nout, factor, tolerance=0.001):
    """ChangePixelSize(other (nout x nout), factor, tolerance, return_fft=True)
    of a real square image: the half spectrum of the result, scaled 1/N as
    ForwardFFT leaves it."""
    nin = img.shape[0]
    factor = f32(factor)
    tol = f32(tolerance)
    if abs(float(f32(factor - f32(1.0)))) < float(tol):
        clipped = O.clip_into_real(img, nout, nout, 0.0)
        return O.rfft2(clipped) / (nout * nout)
    old = nin
    min_dim = nin
    if tol < f32(1.0) / f32(f32(min_dim) * factor):
        inter = f32(f32(1.0) / f32(tol * f32(min_dim)))
        pad = int(f32(f32(old) * inter))
        if (old % 2 == 0) != (pad % 2 == 0):
            pad += 1
        new = int(f32(f32(pad) / factor))
        if (old % 2 == 0) != (new % 2 == 0):
            new += 1
    else:
        pad = int(f32(f32(old) * factor))
        if (old % 2 == 0) != (pad % 2 == 0):
            pad += 1
        new = old
    pv = 0.0
    if pad > old:
        pv = float(average_in_disc(img, f32(0.45) * f32(min_dim)))
    big = O.clip_into_real(img, pad, pad, pv)
    spec = O.rfft2(big) / (pad * pad)
    spec = O.clip_into_fourier(spec, pad, new, new, 0.0)
    if new == nout:
        return spec
    back = O.irfft2(spec, new)
    out = O.clip_into_real(back, nout, nout, pv)
    return O.rfft2(out) / (nout * nout)


def template_score(template_spec, T, phi, theta, psi, filt, particle_spec, factor=1.0):
    """TemplateScore (refine_template.cpp:24-80): (value, x, y)."""
    TP = template_spec.shape[0]
    sl = O.extract_slice(template_spec, O.euler_matrix(phi, theta, psi))
    sl = O.swap_quadrants(sl, TP)
    proj = O.irfft2(sl, TP)
    spec = change_pixel_size_fft(proj, T, factor)
    spec = spec * filt
    spec[0, 0] = 0
    spec = spec / math.sqrt(fourier_sum_of_squares(spec, T))
    z = np.conj(spec) * particle_spec
    cc = O.irfft2(z, T)
    px, py, v = O.find_peak_integer(cc)
    return float(v), float(px), float(py)


def refine_whiten(image):
    """refine_template.cpp:612-630: as match_template's whitening without the
    quadrant swap, then BackwardFFT (even sizes: the swap is (-1)^(x+y))."""
    ny, nx = image.shape
    assert nx % 2 == 0 and ny % 2 == 0
    spec, curve = O.whiten_image(image.astype(np.float64))
    sign = np.where((np.arange(ny)[:, None] + np.arange(nx // 2 + 1)[None, :]) % 2 == 0, 1.0, -1.0)
    return O.irfft2(spec * sign, nx), curve


def window_particle(img, peak_x, peak_y, T):
    ny, nx = img.shape
    n = nx * ny
    shifted = -int(peak_x) - nx * int(peak_y)
    shifted = int(math.remainder(float(f32(shifted)), float(f32(n))))
    if shifted < 0:
        shifted += n
    flat = img.reshape(-1)
    out = np.zeros((T, T), np.float64)
    for jj in range(T):
        j = ny // 2 + (jj - T // 2)
        for ii in range(T):
            i = nx // 2 + (ii - T // 2)
            if 0 <= i < nx and 0 <= j < ny:
                out[jj, ii] = flat[((j * nx + i) - shifted) % n]
    return out


def particle_spectrum(window):
    T = window.shape[0]
    return O.swap_quadrants(O.rfft2(window) / (T * T), T)


def find_peaks(scaled_mip, threshold, min_peak_radius):
    z = scaled_mip.astype(np.float32).copy()
    ny, nx = z.shape
    out = []
    cap = nx * ny // 100
    jj, ii = np.mgrid[0:ny, 0:nx]
    while True:
        sub = z[50:min(ny - 50 + 1, ny), 50:min(nx - 50 + 1, nx)]
        k = int(np.argmax(sub))
        by, bx = divmod(k, sub.shape[1])
        best = float(sub[by, bx])
        by += 50
        bx += 50
        if best < threshold or len(out) >= cap:
            break
        out.append((bx - nx // 2, by - ny // 2, best))
        d = ((jj - by).astype(np.float64) ** 2).astype(np.float32) + ((ii - bx).astype(np.float64) ** 2).astype(np.float32)
        z[d <= f32(min_peak_radius)] = -FLT_MAX
    return out


def _round(a):
    a = float(f32(a))
    return int(a + 0.5) if a > 0 else int(a - 0.5)


class _Local:
    """A worker's copies of the parameter maps, FFTW-padded addressing."""

    def __init__(self, maps, pitch):
        self.maps, self.pitch, self.over = maps, pitch, [dict() for _ in range(5)]
        self.keys = ("psi", "theta", "phi", "defocus", "pixel_size")

    def read(self, name, addr):
        ny, nx = self.maps[name].shape
        if addr < 0:
            return f32(0)
        y, x = divmod(addr, self.pitch)
        if y >= ny or x >= nx:
            return f32(0)
        return f32(self.maps[name][y, x])

    def get(self, which, addr):
        return self.over[which].get(addr, self.read(self.keys[which], addr))

    def set(self, which, addr, v):
        self.over[which][addr] = f32(v)


def refine(maps, peaks, prm, T, score, log=None):
    """The descent of refine_template.cpp:636-1130 with one worker (the
    reference's single-thread order).  maps: dict of compact images; peaks:
    (x, y) relative to the centre; prm: dict of the parameters; score(c) ->
    (value, x, y) for c = (phi, theta, psi, defocus1, defocus2, factor, k)."""
    ny, nx = maps["psi"].shape
    pitch = nx + (2 if nx % 2 == 0 else 1)
    pixel_size = f32(prm["pixel_size"])
    defocus_search_range = f32(prm["defocus_search_range"])
    defocus_refine_step = f32(f32(2.0) * f32(prm["defocus_search_step"]))
    pixel_size_search_range = f32(prm["pixel_size_search_range"])
    pixel_size_refine_step = f32(f32(2.0) * f32(prm["pixel_size_search_step"]))
    if defocus_refine_step <= 0:
        defocus_search_range, defocus_refine_step = f32(0), f32(100)
    if pixel_size_refine_step <= 0:
        pixel_size_search_range, pixel_size_refine_step = f32(0), f32(100)
    defocus_step = max(defocus_refine_step, f32(100))
    ang, ipa = f32(prm["angular_step"]), f32(prm["in_plane_angular_step"])
    d1, d2 = f32(prm["defocus1"]), f32(prm["defocus2"])
    box = f32(math.sqrt(float(f32(T * T))))
    out = {k: (np.zeros_like(maps[k]) if k in ("mip", "scaled_mip") else maps[k].astype(np.float32).copy())
           for k in ("mip", "scaled_mip", "psi", "theta", "phi", "defocus", "pixel_size")}
    local = _Local(maps, pitch)
    rows = []
    for k, (fx, fy) in enumerate(peaks):
        memo = {}

        def ev(c):
            key = tuple(np.float32(v).tobytes() for v in c[:6])
            if key not in memo:
                memo[key] = score(c)
                if log is not None:
                    log.append(c)
            return memo[key]

        px, py = int(f32(fx) + f32(nx // 2)), int(f32(fy) + f32(ny // 2))
        cur = py * pitch + px
        st = dict(phi=local.get(2, cur), theta=local.get(1, cur), psi=local.get(0, cur), defocus=local.get(3, cur),
                  pixel=local.get(4, cur))
        sc_here, mip_here = f32(maps["scaled_mip"][py, px]), f32(maps["mip"][py, px])
        best = dict(score=f32(-FLT_MAX), peak=(0.0, 0.0, 0.0), addr=cur, off=f32(0))
        cand = dict(phi=st["phi"], theta=st["theta"], psi=st["psi"], df1=f32(d1 + st["defocus"]),
                    df2=f32(d2 + st["defocus"]), factor=f32(1.0))

        def c_now():
            return (cand["phi"], cand["theta"], cand["psi"], cand["df1"], cand["df2"], cand["factor"], k)

        def improve(s):
            best["peak"] = s
            best["score"] = f32(s[0])
            best["addr"] = cur + pitch * _round(s[2]) + _round(s[1])
            best["off"] = f32(math.sqrt(float(f32(f32(s[1]) ** 2 + f32(s[2]) ** 2))))

        start = ev(c_now())
        starting = f32(f32(start[0]) * box)
        starting = f32(f32(f32(f32(1.0) * sc_here) * starting) / mip_here)
        if defocus_search_range != 0:
            nd = _round(f32(defocus_search_range / defocus_step))
            for dis in range(-nd, nd + 1):
                off = f32(f32(dis) * defocus_step)
                cand["df1"], cand["df2"] = f32(f32(d1 + st["defocus"]) + off), f32(f32(d2 + st["defocus"]) + off)
                s = ev(c_now())
                if f32(s[0]) > best["score"]:
                    improve(s)
                    local.set(3, best["addr"], f32(st["defocus"] + off))
            st["defocus"] = local.get(3, best["addr"])
        idx = dict(phi=0, theta=0, psi=0)

        def descent(on_improve):
            for kk in (0, 1, -1):
                while True:
                    bphi = best["score"]
                    idx["phi"] += kk
                    for jj in (0, 1, -1):
                        while True:
                            bth = best["score"]
                            idx["theta"] += jj
                            for ii in (0, 1, -1):
                                while True:
                                    bpsi = best["score"]
                                    idx["psi"] += ii
                                    cand["phi"] = f32(st["phi"] + f32(f32(idx["phi"]) * ang))
                                    cand["theta"] = f32(st["theta"] + f32(f32(idx["theta"]) * ang))
                                    cand["psi"] = f32(st["psi"] + f32(f32(idx["psi"]) * ipa))
                                    s = ev(c_now())
                                    if f32(s[0]) > best["score"]:
                                        improve(s)
                                        local.set(0, best["addr"], cand["psi"])
                                        local.set(1, best["addr"], cand["theta"])
                                        local.set(2, best["addr"], cand["phi"])
                                        on_improve()
                                    if not best["score"] > bpsi:
                                        break
                                idx["psi"] -= ii
                            if not best["score"] > bth:
                                break
                        idx["theta"] -= jj
                    if not best["score"] > bphi:
                        break
                idx["phi"] -= kk

        di = [0]
        mult = f32(defocus_step / defocus_refine_step)
        while mult > f32(0.5):
            for ll in (0, 1, -1):
                if ll != 0 and defocus_refine_step == 0:
                    break
                while True:
                    bdf = best["score"]
                    if defocus_search_range != 0:
                        di[0] += _round(f32(mult * f32(ll)))
                    off = f32(f32(di[0]) * defocus_refine_step)
                    cand["df1"], cand["df2"] = f32(f32(d1 + st["defocus"]) + off), f32(f32(d2 + st["defocus"]) + off)

                    def on_df():
                        local.set(3, best["addr"], f32(st["defocus"] + f32(f32(di[0]) * defocus_refine_step)))
                        local.set(4, best["addr"], st["pixel"])
                    descent(on_df)
                    if not best["score"] > bdf:
                        break
                if defocus_search_range != 0:
                    di[0] -= ll
            mult = f32(mult / f32(2.0))
        for name, w in (("phi", 2), ("theta", 1), ("psi", 0), ("defocus", 3), ("pixel", 4)):
            st[name] = local.get(w, best["addr"])
        idx.update(phi=0, theta=0, psi=0)
        cand["df1"], cand["df2"] = f32(d1 + st["defocus"]), f32(d2 + st["defocus"])
        cand["phi"], cand["theta"], cand["psi"] = st["phi"], st["theta"], st["psi"]
        if pixel_size_search_range != 0:
            ns = _round(f32(pixel_size_search_range / pixel_size_refine_step))
            for sis in range(-ns, ns + 1):
                cand["factor"] = f32(f32(f32(pixel_size + st["pixel"]) + f32(f32(sis) * pixel_size_refine_step)) / pixel_size)
                s = ev(c_now())
                if f32(s[0]) > best["score"]:
                    improve(s)
                    local.set(4, best["addr"], f32(st["pixel"] + f32(f32(sis) * pixel_size_refine_step)))
            st["pixel"] = local.get(4, best["addr"])
        idx.update(phi=0, theta=0, psi=0)
        si = [0]
        mult = f32(1.0)
        while mult > f32(0.5):
            for ll in (0, 1, -1):
                if ll != 0 and pixel_size_refine_step == 0:
                    break
                while True:
                    bps = best["score"]
                    if pixel_size_search_range != 0:
                        si[0] += _round(f32(mult * f32(ll)))
                    cand["factor"] = f32(f32(f32(pixel_size + st["pixel"]) + f32(f32(si[0]) * pixel_size_refine_step)) / pixel_size)

                    def on_px():
                        local.set(3, best["addr"], st["defocus"])
                        local.set(4, best["addr"], f32(st["pixel"] + f32(f32(si[0]) * pixel_size_refine_step)))
                    descent(on_px)
                    if not best["score"] > bps:
                        break
                if pixel_size_search_range != 0:
                    si[0] -= ll
            mult = f32(mult / f32(2.0))
        bs = best["score"]
        best_scaled = f32(f32(f32(f32(f32(1.0) * sc_here) * bs) / mip_here) * box)
        best_mip = f32(f32(f32(1.0) * bs) * box)
        a = best["addr"]
        vals = [local.get(w, a) for w in (0, 1, 2, 3, 4)]   # psi theta phi defocus pixel
        bx_, by_ = best["peak"][1], best["peak"][2]
        rows.append([f32(f32(fx) + f32(bx_)), f32(f32(fy) + f32(by_)), *vals, best_scaled,
                     f32(f32(bx_) * pixel_size), f32(f32(by_) * pixel_size),
                     f32(vals[0] - local.read("psi", cur)), f32(vals[1] - local.read("theta", cur)),
                     f32(vals[2] - local.read("phi", cur)), f32(vals[3] - local.read("defocus", cur)),
                     f32(vals[4] - local.read("pixel_size", cur)), f32(best_scaled - starting)])
        y, x = divmod(a, pitch)
        if a >= 0 and y < ny and x < nx and (f32(best["off"] * pixel_size) <= f32(prm["xy_change_threshold"])
                                             or not prm["exclude_above_xy_threshold"]):
            out["scaled_mip"][y, x] = best_scaled
            out["mip"][y, x] = best_mip
            for name, v in zip(("psi", "theta", "phi", "defocus", "pixel_size"), vals):
                out[name][y, x] = v
    return out, np.array(rows, np.float32).reshape(-1, 16)
