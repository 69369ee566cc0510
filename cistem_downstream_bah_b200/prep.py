"""Host-side preparation of the search inputs (vectorised numpy).

This is the caller's side of the search core, as match_template's
DoCalculation is in the reference: whitening of the micrograph
(match_template.cpp:703-724), the template spectrum (:842-845), the projection
filter per defocus plane (:895-898), the search grid (:662-697), the
micrograph-size factorisation (:527-596) and the final statistics
(:1176-1370).  Numerics follow the reference CPU path; array layouts are
compact (no FFTW row padding): real images (ny, nx), half spectra
(ny, nx//2+1).
"""
from __future__ import annotations

import numpy as np

HISTOGRAM_BINS = 512
HISTOGRAM_MIN = -12.5
HISTOGRAM_MAX = 22.5
CIS_PIF = np.float32(3.14159265359)


def _logical(n):
    """Logical Fourier coordinate of each physical index (image.cpp:6899-6909)."""
    i = np.arange(n)
    first_neg = n // 2 if n % 2 == 0 else n // 2 + 1
    return np.where(i >= first_neg, i - n, i)


def histogram_scaled(nx, ny):
    """histogram_min_scaled / histogram_step_scaled (match_template.cpp:633-637)."""
    sq = np.sqrt(float(nx * ny))
    step = np.float32((HISTOGRAM_MAX - HISTOGRAM_MIN) / np.float32(HISTOGRAM_BINS))
    return HISTOGRAM_MIN / sq, float(step) / sq


def whitening_curve_points(nx):
    return int((nx / 2.0 + 1.0) * float(np.sqrt(np.float32(2.0))) + 1.0)


def _curve_axis(npts):
    hi = np.float32(0.5) * np.sqrt(np.float32(2.0))
    i = np.arange(npts, dtype=np.float32)
    return (i * (hi - np.float32(0.0)) / np.float32(npts - 1) + np.float32(0.0)).astype(np.float32)


def _curve_interp(xaxis, y, f):
    """Curve::ReturnLinearInterpolationFromX (curve.cpp:377-397) for many x."""
    n = len(xaxis)
    idx = np.searchsorted(xaxis, f, side="right") - 1
    idx = np.clip(idx, 0, n - 1)
    last = idx >= n - 1
    i0 = np.minimum(idx, n - 2)
    d = (f - xaxis[i0]) / (xaxis[i0 + 1] - xaxis[i0])
    v = y[i0] * (1.0 - d) + y[i0 + 1] * d
    return np.where(last, y[n - 1], v)


def whiten(image):
    """Whitened, unit-norm half spectrum and the whitening curve of a real
    micrograph (match_template.cpp:711-724)."""
    img = np.array(image, dtype=np.float64)
    ny, nx = img.shape
    n = img.size
    # ReplaceOutliersWithMean(5) (image.cpp:986-1007)
    mean = np.float32(img.mean())
    sigma = np.sqrt(np.float32(abs(np.float32((img * img).mean() - img.mean() ** 2))))
    vmax, vmin = mean + np.float32(5.0) * sigma, mean - np.float32(5.0) * sigma
    img = np.where((img > vmax) | (img < vmin), float(mean), img)
    spec = np.fft.rfft2(img) / n
    # SwapRealSpaceQuadrants for an object centred in the box
    kx = np.arange(nx // 2 + 1)
    ky = _logical(ny)
    if nx % 2 == 0 and ny % 2 == 0:
        sign = np.where(((ky[:, None] + kx[None, :]) & 1) == 1, -1.0, 1.0)
        spec = spec * sign
    else:
        ph = -2 * np.pi * ((nx // 2) * kx[None, :] / nx + (ny // 2) * ky[:, None] / ny)
        spec = spec * np.exp(1j * ph)
    spec[0, 0] = 0
    # Compute1DPowerSpectrumCurve (image.cpp:7135-7201)
    npts = whitening_curve_points(nx)
    xa = _curve_axis(npts)
    vx = np.float32(1.0 / nx)
    vy = np.float32(1.0 / ny)
    sx = (kx.astype(np.float32) * vx) ** 2
    sy = (ky.astype(np.float32) * vy) ** 2
    f = np.sqrt((sx[None, :] + sy[:, None]).astype(np.float32))
    keep = np.ones(spec.shape, bool)
    keep[ny // 2 if ny % 2 == 0 else ny // 2 + 1:, 0] = False     # explicit Hermitian mates
    fk = f[keep]
    pw = np.abs(spec[keep]) ** 2
    dx = xa[1] - xa[0]
    i0 = ((fk - xa[0]) / dx).astype(np.int64)
    last = i0 >= npts - 1
    i0c = np.minimum(i0, npts - 2)
    d = np.where(last, 0.0, (fk - xa[i0c]) / (xa[i0c + 1] - xa[i0c]))
    acc = np.zeros(npts)
    cnt = np.zeros(npts)
    np.add.at(acc, np.where(last, npts - 1, i0c), pw * (1.0 - d))
    np.add.at(acc, np.where(last, npts - 1, i0c + 1), np.where(last, 0.0, pw * d))
    np.add.at(cnt, np.where(last, npts - 1, i0c), 1.0 - d)
    np.add.at(cnt, np.where(last, npts - 1, i0c + 1), np.where(last, 0.0, d))
    curve = np.where(cnt > 0, acc / np.where(cnt > 0, cnt, 1), 0.0)
    curve = np.sqrt(curve)
    curve = np.where(curve != 0, 1.0 / np.where(curve != 0, curve, 1), 0.0)
    curve = curve * (1.0 / curve.max())
    # ApplyCurveFilter (image.cpp:7284-7310): frequency via double sqrt, cast to float
    fa = np.sqrt(np.float64(kx.astype(np.float32) * vx)[None, :] ** 2 +
                 np.float64(ky.astype(np.float32) * vy)[:, None] ** 2).astype(np.float32)
    spec = spec * _curve_interp(xa, curve, fa)
    spec[0, 0] = 0
    # / sqrt(ReturnSumOfSquares) with the Hermitian weights of image.cpp:307-330
    p = np.abs(spec) ** 2
    w = np.ones(spec.shape)
    edge_x = np.zeros(nx // 2 + 1, bool)
    edge_x[0] = True
    if nx % 2 == 0:
        edge_x[nx // 2] = True
    edge_y = (ky == 0) | ((ky == -(ny // 2)) & (nx % 2 == 0))
    w[np.ix_(edge_y, edge_x)] = 0.5
    neg = ky < 0
    both = np.zeros(spec.shape, bool)
    both[np.ix_(~edge_y & neg, edge_x)] = True
    w[both] = 0.0
    spec = spec / np.sqrt(2.0 * (p * w).sum())
    return spec.astype(np.complex64), curve


def template_spectrum(volume):
    """Quadrant-swapped template spectrum for a pixel-size factor of 1
    (ChangePixelSize + ZeroCentralPixel + SwapRealSpaceQuadrants,
    match_template.cpp:842-845)."""
    vol = np.asarray(volume, dtype=np.float64)
    T = vol.shape[0]
    spec = np.fft.rfftn(vol) / vol.size
    spec[0, 0, 0] = 0
    k = _logical(T)
    i = np.arange(T // 2 + 1)
    if T % 2 == 0:
        par = (k[:, None, None] + k[None, :, None] + i[None, None, :]) & 1
        spec = spec * np.where(par == 1, -1.0, 1.0)
    else:
        c = T // 2
        ph = -2 * np.pi * c * (k[:, None, None] + k[None, :, None] + i[None, None, :]) / T
        spec = spec * np.exp(1j * ph)
    return spec.astype(np.complex64)


def projection_filter(T, curve, *, kv, cs_mm, amplitude_contrast, defocus1, defocus2, astigmatism_angle=0.0,
                      pixel_size, phase_shift_deg=0.0, defocus_offset=0.0):
    """CTF x whitening filter on the T x T half plane (CalculateCTFImage +
    ApplyCurveFilter, match_template.cpp:895-898; ctf.cpp:79-130, 445-561)."""
    f32 = np.float32
    kv, cs_mm, amp = f32(kv), f32(cs_mm), f32(amplitude_contrast)
    px = f32(pixel_size)
    lam = f32(f32(12.2639) / np.sqrt(f32(f32(1000.0) * kv + 0.97845e-6 * (f32(1000.0) * kv) ** 2))) / px
    lam2 = lam * lam
    cs = f32(cs_mm * 10000000.0 / px)
    act = f32(np.pi / 2.0) if abs(amp - 1.0) < 1e-3 else np.arctan(amp / np.sqrt(f32(1.0 - amp * amp)))
    phase = f32(f32(phase_shift_deg) * CIS_PIF / 180.0)
    df1 = f32((f32(defocus1) + f32(defocus_offset)) / px)
    df2 = f32((f32(defocus2) + f32(defocus_offset)) / px)
    az0 = f32(f32(astigmatism_angle) * CIS_PIF / 180.0)
    v = f32(1.0 / T)
    y = (_logical(T).astype(f32) * v)[:, None]
    x = (np.arange(T // 2 + 1).astype(f32) * v)[None, :]
    az = np.arctan2(y, x).astype(f32)
    az[0, 0] = 0
    g2 = (x * x + y * y).astype(f32)
    if df1 == 0 and df2 == 0:
        ctf = np.full(g2.shape, -0.7, f32)
    else:
        df = f32(0.5) * (df1 + df2 + np.cos(f32(2.0) * (az - az0)) * (df1 - df2))
        chi = CIS_PIF * lam * g2 * (df - f32(0.5) * lam2 * g2 * cs) + phase + act
        ctf = -np.sin(chi.astype(f32))
    fa = np.sqrt(np.float64(x) ** 2 + np.float64(y) ** 2).astype(f32)
    xa = _curve_axis(len(curve))
    w = _curve_interp(xa, np.asarray(curve, np.float64), fa)
    out = np.where(fa <= 1.0, ctf * w, 0.0)
    return out.astype(np.float32)


def search_grid(angular_step, symmetry="C1"):
    """(phi, theta) search positions: EulerSearch::InitGrid + C1 theta_max=180 +
    CalculateGridSearchPositions(false) (euler_search.cpp:129-260, match_template.cpp:687-697)."""
    f32 = np.float32
    t = symmetry[0].upper()
    num = int(symmetry[1:]) if len(symmetry) > 1 else 0
    limits = {"C": (360.0 / max(num, 1), 90.0), "D": (360.0 / max(num, 1), 90.0), "T": (180.0, 54.7),
              "O": (90.0, 54.7), "I": (180.0, 31.7)}
    if t not in limits or (t in "CD" and num <= 0):
        raise ValueError(f"bad symmetry {symmetry}")
    phi_max, theta_max = f32(limits[t][0]), f32(limits[t][1])
    if t == "C" and num == 1:
        theta_max = f32(180.0)
    step = f32(angular_step)
    theta_step = f32(theta_max / f32(int(theta_max / step + f32(0.5))))
    out = []
    theta = f32(0.0)
    while float(theta) < float(theta_max) + float(theta_step) / 2.0:
        if theta == 0.0 or theta == 180.0:
            phi_step = phi_max
        else:
            rad = f32(float(f32(theta * CIS_PIF)) / 180.0)
            phi_step = f32(abs(step / np.sin(rad)))
            if phi_step > phi_max:
                phi_step = phi_max
            phi_step = f32(phi_max / f32(int(phi_max / phi_step + f32(0.5))))
        phi = f32(0.0)
        while phi < phi_max:
            out.append((phi, theta))
            phi = f32(phi + phi_step)
        theta = f32(theta + theta_step)
    return np.array(out, dtype=np.float32).reshape(-1, 2)


def factorize_dimension(original, template_size):
    """Padded size of one micrograph dimension (match_template.cpp:539-583)."""
    def small(n, largest):
        for f in range(2, largest + 1):
            if n == 1:
                break
            while n % f == 0:
                n //= f
        return n == 1

    def upper(w, lf):
        n = w + 1 if w % 2 else w
        while n < 10000 * w and not small(n, lf):
            n += 1
        return n

    def lower(w, lf):
        n = w - 1 if w % 2 else w
        while n >= 2 and not small(n, lf):
            n -= 1
        return n

    for p in (2, 3, 5, 7, 9, 13):
        neg, pos = lower(original, p), upper(original, p)
        if np.float32(original - neg) < np.float32(template_size) * np.float32(0.000001):
            return neg
        if np.float32(pos - original) < np.float32(original) * np.float32(0.1):
            return pos
    return original


def finalize(mip, sum_, sumsq, n_total, nx, ny):
    """MIP x sqrt(N), mean, standard deviation and z-score of a local run
    (match_template.cpp:1221-1310)."""
    sq = np.float32(np.sqrt(float(nx * ny)))
    s = np.asarray(sum_, np.float64) / np.float32(n_total)
    var = np.asarray(sumsq, np.float64) / np.float32(n_total) - (s.astype(np.float32).astype(np.float64)) ** 2
    sd = np.where(var > 0, np.sqrt(var.astype(np.float32)).astype(np.float64) * sq, 0.0)
    avg = s * sq
    m = np.asarray(mip, np.float32) * sq
    z = np.where(sd > 0, ((m.astype(np.float64) - avg).astype(np.float32) / sd), 0.0).astype(np.float32)
    return m, z, avg.astype(np.float32), sd.astype(np.float32)
