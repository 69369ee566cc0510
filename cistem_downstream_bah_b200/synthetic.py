"""Seeded synthetic inputs for the search (no public dataset is involved).

Templates are sums of isotropic 3-D Gaussian atoms (unit weight, sigma in
Angstrom) drawn uniformly in a ball; micrographs hold exact projections of
the rotated template (the line integral of a 3-D Gaussian is a 2-D Gaussian),
multiplied by a CTF in Fourier space and overlaid with white Gaussian noise
at a stated per-particle SNR.  Atom centres are splatted with linear weights
and the Gaussian profile is applied in Fourier space, which keeps generation
fast at 4096^2.
"""
from __future__ import annotations

import numpy as np


def _random_rotations(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    R = np.empty((n, 3, 3))
    R[:, 0, 0] = 1 - 2 * (y * y + z * z); R[:, 0, 1] = 2 * (x * y - z * w); R[:, 0, 2] = 2 * (x * z + y * w)
    R[:, 1, 0] = 2 * (x * y + z * w); R[:, 1, 1] = 1 - 2 * (x * x + z * z); R[:, 1, 2] = 2 * (y * z - x * w)
    R[:, 2, 0] = 2 * (x * z - y * w); R[:, 2, 1] = 2 * (y * z + x * w); R[:, 2, 2] = 1 - 2 * (x * x + y * y)
    return R


def atoms_in_ball(rng, n_atoms, radius):
    d = rng.standard_normal((n_atoms, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = radius * rng.random(n_atoms) ** (1.0 / 3.0)
    return d * r[:, None]


def _gauss_ft(shape, sigma_px):
    ks = [np.fft.fftfreq(n) for n in shape[:-1]] + [np.fft.rfftfreq(shape[-1])]
    g = np.ones([len(k) for k in ks])
    for ax, k in enumerate(ks):
        sh = [1] * len(ks)
        sh[ax] = len(k)
        g = g * np.exp(-2.0 * (np.pi * sigma_px * k.reshape(sh)) ** 2)
    return g


def template_volume(box, pixel_size, n_atoms, radius_A, sigma_A=1.5, seed=0):
    """Gaussian-atom template volume (box^3, float32, zero edge mean)."""
    rng = np.random.default_rng(seed)
    xyz = atoms_in_ball(rng, n_atoms, radius_A) / pixel_size + box / 2
    vol = np.zeros((box, box, box))
    base = np.floor(xyz).astype(np.int64)
    frac = xyz - base
    for dz in (0, 1):
        for dy in (0, 1):
            for dx in (0, 1):
                w = (frac[:, 0] if dx else 1 - frac[:, 0]) * (frac[:, 1] if dy else 1 - frac[:, 1]) * \
                    (frac[:, 2] if dz else 1 - frac[:, 2])
                ix, iy, iz = base[:, 0] + dx, base[:, 1] + dy, base[:, 2] + dz
                ok = (ix >= 0) & (ix < box) & (iy >= 0) & (iy < box) & (iz >= 0) & (iz < box)
                np.add.at(vol, (iz[ok], iy[ok], ix[ok]), w[ok])
    vol = np.fft.irfftn(np.fft.rfftn(vol) * _gauss_ft(vol.shape, sigma_A / pixel_size), s=vol.shape, axes=(0, 1, 2))
    edge = np.concatenate([vol[0].ravel(), vol[-1].ravel(), vol[:, 0].ravel(), vol[:, -1].ravel(),
                           vol[:, :, 0].ravel(), vol[:, :, -1].ravel()])
    return (vol - edge.mean()).astype(np.float32)


def ctf_2d(ny, nx, pixel_size, defocus_A, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07):
    """CTF on the rfft2 grid, same formula as the search's projection filter."""
    lam = 12.2639 / np.sqrt(1000.0 * kv + 0.97845e-6 * (1000.0 * kv) ** 2)
    ky = np.fft.fftfreq(ny)[:, None] / pixel_size
    kx = np.fft.rfftfreq(nx)[None, :] / pixel_size
    g2 = kx * kx + ky * ky
    cs = cs_mm * 1e7
    w = np.arctan(amplitude_contrast / np.sqrt(1 - amplitude_contrast ** 2))
    chi = np.pi * lam * g2 * (defocus_A - 0.5 * lam * lam * g2 * cs) + w
    return -np.sin(chi)


def micrograph(ny, nx, pixel_size, n_atoms, radius_A, n_particles, snr, defocus_A, sigma_A=1.5, seed=0,
               atom_seed=None):
    """Synthetic micrograph and ground truth (positions in pixels, rotation matrices)."""
    rng = np.random.default_rng(seed)
    atoms = atoms_in_ball(np.random.default_rng(seed if atom_seed is None else atom_seed), n_atoms, radius_A) / pixel_size
    diam = 2 * radius_A / pixel_size
    positions = []
    tries = 0
    while len(positions) < n_particles and tries < 100000:
        tries += 1
        p = np.array([rng.uniform(diam / 2, nx - diam / 2), rng.uniform(diam / 2, ny - diam / 2)])
        if all(np.hypot(*(p - q)) >= diam for q in positions):
            positions.append(p)
    positions = np.array(positions).reshape(-1, 2)
    rots = _random_rotations(rng, len(positions))
    img = np.zeros((ny, nx))
    for p, R in zip(positions, rots):
        xy = (atoms @ R.T)[:, :2] + p
        base = np.floor(xy).astype(np.int64)
        f = xy - base
        for dy in (0, 1):
            for dx in (0, 1):
                w = (f[:, 0] if dx else 1 - f[:, 0]) * (f[:, 1] if dy else 1 - f[:, 1])
                ix, iy = base[:, 0] + dx, base[:, 1] + dy
                ok = (ix >= 0) & (ix < nx) & (iy >= 0) & (iy < ny)
                np.add.at(img, (iy[ok], ix[ok]), w[ok])
    spec = np.fft.rfft2(img) * _gauss_ft(img.shape, sigma_A / pixel_size) * ctf_2d(ny, nx, pixel_size, defocus_A)
    signal = np.fft.irfft2(spec, s=img.shape)
    # per-particle SNR = variance of the signal within the particle footprints / noise variance
    yy, xx = np.mgrid[0:ny, 0:nx]
    mask = np.zeros((ny, nx), bool)
    r = radius_A / pixel_size
    for p in positions:
        x0, x1 = int(max(0, p[0] - r)), int(min(nx, p[0] + r + 1))
        y0, y1 = int(max(0, p[1] - r)), int(min(ny, p[1] + r + 1))
        sub = (xx[y0:y1, x0:x1] - p[0]) ** 2 + (yy[y0:y1, x0:x1] - p[1]) ** 2 <= r * r
        mask[y0:y1, x0:x1] |= sub
    var_sig = signal[mask].var() if mask.any() else signal.var()
    sigma_n = np.sqrt(var_sig / snr) if snr > 0 else 0.0
    out = signal + rng.standard_normal(signal.shape) * sigma_n
    return out.astype(np.float32), {"positions": positions, "rotations": rots, "noise_sigma": sigma_n}
