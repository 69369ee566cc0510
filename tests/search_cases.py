"""Seeded search cases shared by the parity tests and smoke(): synthetic
template + micrograph prepared by the oracle's restatement of the reference
preparation (template FFT + quadrant swap, whitening, CTF x whitening filter)."""
import numpy as np

from cistem_downstream_bah_b200 import synthetic
from oracle import oracle as O

HIST_BINS = 512
HIST_MIN, HIST_MAX = -12.5, 22.5   # match_template.cpp:45-47


def histogram_scaled(X, Y):
    sq = np.sqrt(float(X * Y))
    step = (HIST_MAX - HIST_MIN) / HIST_BINS
    return HIST_MIN / sq, step / sq


def make_case(T=32, X=256, Y=256, pixel_size=2.0, n_particles=3, snr=0.5, defocus=8000.0, angular_step=30.0,
              psi_step=30.0, seed=7, n_orient=None):
    vol = synthetic.template_volume(T, pixel_size, n_atoms=600, radius_A=T * pixel_size * 0.3, seed=seed)
    mic, truth = synthetic.micrograph(Y, X, pixel_size, n_atoms=600, radius_A=T * pixel_size * 0.3,
                                      n_particles=n_particles, snr=snr, defocus_A=defocus, seed=seed + 1, atom_seed=seed)
    tspec = O.prepare_template(vol.astype(np.float64))
    ispec, curve = O.whiten_image(mic.astype(np.float64))
    filt = O.projection_filter(T, curve, kv=300.0, cs_mm=2.7, amplitude_contrast=0.07, defocus1=defocus,
                               defocus2=defocus, pixel_size=pixel_size)
    grid = O.search_grid(angular_step)
    psis = O.psi_list(0.0, psi_step, 360.0)
    ang = O.orientation_list(grid, psis)
    if n_orient is not None:
        ang = ang[:n_orient]
    hmin, hstep = histogram_scaled(X, Y)
    return dict(T=T, X=X, Y=Y, tspec=tspec, ispec=ispec, curve=curve, filt=filt, angles=ang, hmin=hmin, hstep=hstep,
                pixel_size=pixel_size, defocus=defocus, truth=truth, micrograph=mic, volume=vol)
