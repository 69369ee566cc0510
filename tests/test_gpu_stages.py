"""Kernel-level parity: each intermediate of one orientation against an
independent numpy computation of the same stage (needs a B200).

Stages (tm_debug_stage_buffers): filtered slice after the inverse FFT along
y; real projection; (edge mean, 1/sigma); row spectra of the normalised
projection; correlation spectrum after the inverse FFT along y.  Tolerance:
2e-5 of each stage's largest magnitude (FP32 kernels vs FP64 references).
"""
import numpy as np
import pytest

from cistem_downstream_bah_b200 import core
from oracle import oracle as O
from tests.search_cases import make_case

pytestmark = pytest.mark.gpu


def _stage_refs(case, o):
    T, X, Y = case["T"], case["X"], case["Y"]
    phi, theta, psi = case["angles"][o]
    sl = O.extract_slice(case["tspec"], O.euler_matrix(phi, theta, psi))
    ky = np.where(np.arange(T) >= T // 2, np.arange(T) - T, np.arange(T))
    sign = np.where(((ky[:, None] + np.arange(T // 2 + 1)[None, :]) & 1) == 1, -1.0, 1.0)
    sl = sl * case["filt"] * sign
    s_col = np.fft.ifft(sl, axis=0) * T
    proj = O.irfft2(sl, T)
    edge = np.concatenate([proj[0], proj[-1], proj[1:-1, 0], proj[1:-1, -1]])
    e = np.float32(edge.mean())
    p = proj - e
    n, N = T * T, X * Y
    var = (p * p).mean() * n / N - (p.mean() * n / N) ** 2
    q = p / np.sqrt(var)
    rows = np.fft.rfft(q, n=X, axis=1)
    F = np.fft.fft(rows, n=Y, axis=0)
    kx = np.arange(X // 2 + 1)
    x0, y0 = X // 2 - T // 2, Y // 2 - T // 2
    ph = np.exp(2j * np.pi * ((kx * x0) % X)[None, :] / X) * np.exp(2j * np.pi * ((np.arange(Y) * y0) % Y)[:, None] / Y)
    Ip = case["ispec"] * ph / N
    Ip[0, 0] = 0
    cols = np.fft.ifft(Ip * np.conj(F), axis=0) * Y
    return dict(slice=s_col, projection=proj, normalisation=np.array([e, 1 / np.sqrt(var)]), rows=rows, columns=cols)


@pytest.mark.parametrize("geom", [(32, 256, 256), (32, 512, 256), (64, 1024, 1024)])
def test_stage_buffers(geom):
    T, X, Y = geom
    case = make_case(T=T, X=X, Y=Y, n_orient=30)
    with core.SearchCore(X, Y, T, histogram_min_scaled=case["hmin"], histogram_step_scaled=case["hstep"]) as sc:
        sc.set_template(case["tspec"])
        sc.set_image(case["ispec"])
        for o in (3, 17):
            got = sc.stage_buffers(case["filt"], case["angles"][o])
            ref = _stage_refs(case, o)
            for k in ("slice", "projection", "rows", "columns"):
                err = np.abs(got[k] - ref[k]).max() / np.abs(ref[k]).max()
                assert err < 2e-5, (geom, o, k, err)
            assert abs(got["normalisation"][0] - ref["normalisation"][0]) <= 1e-5 * np.abs(ref["projection"]).max()
            assert abs(got["normalisation"][1] / ref["normalisation"][1] - 1) < 1e-5
