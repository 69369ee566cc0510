"""Timed CPU baseline: the reference's CPU inner loop in FP32 on pocketfft.

TEST AND BASELINE INFRASTRUCTURE.  Only bench.py's CPU legs (the `cpu_baseline`
object and `--impl reference`) and tests/ use this module; nothing in the
library imports it.

The reference's CPU path (match_template.cpp:1004-1149) runs, per orientation,
ExtractSlice, the filter, a backward FFT of the T x T slice, the
normalisation, ClipIntoLargerRealSpace2D, a forward X x Y FFT (FFTW, single
precision), the conjugate multiply with the whitened micrograph spectrum, the
backward X x Y FFT and the per-pixel MIP / sum / sum-of-squares / histogram
update, one orientation after another in each worker.  The two X x Y
transforms are almost all of the work.  This restatement keeps that loop and
its order, and does the two large transforms with pocketfft (scipy.fft,
float32, one transform per worker thread), a library comparable in speed to
FFTW for these sizes; the slice, filter and normalisation of the small T x T
projection come from the C oracle (oracle/tm_oracle.c, FP32 build).  Workers
are host threads over contiguous orientation ranges, as the reference runs
one orientation range per process; their results are merged in orientation
order.  tests/test_cpu_port.py checks it against the FP64 oracle.
"""
import threading

import numpy as np
import scipy.fft as sfft

from oracle import oracle as O


def _worker(tspec, ispec_c64, filt, angles, o0, o1, X, Y, hist_min, hist_step, bins, out):
    T = tspec.shape[0]
    x0, y0 = X // 2 - T // 2, Y // 2 - T // 2
    mip = np.full((Y, X), -np.finfo(np.float32).max, np.float32)
    best = np.full((Y, X), -1, np.int32)
    s = np.zeros((Y, X), np.float64)
    q = np.zeros((Y, X), np.float64)
    hist = np.zeros(bins + 1, np.int64)
    padded = np.zeros((Y, X), np.float32)
    rows = 256   # the per-pixel update runs over blocks of rows (bounded temporaries)
    for o in range(o0, o1):
        # slice, filter, backward FFT, normalisation (the C oracle, FP32)
        proj = O.normalised_projection(tspec, filt, angles, o, X, Y, bits=32)
        padded[y0:y0 + T, x0:x0 + T] = proj
        # ForwardFFT scaled by 1/N, ZeroCentralPixel, conj(P) I, unscaled BackwardFFT
        spec = sfft.rfft2(padded, norm="forward", workers=1)
        spec[0, 0] = 0
        np.conjugate(spec, out=spec)
        spec *= ispec_c64
        cc = sfft.irfft2(spec, s=(Y, X), norm="forward", workers=1)
        for r0 in range(0, Y, rows):
            c = cc[r0:r0 + rows]
            m = mip[r0:r0 + rows]
            upd = c > m
            np.copyto(m, c, where=upd)
            best[r0:r0 + rows][upd] = o
            cd = c.astype(np.float64)
            s[r0:r0 + rows] += cd
            q[r0:r0 + rows] += cd * cd
            b = ((cd - hist_min) / hist_step).astype(np.int64)
            hist += np.bincount(b[(b >= 0) & (b <= bins)], minlength=bins + 1)
    out.update(mip=mip, best=best, sum=s, sumsq=q, hist=hist)


def search(tspec, ispec, filt, angles, X, Y, *, hist_min_scaled, hist_step_scaled, hist_bins=512, threads=1):
    """The plane search over `angles` on `threads` host threads (contiguous
    orientation ranges, merged in order: strict > keeps the first maximum).
    Returns mip (float32), best (orientation index, int32), sum and sum of
    squares (float64), each Y x X, and the histogram (hist_bins + 1 counts,
    the last one the reference's out-of-range bin)."""
    n = len(angles)
    threads = max(1, min(threads, n))
    tspec = np.ascontiguousarray(tspec, np.complex64)
    ispec_c64 = np.ascontiguousarray(np.asarray(ispec).reshape(Y, X // 2 + 1), np.complex64)
    filt = np.ascontiguousarray(filt, np.float32)
    angles = np.ascontiguousarray(angles, np.float32)
    outs = [dict() for _ in range(threads)]
    ranges = [(n * k // threads, n * (k + 1) // threads) for k in range(threads)]
    ws = [threading.Thread(target=_worker, args=(tspec, ispec_c64, filt, angles, o0, o1, X, Y, hist_min_scaled,
                                                 hist_step_scaled, hist_bins, outs[k]))
          for k, (o0, o1) in enumerate(ranges)]
    for w in ws:
        w.start()
    for w in ws:
        w.join()
    res = dict(outs[0])
    for r in outs[1:]:
        upd = r["mip"] > res["mip"]
        res["mip"] = np.where(upd, r["mip"], res["mip"])
        res["best"] = np.where(upd, r["best"], res["best"])
        res["sum"] = res["sum"] + r["sum"]
        res["sumsq"] = res["sumsq"] + r["sumsq"]
        res["hist"] = res["hist"] + r["hist"]
    return res
