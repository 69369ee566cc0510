"""tm_run_plane_noalloc against the context entry points (needs a B200).

The allocation-free entry point is for callers that cannot call cudaMalloc
(framework-owned memory pools, plugins given pre-allocated buffers).  Here
the caller's device buffers come from torch, which stands in for such a host
allocator; the test runs two planes in a row through both entry points on
the same inputs, for each compiled geometry, and compares every running
result.  Tolerances are those of the parity tests:
MIP within 1e-4 relative, sums within 1e-5 of their scale, histogram within
0.1% (+2); best orientation and defocus identical on all but 0.1% of pixels
(near-ties can resolve differently because the prepared micrograph spectrum
is built on the device here and on the host in the context path).
"""
import ctypes

import numpy as np
import pytest

from cistem_downstream_bah_b200 import core
from oracle import oracle as O
from tests.search_cases import make_case

pytestmark = pytest.mark.gpu


def _dev(torch, arr, dtype):
    return torch.from_numpy(np.ascontiguousarray(arr).view(dtype)).cuda()


@pytest.mark.parametrize("T,X,Y,step", [(32, 256, 256, 45.0), (32, 512, 512, 60.0), (64, 512, 512, 60.0)])
def test_noalloc_matches_context_entry_points_two_calls(T, X, Y, step):
    torch = pytest.importorskip("torch")
    case = make_case(T=T, X=X, Y=Y, angular_step=step, psi_step=step)
    X, Y, T = case["X"], case["Y"], case["T"]
    ang = case["angles"]
    half = len(ang) // 2
    calls = [(ang[:half], 0.0), (ang[half:], 200.0)]
    filt2 = O.projection_filter(T, case["curve"], kv=300.0, cs_mm=2.7, amplitude_contrast=0.07,
                                defocus1=case["defocus"], defocus2=case["defocus"], pixel_size=case["pixel_size"],
                                defocus_offset=200.0)
    filters = [case["filt"], filt2]

    # context entry points
    with core.SearchCore(X, Y, T, histogram_min_scaled=case["hmin"], histogram_step_scaled=case["hstep"]) as sc:
        sc.set_template(case["tspec"])
        sc.set_image(case["ispec"])
        for (a, df), f in zip(calls, filters):
            sc.run_plane(f, a, defocus_offset=df)
        ref = sc.results()

    # allocation-free entry point on caller-owned device buffers
    L = core.load()
    n = X * Y
    d_t = _dev(torch, case["tspec"].astype(np.complex64), np.float32)
    d_i = _dev(torch, case["ispec"].astype(np.complex64), np.float32)
    d_f = [_dev(torch, f.astype(np.float32), np.float32) for f in filters]
    d_mip = torch.full((n,), -np.finfo(np.float32).max, dtype=torch.float32, device="cuda")
    d_best = torch.full((n,), -1, dtype=torch.int32, device="cuda")
    d_sum = torch.zeros(n, dtype=torch.float64, device="cuda")
    d_sq = torch.zeros(n, dtype=torch.float64, device="cuda")
    d_hist = torch.zeros(512, dtype=torch.int64, device="cuda")
    dims = core.TmDims(X, Y, T, 512, case["hmin"], case["hstep"], 0, 0)
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    first = 0
    for (a, df), f in zip(calls, d_f):
        a = np.ascontiguousarray(a, np.float32)
        rc = L.tm_run_plane_noalloc(0, ctypes.byref(dims), p(d_t), p(d_i), p(f), a.ctypes.data_as(ctypes.c_void_p),
                                    len(a), first, p(d_mip), p(d_best), p(d_sum), p(d_sq), p(d_hist), None)
        assert rc == core.TM_OK, rc
        assert torch.cuda.current_device() == 0
        first += len(a)
    mip = d_mip.cpu().numpy()
    best = d_best.cpu().numpy()
    s = d_sum.cpu().numpy()
    q = d_sq.cpu().numpy()
    hist = d_hist.cpu().numpy()

    scale = np.abs(ref["mip"]).max()
    assert np.abs(mip - ref["mip"]).max() / scale < 1e-4
    # decode the orientation index with the call order's angle and defocus tables
    all_ang = np.concatenate([c[0] for c in calls])
    dfs = np.concatenate([np.full(len(c[0]), c[1], np.float32) for c in calls])
    assert best.min() >= 0
    # the prepared spectrum is built on the device here and on the host there, so
    # ties closer than FP32 rounding may resolve differently: allow 0.1% of pixels
    for k, col in (("phi", 0), ("theta", 1), ("psi", 2)):
        assert (all_ang[best, col] != ref[k]).mean() <= 1e-3, k
    assert (dfs[best] != ref["defocus"]).mean() <= 1e-3
    assert np.abs(s - ref["sum"]).max() / np.abs(ref["sum"]).max() < 1e-5
    assert np.abs(q - ref["sumsq"]).max() / np.abs(ref["sumsq"]).max() < 1e-5
    assert np.all(np.abs(hist - ref["hist"]) <= 0.001 * ref["hist"] + 2)


def test_noalloc_rejects_unsupported_geometry():
    torch = pytest.importorskip("torch")
    L = core.load()
    # no compiled no-alloc variant (its intermediates would not fit the fixed array)
    dims = core.TmDims(4096, 4096, 256, 512, -0.003, 1e-5, 0, 0)
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(buf.data_ptr())
    a = np.zeros(3, np.float32)
    rc = L.tm_run_plane_noalloc(0, ctypes.byref(dims), p, p, p, a.ctypes.data_as(ctypes.c_void_p), 1, 0,
                                p, p, p, p, p, None)
    assert rc == core.TM_ERR_UNSUPPORTED
