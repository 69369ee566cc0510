"""ctypes bindings of the C++ host preparation library (lib/libtm_host.so).

The library holds the host side of match_template that runs once per
micrograph or plane -- whitening, template spectrum (with the pixel-size
change), projection filter, search grid, factorisation and MRC I/O -- in C++
(host/*.cpp).  These bindings let Python callers and the tests use it; the
match_template program (lib/match_template) links the same sources.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libtm_host.so")
CLI_PATH = os.path.join(_HERE, "lib", "match_template")
MERGE_CLI_PATH = os.path.join(_HERE, "lib", "match_template_merge")
REFINE_CLI_PATH = os.path.join(_HERE, "lib", "refine_template")
_lib = None

EXPORTED = [
    "tmh_whiten", "tmh_template_spectrum", "tmh_projection_filter", "tmh_search_grid", "tmh_psi_list",
    "tmh_factorize_dimension", "tmh_is_power_of_two", "tmh_angular_step", "tmh_erfcinv", "tmh_edge_mean",
    "tmh_clip_into", "tmh_rotate90", "tmh_mrc_info", "tmh_mrc_read", "tmh_mrc_write", "tmh_find_peaks",
    "tmh_projection_montage", "tmh_job_search_ranges", "tmh_pack_worker_result", "tmh_merge_results",
    "tmh_refine_whiten", "tmh_refine_find_peaks", "tmh_window_particle", "tmh_cosine_mask", "tmh_pixel_size_operator",
    "tmh_padded_template_spectrum", "tmh_refine_synthetic",
]


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run cistem_downstream_bah_b200/build.py first")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        f, i, d = ctypes.c_float, ctypes.c_int, ctypes.c_double
        L.tmh_whiten.argtypes = [i, i, P, P, P, i]
        L.tmh_whiten.restype = i
        L.tmh_template_spectrum.argtypes = [i, P, f, P]
        L.tmh_projection_filter.argtypes = [i, P, i, f, f, f, f, f, f, f, f, f, P]
        L.tmh_search_grid.argtypes = [ctypes.c_char_p, f, P, i]
        L.tmh_search_grid.restype = i
        L.tmh_psi_list.argtypes = [f, f, f, P, i]
        L.tmh_psi_list.restype = i
        L.tmh_factorize_dimension.argtypes = [i, i]
        L.tmh_factorize_dimension.restype = i
        L.tmh_is_power_of_two.argtypes = [i]
        L.tmh_is_power_of_two.restype = i
        L.tmh_angular_step.argtypes = [f, f]
        L.tmh_angular_step.restype = f
        L.tmh_erfcinv.argtypes = [d]
        L.tmh_erfcinv.restype = d
        L.tmh_edge_mean.argtypes = [i, i, P]
        L.tmh_edge_mean.restype = f
        L.tmh_clip_into.argtypes = [i, i, P, i, i, f, P]
        L.tmh_rotate90.argtypes = [i, i, P, i, P]
        L.tmh_mrc_info.argtypes = [ctypes.c_char_p, P, P]
        L.tmh_mrc_info.restype = i
        L.tmh_mrc_read.argtypes = [ctypes.c_char_p, P]
        L.tmh_mrc_read.restype = i
        L.tmh_mrc_write.argtypes = [ctypes.c_char_p, i, i, i, P, f]
        L.tmh_mrc_write.restype = i
        L.tmh_find_peaks.argtypes = [i, i, P, P, P, P, P, P, f, i, i, f, P, i]
        L.tmh_find_peaks.restype = i
        L.tmh_projection_montage.argtypes = [i, P, i, P, i, i, P]
        L.tmh_job_search_ranges.argtypes = [i, i, P]
        L.tmh_job_search_ranges.restype = i
        lg = ctypes.c_long
        L.tmh_pack_worker_result.argtypes = [i, i, P, lg, lg, i, f, d, P, i, P, lg]
        L.tmh_pack_worker_result.restype = lg
        L.tmh_merge_results.argtypes = [i, P, P, i, P, P, P]
        L.tmh_merge_results.restype = i
        L.tmh_refine_whiten.argtypes = [i, i, P, P]
        L.tmh_refine_whiten.restype = i
        L.tmh_refine_find_peaks.argtypes = [i, i, P, f, f, P, i]
        L.tmh_refine_find_peaks.restype = i
        L.tmh_window_particle.argtypes = [i, i, P, i, i, i, P]
        L.tmh_cosine_mask.argtypes = [i, P, f, f]
        L.tmh_pixel_size_operator.argtypes = [i, i, f, P, P, P, P, P]
        L.tmh_pixel_size_operator.restype = i
        L.tmh_padded_template_spectrum.argtypes = [i, i, P, P]
        L.tmh_refine_synthetic.argtypes = [i, i, P, i, P, P, P, P, P, P, lg]
        L.tmh_refine_synthetic.restype = lg
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def whiten(image):
    img = _f32(image)
    ny, nx = img.shape
    spec = np.zeros((ny, nx // 2 + 1), np.complex64)
    curve = np.zeros(4 * nx + 16, np.float64)
    n = lib().tmh_whiten(nx, ny, _p(img), _p(spec), _p(curve), len(curve))
    return spec, curve[:n].copy()


def template_spectrum(volume, factor=1.0):
    vol = _f32(volume)
    T = vol.shape[0]
    out = np.zeros((T, T, T // 2 + 1), np.complex64)
    lib().tmh_template_spectrum(T, _p(vol), float(factor), _p(out))
    return out


def projection_filter(T, curve, *, kv, cs_mm, amplitude_contrast, defocus1, defocus2, astigmatism_angle=0.0,
                      pixel_size, phase_shift_deg=0.0, defocus_offset=0.0):
    c = np.ascontiguousarray(curve, np.float64)
    out = np.zeros((T, T // 2 + 1), np.float32)
    lib().tmh_projection_filter(T, _p(c), len(c), kv, cs_mm, amplitude_contrast, defocus1, defocus2,
                                astigmatism_angle, pixel_size, phase_shift_deg, defocus_offset, _p(out))
    return out


def search_grid(angular_step, symmetry="C1"):
    n = lib().tmh_search_grid(symmetry.encode(), angular_step, None, 0)
    if n < 0:
        raise ValueError(f"bad symmetry {symmetry}")
    out = np.zeros((n, 2), np.float32)
    lib().tmh_search_grid(symmetry.encode(), angular_step, _p(out), n)
    return out


def psi_list(start, step, max_):
    n = lib().tmh_psi_list(start, step, max_, None, 0)
    out = np.zeros(n, np.float32)
    lib().tmh_psi_list(start, step, max_, _p(out), n)
    return out


def factorize_dimension(original, template_size):
    return lib().tmh_factorize_dimension(int(original), int(template_size))


def edge_mean(img):
    a = _f32(img)
    return lib().tmh_edge_mean(a.shape[1], a.shape[0], _p(a))


def clip_into(img, ox, oy, pad=0.0):
    a = _f32(img)
    out = np.zeros((oy, ox), np.float32)
    lib().tmh_clip_into(a.shape[1], a.shape[0], _p(a), ox, oy, pad, _p(out))
    return out


def rotate90(img, positive=True):
    a = _f32(img)
    out = np.zeros((a.shape[1], a.shape[0]), np.float32)
    lib().tmh_rotate90(a.shape[1], a.shape[0], _p(a), int(positive), _p(out))
    return out


def read_mrc(path):
    """(data [z][y][x] float32, pixel size) of an MRC file (modes 0, 1, 2, 6, 12)."""
    dims = np.zeros(3, np.int32)
    px = np.zeros(1, np.float32)
    if lib().tmh_mrc_info(str(path).encode(), _p(dims), _p(px)) != 0:
        raise OSError(f"cannot read MRC file {path}")
    out = np.zeros((dims[2], dims[1], dims[0]), np.float32)
    if lib().tmh_mrc_read(str(path).encode(), _p(out)) != 0:
        raise OSError(f"cannot read MRC file {path}")
    return out, float(px[0])


def write_mrc(path, data, pixel_size=1.0):
    a = _f32(data)
    if a.ndim == 2:
        a = a[None]
    nz, ny, nx = a.shape
    if lib().tmh_mrc_write(str(path).encode(), nx, ny, nz, _p(a), pixel_size) != 0:
        raise OSError(f"cannot write MRC file {path}")


def find_peaks(scaled_mip, psi, theta, phi, defocus, pixel, threshold, min_peak_radius, template_size, pixel_size,
               max_peaks=1000):
    """Peak records (one row each: x_pos, y_pos, psi, theta, phi, defocus,
    pixel_size, peak_height, x, y) of a scaled MIP, as the reference's result
    aggregation finds them."""
    arrs = [_f32(a) for a in (scaled_mip, psi, theta, phi, defocus, pixel)]
    ny, nx = arrs[0].shape
    out = np.zeros((max_peaks, 10), np.float32)
    n = lib().tmh_find_peaks(nx, ny, *[_p(a) for a in arrs], float(threshold), int(min_peak_radius),
                             int(template_size), float(pixel_size), _p(out), max_peaks)
    return out[:n].copy()


def projection_montage(volume, peaks_xy_angles, nx, ny):
    """Result image of the reference's aggregation: projections of the template
    at each peak's angles, added where positive, centred on the peaks.
    peaks_xy_angles: rows (x, y, psi, theta, phi), pixel coordinates."""
    vol = _f32(volume)
    pk = _f32(np.asarray(peaks_xy_angles, np.float32).reshape(-1, 5))
    out = np.zeros((ny, nx), np.float32)
    lib().tmh_projection_montage(vol.shape[0], _p(vol), len(pk), _p(pk), nx, ny, _p(out))
    return out


def job_search_ranges(n_positions, n_jobs):
    """[(first, last)] search positions of each job, as the reference's panel
    splits one image's search (MatchTemplatePanel.cpp:674-784)."""
    out = np.zeros(2 * max(n_jobs, 0), np.int32)
    n = lib().tmh_job_search_ranges(int(n_positions), int(n_jobs), _p(out))
    return [(int(out[2 * k]), int(out[2 * k + 1])) for k in range(n)]


WORKER_MAPS = ("mip", "psi", "theta", "phi", "defocus", "pixel", "sum", "sumsq")


def pack_worker_result(maps, original_x, original_y, remove_npix_from_edge, number_of_ccs, sqrt_input_pixels,
                       histogram):
    """The flat float32 result array a worker job sends to its master.
    maps: dict of the 8 WORKER_MAPS, each (ny, nx) on the worker's padded box."""
    m = np.stack([_f32(maps[k]) for k in WORKER_MAPS])
    _, ny, nx = m.shape
    m = np.ascontiguousarray(m)
    h = np.ascontiguousarray(histogram, dtype=np.int64)
    n = lib().tmh_pack_worker_result(nx, ny, _p(m), int(original_x), int(original_y), int(remove_npix_from_edge),
                                     float(number_of_ccs), float(sqrt_input_pixels), _p(h), len(h), None, 0)
    if n < 0:
        raise ValueError("bad worker maps")
    out = np.zeros(n, np.float32)
    lib().tmh_pack_worker_result(nx, ny, _p(m), int(original_x), int(original_y), int(remove_npix_from_edge),
                                 float(number_of_ccs), float(sqrt_input_pixels), _p(h), len(h), _p(out), n)
    return out


MASTER_MAPS = ("mip", "psi", "theta", "phi", "defocus", "pixel", "scaled_mip", "avg", "std")


def merge_results(arrays, use_gpu=True):
    """The master over worker result arrays (in order): dict of the 9
    MASTER_MAPS, the 512 x 4 histogram table ("rows"), the expected threshold
    and the number of correlation maps."""
    arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in arrays]
    nx, ny = int(arrs[0][0]), int(arrs[0][1])
    ptrs = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    sizes = np.array([a.size for a in arrs], np.int64)
    maps = np.zeros((9, ny, nx), np.float32)
    rows = np.zeros((512, 4), np.float64)
    stats = np.zeros(2, np.float64)
    if lib().tmh_merge_results(len(arrs), ptrs, _p(sizes), 1 if use_gpu else 0, _p(maps), _p(rows), _p(stats)) != 0:
        raise ValueError("malformed or mismatching result arrays")
    out = {k: maps[i] for i, k in enumerate(MASTER_MAPS)}
    out.update(rows=rows, expected_threshold=float(stats[0]), number_of_ccs=float(stats[1]))
    return out


# ----------------------------------------------------------------------------- refine_template
def refine_whiten(image):
    """Whitened micrograph of refine_template, in real space."""
    img = _f32(image)
    ny, nx = img.shape
    out = np.zeros((ny, nx), np.float32)
    lib().tmh_refine_whiten(nx, ny, _p(img), _p(out))
    return out


def refine_find_peaks(scaled_mip, threshold, min_peak_radius, max_out=100000):
    z = _f32(scaled_mip)
    ny, nx = z.shape
    out = np.zeros((max_out, 3), np.float32)
    n = lib().tmh_refine_find_peaks(nx, ny, _p(z), float(threshold), float(min_peak_radius), _p(out), max_out)
    return out[:min(n, max_out)].copy()


def window_particle(image, peak_x, peak_y, T):
    img = _f32(image)
    ny, nx = img.shape
    out = np.zeros((T, T), np.float32)
    lib().tmh_window_particle(nx, ny, _p(img), int(peak_x), int(peak_y), int(T), _p(out))
    return out


def cosine_mask(image, radius, edge):
    img = np.array(image, dtype=np.float32)
    lib().tmh_cosine_mask(img.shape[0], _p(img), float(radius), float(edge))
    return img


def pixel_size_operator(nin, nout, factor):
    """(info dict, ar, ai, brt, bit) of the host's ChangePixelSize operator."""
    ar = np.zeros((nout, nin), np.float32)
    ai = np.zeros((nout, nin), np.float32)
    brt = np.zeros((nin, nout), np.float32)
    bit = np.zeros((nin, nout), np.float32)
    info = np.zeros(4, np.int32)
    if lib().tmh_pixel_size_operator(int(nin), int(nout), float(factor), _p(ar), _p(ai), _p(brt), _p(bit), _p(info)):
        raise ValueError("unsupported pixel-size change")
    return dict(identity=bool(info[0]), pad=int(info[1]), new=int(info[2]), has_pad_value=bool(info[3])), ar, ai, brt, bit


def padded_template_spectrum(volume, TP):
    vol = _f32(volume)
    T = vol.shape[0]
    out = np.zeros((TP, TP, TP // 2 + 1), np.complex64)
    lib().tmh_padded_template_spectrum(T, int(TP), _p(vol), _p(out))
    return out


REFINE_MAPS = ("mip", "scaled_mip", "psi", "theta", "phi", "defocus", "pixel_size")


def refine_synthetic(maps, peaks_xy, targets, params, max_log=2000000):
    """refine_template's descent with the synthetic score of
    tmh_refine_synthetic: (maps out, per-peak rows, log of scored candidates)."""
    m = np.ascontiguousarray(np.stack([_f32(maps[k]) for k in REFINE_MAPS]))
    _, ny, nx = m.shape
    pk = np.ascontiguousarray(peaks_xy, dtype=np.float32)
    tg = np.ascontiguousarray(targets, dtype=np.float64)
    pr = np.ascontiguousarray(params, dtype=np.float32)
    out = np.zeros_like(m)
    per = np.zeros((len(pk), 16), np.float32)
    log = np.zeros((max_log, 6), np.float32)
    n = lib().tmh_refine_synthetic(nx, ny, _p(m), len(pk), _p(pk), _p(tg), _p(pr), _p(out), _p(per), _p(log), max_log)
    return {k: out[i] for i, k in enumerate(REFINE_MAPS)}, per, log[:min(n, max_log)].copy()

