"""ctypes bindings of the search core's C ABI (include/tm_b200.h).

``SearchCore`` is a thin object over one ``tm_ctx``; ``TemplateMatchingCore``
mirrors the reference class of the same name (src/gpu/TemplateMatchingCore.h:
55-179): ``Init`` takes the prepared template and micrograph spectra and the
search ranges, ``RunInnerLoop`` runs one (pixel size, defocus) plane over the
orientation range ``[first_search_position, last_search_position]`` x psi, and
the results are read back like the reference's device images.

The library must exist and load: there is no fallback.  Building it needs only
nvcc (``python -m cistem_downstream_bah_b200.build``); running it needs a GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

TM_OK = 0
TM_ERR_INVALID = -1
TM_ERR_CUDA = -2
TM_ERR_UNSUPPORTED = -3
TM_ERR_OOM = -4
TM_ERR_TIMEOUT = -5
TM_ERR_CANCELLED = -6
PRECISION_FP32 = 0
PRECISION_FP16_TENSOR = 1

EXPORTED = [
    "tm_create", "tm_set_template", "tm_set_image", "tm_reset_results", "tm_run_plane",
    "tm_get_results", "tm_correlations_computed", "tm_last_timing", "tm_debug_stage_buffers", "tm_destroy",
    "tm_last_error", "tm_version", "tm_run_plane_noalloc", "tm_autotune_batch", "tm_orientation_batch",
    "tm_refine_create", "tm_refine_set_particle", "tm_refine_set_filter", "tm_refine_set_operator",
    "tm_refine_score", "tm_refine_last_error", "tm_refine_destroy", "tm_set_micrograph", "tm_whiten_micrograph",
    "tm_set_template_volume", "tm_template_spectrum", "tm_set_normalization_pixels", "tm_pnet_create",
    "tm_pnet_param_count", "tm_pnet_set_params", "tm_pnet_get_params", "tm_pnet_forward", "tm_pnet_gradients",
    "tm_pnet_train_step", "tm_pnet_last_error", "tm_pnet_destroy", "tm_set_image_set", "tm_run_plane_images",
    "tm_get_image_results", "tm_set_precision", "tm_get_precision", "tm_debug_gemm",
]


class TmDims(ctypes.Structure):
    _fields_ = [
        ("image_x", ctypes.c_int), ("image_y", ctypes.c_int), ("template_size", ctypes.c_int),
        ("histogram_bins", ctypes.c_int),
        ("histogram_min_scaled", ctypes.c_double), ("histogram_step_scaled", ctypes.c_double),
        ("orientation_batch", ctypes.c_int), ("device", ctypes.c_int),
    ]


PROGRESS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_void_p)

_LIB = None


class TmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"tm error {code}: {msg}")
        self.code = code


def library_path() -> str:
    return _build.CORE_LIB


def load(build_if_missing: bool = True) -> ctypes.CDLL:
    """Loads libtm_b200.so (building it first when missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        if not build_if_missing:
            raise OSError(f"{path} is missing; run python -m cistem_downstream_bah_b200.build")
        _build.build_core()
    L = ctypes.CDLL(path)
    vp, ip, fp = ctypes.c_void_p, ctypes.c_int, ctypes.c_float
    L.tm_create.argtypes = [ctypes.POINTER(TmDims), ctypes.POINTER(vp)]
    L.tm_set_template.argtypes = [vp, vp, ip]
    L.tm_set_image.argtypes = [vp, vp, ip, ip]
    L.tm_reset_results.argtypes = [vp]
    L.tm_run_plane.argtypes = [vp, vp, vp, ip, fp, fp, PROGRESS_FN, vp]
    L.tm_get_results.argtypes = [vp] + [vp] * 9
    L.tm_correlations_computed.argtypes = [vp]
    L.tm_correlations_computed.restype = ctypes.c_longlong
    L.tm_last_timing.argtypes = [vp] + [ctypes.POINTER(ctypes.c_double)] * 4
    L.tm_debug_stage_buffers.argtypes = [vp] * 8
    L.tm_run_plane_noalloc.argtypes = [ip, ctypes.POINTER(TmDims), vp, vp, vp, vp, ip, ip, vp, vp, vp, vp, vp, vp]
    L.tm_autotune_batch.argtypes = [vp, vp, vp, ip, ctypes.POINTER(ctypes.c_int)]
    L.tm_orientation_batch.argtypes = [vp]
    L.tm_orientation_batch.restype = ctypes.c_int
    L.tm_destroy.argtypes = [vp]
    L.tm_last_error.argtypes = [vp]
    L.tm_last_error.restype = ctypes.c_char_p
    L.tm_version.restype = ctypes.c_char_p
    L.tm_refine_create.argtypes = [ip, ip, ip, vp, ip, ip, ip, ip, ctypes.POINTER(vp)]
    L.tm_refine_set_particle.argtypes = [vp, ip, vp]
    L.tm_refine_set_filter.argtypes = [vp, ip, vp]
    L.tm_refine_set_operator.argtypes = [vp, ip, vp, vp, vp, vp, ip]
    L.tm_refine_score.argtypes = [vp, ip, vp, vp, vp, vp, vp]
    L.tm_refine_last_error.argtypes = [vp]
    L.tm_refine_last_error.restype = ctypes.c_char_p
    L.tm_refine_destroy.argtypes = [vp]
    L.tm_set_micrograph.argtypes = [vp, vp, ip, ip, vp, ip, ctypes.POINTER(ctypes.c_int)]
    L.tm_whiten_micrograph.argtypes = [ip, vp, ip, ip, vp, vp, ip, ctypes.POINTER(ctypes.c_int)]
    L.tm_set_template_volume.argtypes = [vp, vp, ip, fp]
    L.tm_template_spectrum.argtypes = [ip, vp, ip, fp, vp]
    L.tm_set_normalization_pixels.argtypes = [vp, ctypes.c_longlong]
    L.tm_set_image_set.argtypes = [vp, ip, vp]
    L.tm_run_plane_images.argtypes = [vp, vp, vp, ip, vp, ip, fp, fp]
    L.tm_get_image_results.argtypes = [vp, ip, vp, vp, vp, vp]
    L.tm_set_precision.argtypes = [vp, ip]
    L.tm_debug_gemm.argtypes = [ip, ip, ip, ip, vp, vp, vp, fp, ip, ip]
    L.tm_get_precision.argtypes = [vp]
    _LIB = L
    return L


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class SearchCore:
    """One search context on one GPU (tm_create ... tm_destroy)."""

    def __init__(self, image_x, image_y, template_size, *, histogram_min_scaled, histogram_step_scaled,
                 histogram_bins=512, orientation_batch=0, device=0):
        self.L = load()
        self.X, self.Y, self.T = image_x, image_y, template_size
        self.hist_bins = histogram_bins
        d = TmDims(image_x, image_y, template_size, histogram_bins, histogram_min_scaled, histogram_step_scaled,
                   orientation_batch, device)
        h = ctypes.c_void_p()
        rc = self.L.tm_create(ctypes.byref(d), ctypes.byref(h))
        self.h = h
        if rc != TM_OK:
            msg = self.L.tm_last_error(h).decode() if h.value else "tm_create failed"
            if h.value:
                self.L.tm_destroy(h)
            self.h = ctypes.c_void_p()
            raise TmError(rc, msg)

    def _check(self, rc):
        if rc != TM_OK:
            raise TmError(rc, self.L.tm_last_error(self.h).decode())

    def set_template(self, spectrum):
        s = np.ascontiguousarray(spectrum, dtype=np.complex64)
        assert s.shape == (self.T, self.T, self.T // 2 + 1), s.shape
        self._check(self.L.tm_set_template(self.h, _ptr(s), self.T))

    def set_image(self, spectrum):
        s = np.ascontiguousarray(spectrum, dtype=np.complex64)
        assert s.shape == (self.Y, self.X // 2 + 1), s.shape
        self._check(self.L.tm_set_image(self.h, _ptr(s), self.X, self.Y))

    def set_precision(self, precision):
        """PRECISION_FP32 (the parity path) or PRECISION_FP16_TENSOR (FP16
        correlation spectra, tensor-core row transform; tm_set_precision)."""
        self._check(self.L.tm_set_precision(self.h, int(precision)))

    def precision(self):
        return int(self.L.tm_get_precision(self.h))

    def set_template_volume(self, volume, pixel_size_factor=1.0):
        """Prepares the template spectrum on the device from the T^3 volume."""
        v = np.ascontiguousarray(volume, dtype=np.float32)
        assert v.shape == (self.T, self.T, self.T), v.shape
        self._check(self.L.tm_set_template_volume(self.h, _ptr(v), self.T, float(pixel_size_factor)))

    def set_micrograph(self, image):
        """Whitens the padded micrograph on the device and makes it the
        context's image; returns the whitening curve."""
        img = np.ascontiguousarray(image, dtype=np.float32)
        assert img.shape == (self.Y, self.X), img.shape
        cap = int((self.X / 2.0 + 1.0) * float(np.sqrt(np.float32(2.0))) + 1.0) + 8
        curve = np.zeros(cap, np.float64)
        n = ctypes.c_int()
        self._check(self.L.tm_set_micrograph(self.h, _ptr(img), self.X, self.Y, _ptr(curve), cap, ctypes.byref(n)))
        return curve[:n.value].copy()

    def set_normalization_pixels(self, n_pixels):
        """Forms the projection variance over n_pixels instead of the context's
        X*Y (0 restores that): a window cut from a larger whitened micrograph
        then reports that micrograph's correlation values."""
        self._check(self.L.tm_set_normalization_pixels(self.h, ctypes.c_longlong(int(n_pixels))))

    def set_image_set(self, spectra):
        """Several micrograph spectra of this context's size, each with its own results."""
        s = np.ascontiguousarray(spectra, dtype=np.complex64)
        assert s.ndim == 3 and s.shape[1:] == (self.Y, self.X // 2 + 1), s.shape
        self._check(self.L.tm_set_image_set(self.h, len(s), _ptr(s)))
        self.n_images = len(s)

    def run_plane_images(self, projection_filter, euler_angles, images, defocus_offset=0.0, pixel_size_offset=0.0):
        f = np.ascontiguousarray(projection_filter, dtype=np.float32)
        assert f.shape == (self.T, self.T // 2 + 1), f.shape
        a = np.ascontiguousarray(euler_angles, dtype=np.float32).reshape(-1, 3)
        ids = np.ascontiguousarray(images, dtype=np.int32)
        self._check(self.L.tm_run_plane_images(self.h, _ptr(f), _ptr(a), len(a), _ptr(ids), len(ids),
                                               defocus_offset, pixel_size_offset))

    def image_results(self, image):
        n = self.X * self.Y
        out = {k: np.zeros(n, np.float32) for k in ("mip", "psi", "theta", "phi")}
        self._check(self.L.tm_get_image_results(self.h, int(image), _ptr(out["mip"]), _ptr(out["psi"]),
                                                _ptr(out["theta"]), _ptr(out["phi"])))
        return out

    def reset(self):
        self._check(self.L.tm_reset_results(self.h))

    def run_plane(self, projection_filter, euler_angles, defocus_offset=0.0, pixel_size_offset=0.0, progress=None):
        f = np.ascontiguousarray(projection_filter, dtype=np.float32)
        assert f.shape == (self.T, self.T // 2 + 1), f.shape
        a = np.ascontiguousarray(euler_angles, dtype=np.float32).reshape(-1, 3)
        cb = PROGRESS_FN(progress) if progress else PROGRESS_FN()
        self._check(self.L.tm_run_plane(self.h, _ptr(f), _ptr(a), len(a), defocus_offset, pixel_size_offset, cb, None))

    def autotune(self, projection_filter, euler_angles):
        """Picks the orientations per device pass (16, 32, 64 or 128) by timing the
        given orientations (contexts created with orientation_batch=0); clears
        the running results.  Returns the batch."""
        f = np.ascontiguousarray(projection_filter, dtype=np.float32)
        a = np.ascontiguousarray(euler_angles, dtype=np.float32).reshape(-1, 3)
        b = ctypes.c_int(0)
        self._check(self.L.tm_autotune_batch(self.h, _ptr(f), _ptr(a), len(a), ctypes.byref(b)))
        return b.value

    def orientation_batch(self):
        return int(self.L.tm_orientation_batch(self.h))

    def results(self):
        n = self.X * self.Y
        out = {k: np.zeros(n, np.float32) for k in ("mip", "psi", "theta", "phi", "defocus", "pixel")}
        s = np.zeros(n, np.float64)
        q = np.zeros(n, np.float64)
        h = np.zeros(self.hist_bins, np.int64)
        self._check(self.L.tm_get_results(self.h, _ptr(out["mip"]), _ptr(out["psi"]), _ptr(out["theta"]),
                                          _ptr(out["phi"]), _ptr(out["defocus"]), _ptr(out["pixel"]),
                                          _ptr(s), _ptr(q), _ptr(h)))
        out["sum"], out["sumsq"], out["hist"] = s, q, h
        return out

    def correlations_computed(self):
        return int(self.L.tm_correlations_computed(self.h))

    def last_timing(self):
        v = [ctypes.c_double() for _ in range(4)]
        self._check(self.L.tm_last_timing(self.h, *[ctypes.byref(x) for x in v]))
        return {"total_ms": v[0].value, "pass_b_ms": v[1].value, "pass_c_ms": v[2].value, "prep_ms": v[3].value}

    def stage_buffers(self, projection_filter, euler_angle):
        """Intermediates of one orientation (see tm_debug_stage_buffers)."""
        f = np.ascontiguousarray(projection_filter, dtype=np.float32)
        e = np.ascontiguousarray(euler_angle, dtype=np.float32).reshape(3)
        T, hc = self.T, self.X // 2 + 1
        out = dict(slice=np.zeros((T, T // 2 + 1), np.complex64), projection=np.zeros((T, T), np.float32),
                   normalisation=np.zeros(2, np.float32), rows=np.zeros((T, hc), np.complex64),
                   columns=np.zeros((self.Y, hc), np.complex64))
        self._check(self.L.tm_debug_stage_buffers(self.h, _ptr(f), _ptr(e), _ptr(out["slice"]), _ptr(out["projection"]),
                                                  _ptr(out["normalisation"]), _ptr(out["rows"]), _ptr(out["columns"])))
        return out

    def close(self):
        if self.h and self.h.value:
            self.L.tm_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def orientation_list(search_positions, psi_start, psi_step, psi_max, first=0, last=None):
    """(phi, theta, psi) in the reference's loop order for search positions
    [first, last]: position outer, psi inner, psi accumulated in float
    (match_template.cpp:996-1004)."""
    pos = np.asarray(search_positions, dtype=np.float32)
    if last is None:
        last = len(pos) - 1
    psis = []
    p = np.float32(psi_start)
    while p <= np.float32(psi_max):
        psis.append(p)
        p = np.float32(p + np.float32(psi_step))
    psis = np.array(psis, dtype=np.float32)
    sel = pos[first:last + 1]
    out = np.zeros((len(sel) * len(psis), 3), np.float32)
    out[:, 0] = np.repeat(sel[:, 0], len(psis))
    out[:, 1] = np.repeat(sel[:, 1], len(psis))
    out[:, 2] = np.tile(psis, len(sel))
    return out


class TemplateMatchingCore:
    """Mirror of the reference's TemplateMatchingCore (TemplateMatchingCore.h:55-179)."""

    def Init(self, template_reconstruction, input_image, pixel_size_search_range, pixel_size_step, pixel_size,
             defocus_search_range, defocus_step, defocus1, defocus2, psi_max, psi_start, psi_step,
             search_positions, histogram_min_scaled, histogram_step_scaled, histogram_number_of_bins,
             max_padding, first_search_position, last_search_position, total_correlation_positions=0,
             image_x=None, image_y=None, device=0, orientation_batch=0):
        self.image_y = input_image.shape[0]
        self.image_x = image_x if image_x is not None else 2 * (input_image.shape[1] - 1)
        self.T = template_reconstruction.shape[0]
        self.psi_max, self.psi_start, self.psi_step = psi_max, psi_start, psi_step
        self.pixel_size_step, self.defocus_step = pixel_size_step, defocus_step
        self.orientations = orientation_list(search_positions, psi_start, psi_step, psi_max,
                                             first_search_position, last_search_position)
        self.core = SearchCore(self.image_x, self.image_y, self.T, histogram_min_scaled=histogram_min_scaled,
                               histogram_step_scaled=histogram_step_scaled, histogram_bins=histogram_number_of_bins,
                               device=device, orientation_batch=orientation_batch)
        self.core.set_template(template_reconstruction)
        self.core.set_image(input_image)
        self.total_number_of_cccs_calculated = 0

    def RunInnerLoop(self, projection_filter, c_pixel, c_defocus, threadIDX=0, current_correlation_position=0):
        """One plane; like the reference, the per-plane state starts from zero."""
        self.core.reset()
        self.core.run_plane(projection_filter, self.orientations,
                            defocus_offset=float(np.float32(c_defocus) * np.float32(self.defocus_step)),
                            pixel_size_offset=float(np.float32(c_pixel) * np.float32(self.pixel_size_step)))
        r = self.core.results()
        shape = (self.image_y, self.image_x)
        self.d_max_intensity_projection = r["mip"].reshape(shape)
        self.d_best_psi = r["psi"].reshape(shape)
        self.d_best_theta = r["theta"].reshape(shape)
        self.d_best_phi = r["phi"].reshape(shape)
        self.d_sum3 = r["sum"].reshape(shape)
        self.d_sumSq3 = r["sumsq"].reshape(shape)
        self.histogram = r["hist"]
        self.total_number_of_cccs_calculated = len(self.orientations)
        return current_correlation_position + len(self.orientations)


class RefineCore:
    """Batched TemplateScore of refine_template on one GPU (tm_refine_create ...
    tm_refine_destroy): the template spectrum of the projection box TP, particle
    window spectra, projection filters and pixel-size operators in slots."""

    def __init__(self, template_spectrum, T, max_batch=64, max_particles=16, max_filters=64, max_operators=8,
                 device=0):
        self._L = load()
        spec = np.ascontiguousarray(template_spectrum, dtype=np.complex64)
        self.T, self.TP = int(T), int(spec.shape[0])
        self._ctx = ctypes.c_void_p()
        rc = self._L.tm_refine_create(device, self.T, self.TP, _ptr(spec), max_batch, max_particles, max_filters,
                                      max_operators, ctypes.byref(self._ctx))
        self._check(rc, "tm_refine_create")

    def _check(self, rc, what):
        if rc != TM_OK:
            msg = self._L.tm_refine_last_error(self._ctx).decode() if self._ctx else ""
            raise TmError(rc, f"{what}: {msg}")

    def set_particle(self, slot, spectrum):
        a = np.ascontiguousarray(spectrum, dtype=np.complex64)
        self._check(self._L.tm_refine_set_particle(self._ctx, int(slot), _ptr(a)), "tm_refine_set_particle")

    def set_filter(self, slot, filt):
        a = np.ascontiguousarray(filt, dtype=np.float32)
        self._check(self._L.tm_refine_set_filter(self._ctx, int(slot), _ptr(a)), "tm_refine_set_filter")

    def set_operator(self, slot, ar, ai, brt, bit, has_pad_value):
        arrs = [np.ascontiguousarray(x, dtype=np.float32) for x in (ar, ai, brt, bit)]
        self._check(self._L.tm_refine_set_operator(self._ctx, int(slot), *[_ptr(x) for x in arrs],
                                                   1 if has_pad_value else 0), "tm_refine_set_operator")

    def score(self, euler, particle, filt, op):
        """(n, 3) array of (value, x, y)."""
        e = np.ascontiguousarray(euler, dtype=np.float32).reshape(-1, 3)
        n = len(e)
        p = np.ascontiguousarray(particle, dtype=np.int32)
        f = np.ascontiguousarray(filt, dtype=np.int32)
        o = np.ascontiguousarray(op, dtype=np.int32)
        out = np.zeros((n, 3), np.float32)
        self._check(self._L.tm_refine_score(self._ctx, n, _ptr(e), _ptr(p), _ptr(f), _ptr(o), _ptr(out)),
                    "tm_refine_score")
        return out

    def close(self):
        if self._ctx:
            self._L.tm_refine_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def whiten_micrograph(image, device=0):
    """Device whitening of a padded micrograph (tm_whiten_micrograph):
    (half spectrum complex64 (ny, nx//2+1), whitening curve)."""
    L = load()
    img = np.ascontiguousarray(image, dtype=np.float32)
    ny, nx = img.shape
    spec = np.zeros((ny, nx // 2 + 1), np.complex64)
    cap = int((nx / 2.0 + 1.0) * float(np.sqrt(np.float32(2.0))) + 1.0) + 8
    curve = np.zeros(cap, np.float64)
    n = ctypes.c_int()
    rc = L.tm_whiten_micrograph(device, _ptr(img), nx, ny, _ptr(spec), _ptr(curve), cap, ctypes.byref(n))
    if rc != TM_OK:
        raise TmError(rc, "tm_whiten_micrograph failed")
    return spec, curve[:n.value].copy()


def debug_gemm(A, B, C=None, s=0.0, accumulate=False, tensor=True, device=0):
    """(A - s) B (+ C) through the library's device GEMM (tm_debug_gemm):
    tensor=True the tensor-core form, False the CUDA-core form."""
    L = load()
    a = np.ascontiguousarray(A, dtype=np.float32)
    b = np.ascontiguousarray(B, dtype=np.float32)
    M, K = a.shape
    N = b.shape[1]
    c = np.zeros((M, N), np.float32) if C is None else np.array(C, dtype=np.float32, order="C")
    rc = L.tm_debug_gemm(device, M, N, K, _ptr(a), _ptr(b), _ptr(c), float(s), int(bool(accumulate)), int(bool(tensor)))
    if rc != TM_OK:
        raise TmError(rc, "tm_debug_gemm failed")
    return c


def template_spectrum_device(volume, pixel_size_factor=1.0, device=0):
    """Template spectrum prepared on the device (tm_template_spectrum)."""
    L = load()
    v = np.ascontiguousarray(volume, dtype=np.float32)
    T = v.shape[0]
    out = np.zeros((T, T, T // 2 + 1), np.complex64)
    rc = L.tm_template_spectrum(device, _ptr(v), T, float(pixel_size_factor), _ptr(out))
    if rc != TM_OK:
        raise TmError(rc, "tm_template_spectrum failed")
    return out

