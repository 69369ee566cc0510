"""Python access to the CPU oracle (test infrastructure only).

Loads ``oracle/lib/liboracle64.so`` (FP64 restatement of the reference CPU
path of match_template) or ``liboracle32.so`` (the same source built in FP32,
timed as the CPU baseline) and exposes numpy-friendly wrappers.  Only the test
suite, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference
legs import this module; the product library never does.

Layout conventions match the reference's Image class (src/core/image.cpp:
4761-4800) without FFTW row padding: real images are ``(ny, nx)`` arrays, half
spectra are ``(ny, nx//2+1)`` complex arrays, volumes ``(nz, ny, nx)``.
"""
from __future__ import annotations

import ctypes
import os
import struct
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS: dict[int, ctypes.CDLL] = {}


class SearchArgs(ctypes.Structure):
    _fields_ = [
        ("X", ctypes.c_int), ("Y", ctypes.c_int), ("T", ctypes.c_int),
        ("n_orient", ctypes.c_int),
        ("angles", ctypes.c_void_p),
        ("template_spec", ctypes.c_void_p),
        ("image_spec", ctypes.c_void_p),
        ("filter", ctypes.c_void_p),
        ("hist_min_scaled", ctypes.c_double), ("hist_step_scaled", ctypes.c_double),
        ("hist_bins", ctypes.c_int),
        ("defocus_value", ctypes.c_float), ("pixel_value", ctypes.c_float),
    ]


def build():
    """Compile both oracle libraries with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib(bits: int = 64) -> ctypes.CDLL:
    if bits not in _LIBS:
        path = os.path.join(_HERE, "lib", f"liboracle{bits}.so")
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.orc_erfcinv.restype = ctypes.c_double
        L.orc_erfcinv.argtypes = [ctypes.c_double]
        L.orc_angular_step.restype = ctypes.c_float
        L.orc_angular_step.argtypes = [ctypes.c_float, ctypes.c_float]
        L.orc_find_peak_integer.restype = ctypes.c_double
        L.orc_psi_list.argtypes = [ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_void_p, ctypes.c_int]
        L.orc_search_grid.argtypes = [ctypes.c_char, ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_int]
        _LIBS[bits] = L
        assert L.orc_real_size() == bits // 8
    return _LIBS[bits]


def _rdtype(bits):
    return np.float64 if bits == 64 else np.float32


def _cdtype(bits):
    return np.complex128 if bits == 64 else np.complex64


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


# ----------------------------------------------------------------------------- FFTs
def rfft2(img, bits=64):
    """Unnormalised 2-D r2c FFT (FFTW convention)."""
    img = np.ascontiguousarray(img, dtype=_rdtype(bits))
    ny, nx = img.shape
    out = np.zeros((ny, nx // 2 + 1), dtype=_cdtype(bits))
    lib(bits).orc_rfft2(nx, ny, _p(img), _p(out))
    return out


def irfft2(spec, nx, bits=64):
    """Unnormalised 2-D c2r FFT; imaginary parts of DC/Nyquist terms ignored."""
    spec = np.ascontiguousarray(spec, dtype=_cdtype(bits))
    ny = spec.shape[0]
    out = np.zeros((ny, nx), dtype=_rdtype(bits))
    lib(bits).orc_irfft2(nx, ny, _p(spec), _p(out))
    return out


def rfft3(vol, bits=64):
    vol = np.ascontiguousarray(vol, dtype=_rdtype(bits))
    nz, ny, nx = vol.shape
    out = np.zeros((nz, ny, nx // 2 + 1), dtype=_cdtype(bits))
    lib(bits).orc_rfft3(nx, ny, nz, _p(vol), _p(out))
    return out


def cfft(x, sign=-1, bits=64):
    x = np.array(x, dtype=_cdtype(bits))
    lib(bits).orc_cfft(len(x), _p(x), sign)
    return x


# ----------------------------------------------------------------------------- helpers
def euler_matrix(phi, theta, psi):
    m = np.zeros(9, dtype=np.float32)
    lib().orc_euler_matrix(ctypes.c_float(phi), ctypes.c_float(theta), ctypes.c_float(psi), _p(m))
    return m.reshape(3, 3)


def factorize_dimension(original, template_size):
    return lib().orc_factorize_dimension(original, template_size)


def is_power_of_two(n):
    return bool(lib().orc_is_power_of_two(n))


def angular_step(resolution, radius):
    return float(lib().orc_angular_step(resolution, radius))


def erfcinv(x):
    return float(lib().orc_erfcinv(x))


def psi_list(psi_start, psi_step, psi_max):
    n = lib().orc_psi_list(psi_start, psi_step, psi_max, None, 0)
    out = np.zeros(n, dtype=np.float32)
    lib().orc_psi_list(psi_start, psi_step, psi_max, _p(out), n)
    return out


def search_grid(angular_step, symmetry="C1"):
    t = symmetry[0].upper().encode()
    num = int(symmetry[1:]) if len(symmetry) > 1 else 0
    n = lib().orc_search_grid(t, num, angular_step, None, 0)
    if n < 0:
        raise ValueError(f"bad symmetry {symmetry}")
    out = np.zeros((n, 2), dtype=np.float32)
    lib().orc_search_grid(t, num, angular_step, _p(out), n)
    return out


def orientation_list(positions, psis):
    """(phi, theta, psi) triples in the reference's loop order: search
    position outer, psi inner (match_template.cpp:996-1004)."""
    n_pos, n_psi = len(positions), len(psis)
    out = np.zeros((n_pos * n_psi, 3), dtype=np.float32)
    out[:, 0] = np.repeat(positions[:, 0], n_psi)
    out[:, 1] = np.repeat(positions[:, 1], n_psi)
    out[:, 2] = np.tile(psis, n_pos)
    return out


def phase_shift(spec, nx, sx, sy, sz=0.0, bits=64):
    spec = np.array(spec, dtype=_cdtype(bits))
    nz = spec.shape[0] if spec.ndim == 3 else 1
    ny = spec.shape[-2]
    lib(bits).orc_phase_shift(nx, ny, nz, _p(spec), ctypes.c_float(sx), ctypes.c_float(sy), ctypes.c_float(sz))
    return spec


def swap_quadrants(spec, nx, centred=True, bits=64):
    spec = np.array(spec, dtype=_cdtype(bits))
    nz = spec.shape[0] if spec.ndim == 3 else 1
    ny = spec.shape[-2]
    lib(bits).orc_swap_quadrants(nx, ny, nz, _p(spec), int(centred))
    return spec


def extract_slice(template_spec, matrix, bits=64):
    vol = np.ascontiguousarray(template_spec, dtype=_cdtype(bits))
    T = vol.shape[0]
    m = np.ascontiguousarray(np.asarray(matrix, dtype=np.float32).reshape(9))
    out = np.zeros((T, T // 2 + 1), dtype=_cdtype(bits))
    lib(bits).orc_extract_slice(T, _p(vol), _p(m), _p(out))
    return out


def whiten_image(image, bits=64):
    """Whitening of match_template.cpp:703-724; returns (spectrum, curve)."""
    img = np.array(image, dtype=_rdtype(bits))
    ny, nx = img.shape
    n = lib(bits).orc_whitening_curve_points(nx)
    spec = np.zeros((ny, nx // 2 + 1), dtype=_cdtype(bits))
    curve = np.zeros(n, dtype=_rdtype(bits))
    lib(bits).orc_whiten_image(nx, ny, _p(img), _p(spec), _p(curve))
    return spec, curve


def projection_filter(T, curve, *, kv, cs_mm, amplitude_contrast, defocus1, defocus2,
                      astigmatism_angle=0.0, pixel_size, phase_shift_deg=0.0, defocus_offset=0.0, bits=64):
    curve = np.ascontiguousarray(curve, dtype=_rdtype(bits))
    out = np.zeros((T, T // 2 + 1), dtype=_rdtype(bits))
    f = ctypes.c_float
    lib(bits).orc_projection_filter(
        T, f(kv), f(cs_mm), f(amplitude_contrast), f(defocus1), f(defocus2), f(astigmatism_angle),
        f(pixel_size), f(phase_shift_deg), f(defocus_offset), _p(curve), len(curve),
        f(np.float32(0.5) * np.sqrt(np.float32(2.0))), _p(out))
    return out


def prepare_template(volume, bits=64):
    vol = np.ascontiguousarray(volume, dtype=_rdtype(bits))
    T = vol.shape[0]
    out = np.zeros((T, T, T // 2 + 1), dtype=_cdtype(bits))
    lib(bits).orc_prepare_template(T, _p(vol), _p(out))
    return out


# ----------------------------------------------------------------------------- search
class SearchState:
    """Running outputs of the search across planes (reference CPU path
    semantics: MIP initialised to -FLT_MAX, angles to 0)."""

    def __init__(self, X, Y, hist_bins=512):
        n = X * Y
        self.X, self.Y = X, Y
        self.mip = np.full(n, -np.finfo(np.float32).max, dtype=np.float32)
        self.second = np.full(n, -np.finfo(np.float32).max, dtype=np.float32)
        self.psi = np.zeros(n, np.float32)
        self.theta = np.zeros(n, np.float32)
        self.phi = np.zeros(n, np.float32)
        self.defocus = np.zeros(n, np.float32)
        self.pixel = np.zeros(n, np.float32)
        self.sum = np.zeros(n, np.float64)
        self.sumsq = np.zeros(n, np.float64)
        self.hist = np.zeros(hist_bins + 1, np.int64)   # [hist_bins] = reference's OOB bin
        self.hist_bins = hist_bins


def search(state: SearchState, template_spec, image_spec, filt, angles, *, hist_min_scaled, hist_step_scaled,
           defocus_value=0.0, pixel_value=0.0, bits=64):
    """One (pixel size, defocus) plane of the CPU loop, accumulated into state."""
    T = template_spec.shape[0]
    X, Y = state.X, state.Y
    vol = np.ascontiguousarray(template_spec, dtype=_cdtype(bits))
    img = np.ascontiguousarray(image_spec, dtype=_cdtype(bits))
    fl = np.ascontiguousarray(filt, dtype=_rdtype(bits))
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    a = SearchArgs(X, Y, T, len(ang), _p(ang).value, _p(vol).value, _p(img).value, _p(fl).value,
                   hist_min_scaled, hist_step_scaled, state.hist_bins, defocus_value, pixel_value)
    lib(bits).orc_search(ctypes.byref(a), _p(state.mip), _p(state.psi), _p(state.theta), _p(state.phi),
                         _p(state.defocus), _p(state.pixel), _p(state.sum), _p(state.sumsq), _p(state.hist),
                         _p(state.second))
    return state


def correlate_one(template_spec, image_spec, filt, angles, o, X, Y, bits=64):
    T = template_spec.shape[0]
    vol = np.ascontiguousarray(template_spec, dtype=_cdtype(bits))
    img = np.ascontiguousarray(image_spec, dtype=_cdtype(bits))
    fl = np.ascontiguousarray(filt, dtype=_rdtype(bits))
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    a = SearchArgs(X, Y, T, len(ang), _p(ang).value, _p(vol).value, _p(img).value, _p(fl).value,
                   0.0, 1.0, 512, 0.0, 0.0)
    out = np.zeros((Y, X), dtype=_rdtype(bits))
    lib(bits).orc_correlate_one(ctypes.byref(a), o, _p(out))
    return out


def normalised_projection(template_spec, filt, angles, o, X, Y, bits=64):
    T = template_spec.shape[0]
    vol = np.ascontiguousarray(template_spec, dtype=_cdtype(bits))
    fl = np.ascontiguousarray(filt, dtype=_rdtype(bits))
    ang = np.ascontiguousarray(angles, dtype=np.float32)
    a = SearchArgs(X, Y, T, len(ang), _p(ang).value, _p(vol).value, None, _p(fl).value, 0.0, 1.0, 512, 0.0, 0.0)
    out = np.zeros((T, T), dtype=_rdtype(bits))
    lib(bits).orc_normalised_projection(ctypes.byref(a), o, _p(out))
    return out


def finalize(state: SearchState, n_total, sqrt_input_pixels):
    """Statistics of match_template.cpp:1221-1310 (local run)."""
    mip = state.mip.copy()
    s = state.sum.copy()
    q = state.sumsq.copy()
    n = len(mip)
    z = np.zeros(n, np.float32)
    avg = np.zeros(n, np.float32)
    sd = np.zeros(n, np.float32)
    lib().orc_finalize(ctypes.c_long(n), ctypes.c_long(n_total), ctypes.c_double(sqrt_input_pixels),
                       _p(mip), _p(s), _p(q), _p(z), _p(avg), _p(sd))
    return mip, z, avg, sd


# ----------------------------------------------------------------------------- pinned primitives
def clip_into_real(img, ox, oy, pad=0.0, bits=64):
    img = np.ascontiguousarray(img, dtype=_rdtype(bits))
    ny, nx = img.shape
    out = np.zeros((oy, ox), dtype=_rdtype(bits))
    lib(bits).orc_clip_into_real(nx, ny, _p(img), ox, oy, _p(out), ctypes.c_double(pad) if bits == 64 else ctypes.c_float(pad))
    return out


def clip_into_fourier(spec, nx, ox, oy, pad=0.0, bits=64):
    spec = np.ascontiguousarray(spec, dtype=_cdtype(bits))
    ny = spec.shape[0]
    out = np.zeros((oy, ox // 2 + 1), dtype=_cdtype(bits))
    lib(bits).orc_clip_into_fourier(nx, ny, _p(spec), ox, oy, _p(out), ctypes.c_double(pad) if bits == 64 else ctypes.c_float(pad))
    return out


def find_peak_integer(img, min_dist_from_edges=0):
    img = np.ascontiguousarray(img, dtype=np.float64)
    ny, nx = img.shape
    px, py = ctypes.c_float(), ctypes.c_float()
    L = lib()
    L.orc_find_peak_integer.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    v = L.orc_find_peak_integer(nx, ny, _p(img), min_dist_from_edges, ctypes.byref(px), ctypes.byref(py))
    return px.value, py.value, v


def rotate90(img, positive=True):
    img = np.ascontiguousarray(img, dtype=np.float64)
    ny, nx = img.shape
    out = np.zeros((nx, ny), dtype=np.float64)
    lib().orc_rotate90(nx, ny, _p(img), _p(out), int(positive))
    return out


# ----------------------------------------------------------------------------- MRC (tests)
def read_mrc(path):
    """Minimal MRC reader for mode 2 (float32) files: returns (nz, ny, nx)."""
    with open(path, "rb") as f:
        hdr = f.read(1024)
        nx, ny, nz, mode = struct.unpack("<4i", hdr[:16])
        next_ = struct.unpack("<i", hdr[92:96])[0]
        f.seek(1024 + next_)
        if mode != 2:
            raise ValueError(f"unsupported MRC mode {mode}")
        data = np.frombuffer(f.read(4 * nx * ny * nz), dtype="<f4")
    return data.reshape(nz, ny, nx)
