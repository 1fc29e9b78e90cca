"""ctypes access to the reference CPU backend built out of tree. TEST INFRASTRUCTURE ONLY.

``_ref/libope_cpu_ref.so`` is built by ``oracle/Makefile`` from the reference
sources (src/core/{types,iobuffer,processorconfiguration}.cpp and
src/backends/cpu/cpu_backend.cpp) plus ``ref_driver.cpp`` and the FFTW-API
shim. FFT = project shim, not FFTW (FFTW is not installed on either machine).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libope_cpu_ref.so")
# Source tree of the reference (read-only), named by the environment or, failing
# that, recorded by the last oracle build (_ref/reference_tree.txt); there is no
# default. Without either the prebuilt _ref/ libraries are used as they are.
def _reference_tree() -> str:
    t = os.environ.get("OPE_REFERENCE_TREE", "")
    rec = os.path.join(HERE, "_ref", "reference_tree.txt")
    if not t and os.path.exists(rec):
        with open(rec) as f:
            t = f.read().strip()
    return t if t and os.path.isdir(t) else ""


REFERENCE_TREE = _reference_tree()


class RefParams(ctypes.Structure):
    _fields_ = [
        ("signal_length", ctypes.c_int),
        ("ascans_per_bscan", ctypes.c_int),
        ("bscans_per_buffer", ctypes.c_int),
        ("input_dtype", ctypes.c_int),
        ("resampling_enabled", ctypes.c_int),
        ("interpolation", ctypes.c_int),
        ("resampling_coeffs", ctypes.c_float * 4),
        ("windowing_enabled", ctypes.c_int),
        ("window_type", ctypes.c_int),
        ("window_center", ctypes.c_float),
        ("window_fill", ctypes.c_float),
        ("dispersion_enabled", ctypes.c_int),
        ("dispersion_coeffs", ctypes.c_float * 4),
        ("dispersion_factor", ctypes.c_float),
        ("dc_removal_enabled", ctypes.c_int),
        ("dc_window", ctypes.c_int),
        ("log_scaling", ctypes.c_int),
        ("grayscale_min", ctypes.c_float),
        ("grayscale_max", ctypes.c_float),
        ("addend", ctypes.c_float),
        ("multiplicator", ctypes.c_float),
        ("fpn_removal", ctypes.c_int),
        ("fpn_bscan_count", ctypes.c_int),
        ("fpn_continuous", ctypes.c_int),
        ("post_bg_removal", ctypes.c_int),
        ("bg_weight", ctypes.c_float),
        ("bg_offset", ctypes.c_float),
    ]


def build(force: bool = False) -> bool:
    """Compile (or bring up to date) the reference oracle when the reference
    tree is named by OPE_REFERENCE_TREE; otherwise use the prebuilt library."""
    if REFERENCE_TREE and os.path.isdir(REFERENCE_TREE):
        subprocess.run(["make", "-C", HERE, f"REF={REFERENCE_TREE}"] + (["-B"] if force else []), check=True,
                       stdout=subprocess.DEVNULL)
    return os.path.exists(LIB_PATH)


_lib: Optional[ctypes.CDLL] = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"reference oracle not built: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(RefParams)
        fp = ctypes.POINTER(ctypes.c_float)
        L.ope_ref_generate_curves.argtypes = [P, fp, fp, fp, fp]
        L.ope_ref_create.argtypes = [P]
        L.ope_ref_create.restype = ctypes.c_void_p
        L.ope_ref_set_curve.argtypes = [ctypes.c_void_p, ctypes.c_int, fp, ctypes.c_size_t]
        L.ope_ref_process.argtypes = [ctypes.c_void_p, ctypes.c_void_p, fp, ctypes.c_int]
        L.ope_ref_update_params.argtypes = [ctypes.c_void_p, P]
        L.ope_ref_request_fpn.argtypes = [ctypes.c_void_p]
        L.ope_ref_get_fpn.argtypes = [ctypes.c_void_p, fp, ctypes.c_size_t]
        L.ope_ref_set_fpn.argtypes = [ctypes.c_void_p, fp, ctypes.c_size_t]
        L.ope_ref_request_bg.argtypes = [ctypes.c_void_p]
        L.ope_ref_get_bg.argtypes = [ctypes.c_void_p, fp, ctypes.c_size_t]
        L.ope_ref_set_bg.argtypes = [ctypes.c_void_p, fp, ctypes.c_size_t]
        L.ope_ref_destroy.argtypes = [ctypes.c_void_p]
        L.ope_ref_convert_input.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, fp]
        L.ope_ref_klinearization.argtypes = [fp, fp, ctypes.c_int, ctypes.c_int, fp]
        L.ope_ref_windowing.argtypes = [fp, fp, ctypes.c_int, fp]
        L.ope_ref_min_var_mean.argtypes = [fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, fp]
        L.ope_ref_ifft_magnitude.argtypes = [fp, ctypes.c_int, fp]
        L.ope_ref_fft_shim_precision.argtypes = [ctypes.c_int]
        L.ope_ref_rolling_dc.argtypes = [fp, ctypes.c_int, ctypes.c_int, fp]
        L.ope_ref_fft_shim_precision.restype = ctypes.c_int
        _lib = L
    return _lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def make_params(n, ascans, bscans=1, dtype=2, *, resampling=False, interpolation=0,
                resampling_coeffs=(0.0, 1.0, 0.0, 0.0), windowing=False, window_type=0,
                window_center=0.5, window_fill=0.95, dispersion=False,
                dispersion_coeffs=(0.0, 0.0, 0.0, 0.0), dispersion_factor=1.0,
                dc_removal=False, dc_window=64, log_scaling=True, grayscale_min=30.0,
                grayscale_max=100.0, addend=0.0, multiplicator=1.0, fpn_removal=False,
                fpn_bscan_count=1, fpn_continuous=False, post_bg_removal=False,
                bg_weight=1.0, bg_offset=0.0) -> RefParams:
    p = RefParams()
    p.signal_length, p.ascans_per_bscan, p.bscans_per_buffer, p.input_dtype = n, ascans, bscans, dtype
    p.resampling_enabled, p.interpolation = int(resampling), int(interpolation)
    for i in range(4):
        p.resampling_coeffs[i] = resampling_coeffs[i]
        p.dispersion_coeffs[i] = dispersion_coeffs[i]
    p.windowing_enabled, p.window_type = int(windowing), int(window_type)
    p.window_center, p.window_fill = window_center, window_fill
    p.dispersion_enabled, p.dispersion_factor = int(dispersion), dispersion_factor
    p.dc_removal_enabled, p.dc_window = int(dc_removal), dc_window
    p.log_scaling = int(log_scaling)
    p.grayscale_min, p.grayscale_max, p.addend, p.multiplicator = grayscale_min, grayscale_max, addend, multiplicator
    p.fpn_removal, p.fpn_bscan_count, p.fpn_continuous = int(fpn_removal), fpn_bscan_count, int(fpn_continuous)
    p.post_bg_removal, p.bg_weight, p.bg_offset = int(post_bg_removal), bg_weight, bg_offset
    return p


def generate_curves(p: RefParams):
    n = p.signal_length
    r = np.zeros(n, np.float32)
    w = np.zeros(n, np.float32)
    ph = np.zeros(n, np.float32)
    cs = np.zeros(2 * n, np.float32)
    lib().ope_ref_generate_curves(ctypes.byref(p), _fp(r), _fp(w), _fp(ph), _fp(cs))
    return r, w, ph, cs


def set_fft_precision(mode: str) -> None:
    lib().ope_ref_fft_shim_precision(1 if mode == "f32" else 0)


class RefBackend:
    """One reference CpuBackend with generated curves, processing frames synchronously."""

    def __init__(self, p: RefParams):
        self.p = p
        self.h = lib().ope_ref_create(ctypes.byref(p))
        if not self.h:
            raise RuntimeError("reference backend creation failed")

    def set_curve(self, kind: int, data: np.ndarray) -> None:
        d = np.ascontiguousarray(data, dtype=np.float32)
        lib().ope_ref_set_curve(self.h, kind, _fp(d), d.size)

    def process(self, raw: np.ndarray, timeout_ms: int = 600000) -> np.ndarray:
        p = self.p
        out = np.zeros(p.signal_length * p.ascans_per_bscan * p.bscans_per_buffer // 2, np.float32)
        raw = np.ascontiguousarray(raw)
        rc = lib().ope_ref_process(self.h, raw.ctypes.data_as(ctypes.c_void_p), _fp(out), timeout_ms)
        if rc != 0:
            raise RuntimeError(f"reference process failed ({rc})")
        return out.reshape(-1, p.signal_length // 2)

    def request_fpn(self) -> None:
        lib().ope_ref_request_fpn(self.h)

    def fpn_profile(self) -> np.ndarray:
        n = lib().ope_ref_get_fpn(self.h, None, 0)
        out = np.zeros(max(n, 0), np.float32)
        if n > 0:
            lib().ope_ref_get_fpn(self.h, _fp(out), n)
        return out

    def set_fpn(self, prof: np.ndarray) -> None:
        d = np.ascontiguousarray(prof, dtype=np.float32)
        lib().ope_ref_set_fpn(self.h, _fp(d), d.size // 2)

    def request_bg(self) -> None:
        lib().ope_ref_request_bg(self.h)

    def bg_profile(self) -> np.ndarray:
        n = lib().ope_ref_get_bg(self.h, None, 0)
        out = np.zeros(max(n, 0), np.float32)
        if n > 0:
            lib().ope_ref_get_bg(self.h, _fp(out), n)
        return out

    def close(self) -> None:
        if self.h:
            lib().ope_ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def convert_input(raw: np.ndarray, dtype: int) -> np.ndarray:
    """The reference's convertInput of one line of raw samples (ope::DataType dtype)."""
    raw = np.ascontiguousarray(raw)
    out = np.zeros(raw.size, np.float32)
    lib().ope_ref_convert_input(raw.ctypes.data, int(dtype), raw.size, _fp(out))
    return out


def klinearization(x: np.ndarray, curve: np.ndarray, method: int) -> np.ndarray:
    x = np.ascontiguousarray(x, np.float32)
    c = np.ascontiguousarray(curve, np.float32)
    out = np.zeros(x.size, np.float32)
    lib().ope_ref_klinearization(_fp(x), _fp(c), method, x.size, _fp(out))
    return out


def rolling_dc(x: np.ndarray, window: int) -> np.ndarray:
    """The reference's rollingAverageDCRemoval on each row of x (float32)."""
    x = np.ascontiguousarray(x, np.float32)
    out = np.empty_like(x)
    for i in range(x.shape[0]):
        lib().ope_ref_rolling_dc(_fp(x[i]), x.shape[1], int(window), _fp(out[i]))
    return out


def min_var_mean(X: np.ndarray, segments: int = 8) -> np.ndarray:
    h, w = X.shape
    inter = np.empty((h, w, 2), np.float32)
    inter[..., 0] = X.real
    inter[..., 1] = X.imag
    out = np.zeros(2 * w, np.float32)
    lib().ope_ref_min_var_mean(_fp(inter.reshape(-1)), w, h, segments, _fp(out))
    return out
