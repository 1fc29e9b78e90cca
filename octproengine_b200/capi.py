"""ctypes binding of the C ABI in ``include/ope_b200.h``.

This is the Python side of the drop-in boundary: plain pointers, sizes and
status codes. A non-zero status raises :class:`B200Error` carrying the
context's last error message, mirroring how the reference surfaces backend
errors as ``std::runtime_error`` (src/backends/cuda/cuda_backend.cu:14-33) and
how its Python bindings map them to exceptions
(python/octproengine_bindings.cpp:18-36).

The library is loaded from ``octproengine_b200/lib/libope_b200.so`` (built
in-tree by :mod:`octproengine_b200.build`). There is no fallback: if the
library or a GPU is missing, calls fail loudly.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libope_b200.so")

OK = 0
E_INVALID = -1
E_UNSUPPORTED = -2
E_CUDA = -3
E_TIMEOUT = -4
E_STATE = -5
E_NOMEM = -6
E_DEVICE = -7

_STATUS_NAMES = {E_INVALID: "invalid argument", E_UNSUPPORTED: "unsupported", E_CUDA: "CUDA error",
                 E_TIMEOUT: "timeout", E_STATE: "invalid state", E_NOMEM: "out of memory",
                 E_DEVICE: "device error"}


class B200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{_STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


class Config(ctypes.Structure):
    """Mirror of ``ope_b200_config``."""
    _fields_ = [
        ("signal_length", ctypes.c_int32),
        ("ascans_per_bscan", ctypes.c_int32),
        ("bscans_per_buffer", ctypes.c_int32),
        ("input_dtype", ctypes.c_int32),
        ("bitshift", ctypes.c_int32),
        ("resampling_enabled", ctypes.c_int32),
        ("interpolation", ctypes.c_int32),
        ("windowing_enabled", ctypes.c_int32),
        ("dispersion_enabled", ctypes.c_int32),
        ("dc_removal_enabled", ctypes.c_int32),
        ("dc_window", ctypes.c_int32),
        ("log_scaling", ctypes.c_int32),
        ("grayscale_min", ctypes.c_float),
        ("grayscale_max", ctypes.c_float),
        ("addend", ctypes.c_float),
        ("multiplicator", ctypes.c_float),
        ("fpn_removal", ctypes.c_int32),
        ("fpn_bscan_count", ctypes.c_int32),
        ("fpn_continuous", ctypes.c_int32),
        ("post_bg_removal", ctypes.c_int32),
        ("bg_weight", ctypes.c_float),
        ("bg_offset", ctypes.c_float),
        ("bscan_flip", ctypes.c_int32),
        ("sinusoidal_correction", ctypes.c_int32),
        ("float32_as_uint32", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("num_input_buffers", ctypes.c_int32),
        ("dc_split", ctypes.c_int32),
        ("dc_reference_order", ctypes.c_int32),
        ("reserved", ctypes.c_int32 * 7),
    ]


# every symbol include/ope_b200.h declares, with (restype, argtypes)
_P = ctypes.c_void_p
_FP = ctypes.POINTER(ctypes.c_float)
_SZ = ctypes.c_size_t
SIGNATURES = {
    "ope_b200_config_default": (None, [ctypes.POINTER(Config)]),
    "ope_b200_create": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(_P)]),
    "ope_b200_destroy": (None, [_P]),
    "ope_b200_update_config": (ctypes.c_int, [_P, ctypes.POINTER(Config)]),
    "ope_b200_last_error": (ctypes.c_char_p, [_P]),
    "ope_b200_set_resampling_curve": (ctypes.c_int, [_P, _FP, _SZ]),
    "ope_b200_set_dispersion_curve": (ctypes.c_int, [_P, _FP, _SZ]),
    "ope_b200_set_window_curve": (ctypes.c_int, [_P, _FP, _SZ]),
    "ope_b200_process_device": (ctypes.c_int, [_P, _P, _P, _P]),
    "ope_b200_process_device_n": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P]),
    "ope_b200_process_host": (ctypes.c_int, [_P, _P, _P]),
    "ope_b200_process_bins_device": (ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P]),
    "ope_b200_test_inject_copy_stall": (ctypes.c_int, [_P, ctypes.c_uint32]),
    "ope_b200_test_inject_wait_abort": (ctypes.c_int, [_P]),
    "ope_b200_ring_depth": (ctypes.c_int, [_P]),
    "ope_b200_host_register": (ctypes.c_int, [_P, _SZ]),
    "ope_b200_host_unregister": (ctypes.c_int, [_P]),
    "ope_b200_submit": (ctypes.c_int, [_P, _P, ctypes.POINTER(ctypes.c_uint64)]),
    "ope_b200_submit_to": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(ctypes.c_uint64)]),
    "ope_b200_input_released": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_int32]),
    "ope_b200_frame_device_input": (ctypes.c_int, [_P, ctypes.c_uint64, _P, ctypes.POINTER(ctypes.c_void_p)]),
    "ope_b200_wait": (ctypes.c_int, [_P, ctypes.c_uint64, ctypes.c_int32, ctypes.POINTER(_FP)]),
    "ope_b200_release": (ctypes.c_int, [_P, ctypes.c_uint64]),
    "ope_b200_request_fpn_determination": (ctypes.c_int, [_P]),
    "ope_b200_set_fpn_profile": (ctypes.c_int, [_P, _FP, _SZ]),
    "ope_b200_get_fpn_profile": (ctypes.c_int, [_P, _FP, _SZ, ctypes.POINTER(_SZ)]),
    "ope_b200_determine_fpn_noalloc": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P, _P]),
    "ope_b200_request_bg_recording": (ctypes.c_int, [_P]),
    "ope_b200_set_bg_profile": (ctypes.c_int, [_P, _FP, _SZ]),
    "ope_b200_get_bg_profile": (ctypes.c_int, [_P, _FP, _SZ, ctypes.POINTER(_SZ)]),
    "ope_b200_synchronize": (ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int32)]),
    "ope_b200_generate_resampling_curve": (ctypes.c_int, [ctypes.c_int32, _FP, _FP]),
    "ope_b200_generate_dispersion_phase": (ctypes.c_int, [ctypes.c_int32, _FP, _FP]),
    "ope_b200_generate_window_curve": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                                                      ctypes.c_float, _FP]),
    "ope_b200_phase_to_cos_sin": (ctypes.c_int, [_FP, _SZ, _FP]),
    "ope_b200_af_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _FP, ctypes.c_int32,
                                           ctypes.POINTER(_P)]),
    "ope_b200_af_destroy": (None, [_P]),
    "ope_b200_af_set_bitshift": (ctypes.c_int, [_P, ctypes.c_int32]),
    "ope_b200_af_last_error": (ctypes.c_char_p, [_P]),
    "ope_b200_af_forward": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P, ctypes.c_int32, _P, _P, _P]),
    "ope_b200_af_backward": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P, ctypes.c_int32, _P, _P, _P, _P]),
    "ope_b200_af_backward_dispersion": (ctypes.c_int, [_P, _P, ctypes.c_int64, _P, ctypes.c_int32, _P, _P, _P,
                                                        _P]),
    "ope_b200_af_kernel_accessible": (ctypes.c_int, [_P]),
    "ope_b200_af_small_copy": (ctypes.c_int, [_P, _P, ctypes.c_int32, _P]),
    "ope_b200_batch_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(_P)]),
    "ope_b200_batch_destroy": (None, [_P]),
    "ope_b200_batch_last_error": (ctypes.c_char_p, [_P]),
    "ope_b200_batch_run": (ctypes.c_int, [_P, _P]),
    "ope_b200_batch_run_graph": (ctypes.c_int, [_P, _P]),
    "ope_b200_batch_set_tuning": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "ope_b200_batch_get_tuning": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.POINTER(ctypes.c_int32),
                                                 ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float)]),
    "ope_b200_batch_autotune": (ctypes.c_int, [_P, ctypes.c_int32]),
    "ope_b200_op_convert_input": (ctypes.c_int, [_P, ctypes.c_int32, ctypes.c_int64, _FP]),
    "ope_b200_op_klinearization": (ctypes.c_int, [_FP, _FP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64, _FP]),
    "ope_b200_op_window_dispersion": (ctypes.c_int, [_FP, _FP, _FP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int64,
                                                     _FP]),
    "ope_b200_op_dft_magnitude": (ctypes.c_int, [_FP, ctypes.c_int32, ctypes.c_int32, _FP]),
    "ope_b200_op_min_variance_mean": (ctypes.c_int, [_FP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _FP]),
    "ope_b200_op_fpn_removal": (ctypes.c_int, [_FP, _FP, ctypes.c_int32, ctypes.c_int32, _FP]),
    "ope_b200_op_rolling_dc_removal": (ctypes.c_int, [_FP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _FP]),
    "ope_b200_op_bscan_flip": (ctypes.c_int, [_FP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, _FP]),
    "ope_b200_op_sinusoidal_correction": (ctypes.c_int, [_FP, _FP, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                         _FP]),
    "ope_b200_op_truncate": (ctypes.c_int, [_FP, ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                            ctypes.c_float, ctypes.c_int32, ctypes.c_int64, _FP]),
    "ope_b200_op_background_subtraction": (ctypes.c_int, [_FP, _FP, ctypes.c_float, ctypes.c_float, ctypes.c_int32,
                                                          ctypes.c_int64, _FP]),
    "ope_b200_abi_version": (ctypes.c_int, []),
    "ope_b200_device_supported": (ctypes.c_int, [ctypes.c_int32]),
}

_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    """Loads the native library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} missing: build it with `python -m octproengine_b200.build`")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def fptr(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def default_config() -> Config:
    c = Config()
    lib().ope_b200_config_default(ctypes.byref(c))
    return c


# ---- curve generators (bit-identical to ProcessorConfiguration's) ----

def generate_resampling_curve(n: int, coeffs) -> np.ndarray:
    c = np.asarray(coeffs, np.float32)
    out = np.empty(n, np.float32)
    _check(None, lib().ope_b200_generate_resampling_curve(n, fptr(c), fptr(out)))
    return out


def generate_dispersion_phase(n: int, coeffs) -> np.ndarray:
    c = np.asarray(coeffs, np.float32)
    out = np.empty(n, np.float32)
    _check(None, lib().ope_b200_generate_dispersion_phase(n, fptr(c), fptr(out)))
    return out


def generate_window_curve(n: int, window_type: int, center: float, fill: float) -> np.ndarray:
    out = np.empty(n, np.float32)
    _check(None, lib().ope_b200_generate_window_curve(n, int(window_type), center, fill, fptr(out)))
    return out


def phase_to_cos_sin(phase: np.ndarray) -> np.ndarray:
    p = np.ascontiguousarray(phase, np.float32)
    out = np.empty(2 * p.size, np.float32)
    _check(None, lib().ope_b200_phase_to_cos_sin(fptr(p), p.size, fptr(out)))
    return out


def _check(ctx, rc: int) -> None:
    if rc != OK:
        msg = lib().ope_b200_last_error(ctx).decode() if ctx else "see arguments"
        raise B200Error(rc, msg)


class Context:
    """One ``ope_b200_ctx``: the configured chain for one buffer geometry."""

    def __init__(self, cfg: Config):
        self.cfg = cfg
        h = ctypes.c_void_p()
        rc = lib().ope_b200_create(ctypes.byref(cfg), ctypes.byref(h))
        if rc != OK:
            raise B200Error(rc, "context creation failed (see stderr)")
        self.h = h

    # lifecycle
    def close(self) -> None:
        if getattr(self, "h", None):
            lib().ope_b200_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def check(self, rc: int) -> None:
        _check(self.h, rc)

    def update_config(self, cfg: Config) -> None:
        self.check(lib().ope_b200_update_config(self.h, ctypes.byref(cfg)))
        self.cfg = cfg

    # curves
    def set_resampling_curve(self, curve: np.ndarray) -> None:
        c = np.ascontiguousarray(curve, np.float32)
        self.check(lib().ope_b200_set_resampling_curve(self.h, fptr(c), c.size))

    def set_window_curve(self, curve: np.ndarray) -> None:
        c = np.ascontiguousarray(curve, np.float32)
        self.check(lib().ope_b200_set_window_curve(self.h, fptr(c), c.size))

    def set_dispersion_curve(self, cos_sin: np.ndarray) -> None:
        c = np.ascontiguousarray(cos_sin, np.float32)
        self.check(lib().ope_b200_set_dispersion_curve(self.h, fptr(c), c.size))

    # processing
    def process_device(self, d_in: int, d_out: int, stream: int = 0, num_ascans: Optional[int] = None) -> None:
        """Device pointers (ints, e.g. torch ``data_ptr()``) and a cudaStream_t handle."""
        if num_ascans is None:
            self.check(lib().ope_b200_process_device(self.h, d_in, d_out, stream))
        else:
            self.check(lib().ope_b200_process_device_n(self.h, d_in, d_out, int(num_ascans), stream))

    def process_bins_device(self, d_in: int, d_bins: int, num_ascans: int, stream: int = 0) -> None:
        self.check(lib().ope_b200_process_bins_device(self.h, d_in, d_bins, int(num_ascans), stream))

    def inject_copy_stall(self, timeout_us: int) -> None:
        self.check(lib().ope_b200_test_inject_copy_stall(self.h, int(timeout_us)))

    def inject_wait_abort(self) -> None:
        self.check(lib().ope_b200_test_inject_wait_abort(self.h))

    def process_host(self, raw: np.ndarray, out: Optional[np.ndarray] = None) -> np.ndarray:
        n = self.cfg.signal_length
        m = self.cfg.ascans_per_bscan * self.cfg.bscans_per_buffer
        raw = np.ascontiguousarray(raw)
        if out is None:
            out = np.empty((m, n // 2), np.float32)
        self.check(lib().ope_b200_process_host(self.h, raw.ctypes.data_as(ctypes.c_void_p),
                                               out.ctypes.data_as(ctypes.c_void_p)))
        return out

    # streaming ring
    def submit(self, h_in_ptr: int) -> int:
        t = ctypes.c_uint64(0)
        self.check(lib().ope_b200_submit(self.h, h_in_ptr, ctypes.byref(t)))
        return t.value

    def submit_to(self, h_in_ptr: int, h_out_ptr: int) -> int:
        """Like submit, but the frame's output is copied into the caller's host
        buffer h_out_ptr (page-locked for an asynchronous copy)."""
        t = ctypes.c_uint64(0)
        self.check(lib().ope_b200_submit_to(self.h, h_in_ptr, h_out_ptr, ctypes.byref(t)))
        return t.value

    def input_released(self, ticket: int, timeout_ms: int = -1) -> None:
        self.check(lib().ope_b200_input_released(self.h, ticket, timeout_ms))

    def frame_device_input(self, ticket: int, stream_handle: int) -> int:
        """Device address of a submitted frame's input copy; the stream waits for it.
        Valid until release(ticket)."""
        p = ctypes.c_void_p(0)
        self.check(lib().ope_b200_frame_device_input(self.h, ticket, stream_handle, ctypes.byref(p)))
        return int(p.value)

    def wait(self, ticket: int, timeout_ms: int = -1) -> np.ndarray:
        """Waits for the frame; returns a zero-copy view of its output (valid until release)."""
        p = _FP()
        self.check(lib().ope_b200_wait(self.h, ticket, timeout_ms, ctypes.byref(p)))
        n = self.cfg.signal_length
        m = self.cfg.ascans_per_bscan * self.cfg.bscans_per_buffer
        return np.ctypeslib.as_array(p, shape=(m, n // 2))

    def release(self, ticket: int) -> None:
        self.check(lib().ope_b200_release(self.h, ticket))

    def synchronize(self) -> int:
        st = ctypes.c_int32(0)
        self.check(lib().ope_b200_synchronize(self.h, ctypes.byref(st)))
        return st.value

    # fixed-pattern noise
    def request_fpn_determination(self) -> None:
        self.check(lib().ope_b200_request_fpn_determination(self.h))

    def set_fpn_profile(self, interleaved: np.ndarray) -> None:
        p = np.ascontiguousarray(interleaved, np.float32)
        self.check(lib().ope_b200_set_fpn_profile(self.h, fptr(p), p.size // 2))

    def determine_fpn_noalloc(self, d_in: int, num_ascans: int, d_profile: int, stream: int = 0) -> None:
        """FPN profile of the first fpn_bscan_count*A A-scans of a device buffer,
        using the library's static scratch array (no device allocation)."""
        self.check(lib().ope_b200_determine_fpn_noalloc(self.h, d_in, int(num_ascans), d_profile, stream))

    def fpn_profile(self) -> np.ndarray:
        pairs = _SZ(0)
        self.check(lib().ope_b200_get_fpn_profile(self.h, None, 0, ctypes.byref(pairs)))
        out = np.zeros(2 * pairs.value, np.float32)
        if pairs.value:
            self.check(lib().ope_b200_get_fpn_profile(self.h, fptr(out), pairs.value, ctypes.byref(pairs)))
        return out
