"""ctypes access to the reference library with this backend plugged in. TEST INFRASTRUCTURE ONLY.

``_ref/libope_dropin.so`` is built by ``make -C oracle REF=<tree> dropin`` from
a copy of the reference sources with the maintainer's Backend::B200 patch
applied (dropin_patch.py): the reference's own ope::Processor, CpuBackend and
CudaBackend, and this repository's B200Backend compiled against the
reference's ProcessingBackend. ``DropInProcessor(backend, params)`` drives one
``ope::Processor(backend)`` of that library through its public API
(dropin_driver.cpp). FFT of the CPU backend = project shim, not FFTW.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

from oracle.reflib import RefParams, REFERENCE_TREE, make_params  # noqa: F401  (re-exported)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libope_dropin.so")

# ope::Backend in the patched reference library
CUDA, CPU, B200 = 0, 1, 2


def build(force: bool = False) -> bool:
    """Build (or bring up to date) the patched reference library when the
    reference tree is known; otherwise use the prebuilt one."""
    if REFERENCE_TREE and os.path.isdir(REFERENCE_TREE):
        subprocess.run(["make", "-C", HERE, f"REF={REFERENCE_TREE}", "dropin"] + (["-B"] if force else []),
                       check=True, stdout=subprocess.DEVNULL)
    return os.path.exists(LIB_PATH)


def available() -> bool:
    return os.path.exists(LIB_PATH)


_lib: Optional[ctypes.CDLL] = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"drop-in reference library not built: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        fp = ctypes.POINTER(ctypes.c_float)
        L.ope_dropin_create.argtypes = [ctypes.c_int, ctypes.POINTER(RefParams)]
        L.ope_dropin_create.restype = ctypes.c_void_p
        L.ope_dropin_process.argtypes = [ctypes.c_void_p, ctypes.c_void_p, fp, ctypes.c_int]
        L.ope_dropin_request_fpn.argtypes = [ctypes.c_void_p]
        L.ope_dropin_set_fpn.argtypes = [ctypes.c_void_p, fp, ctypes.c_size_t]
        L.ope_dropin_get_fpn.argtypes = [ctypes.c_void_p, fp, ctypes.c_size_t]
        L.ope_dropin_get_fpn.restype = ctypes.c_longlong
        L.ope_dropin_backend.argtypes = [ctypes.c_void_p]
        L.ope_dropin_fft_precision.argtypes = [ctypes.c_int]
        L.ope_dropin_destroy.argtypes = [ctypes.c_void_p]
        L.ope_dropin_last_error.restype = ctypes.c_char_p
        _lib = L
    return _lib


def _fp(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def set_fft_precision(mode: str) -> None:
    """CPU backend's FFT shim: "f64" (exact DFT rounded once) or "f32" (radix-2)."""
    lib().ope_dropin_fft_precision({"f64": 0, "f32": 1}[mode])


class DropInProcessor:
    """One ope::Processor of the patched reference library."""

    def __init__(self, backend: int, p: RefParams):
        self.p = p
        self.h = lib().ope_dropin_create(int(backend), ctypes.byref(p))
        if not self.h:
            raise RuntimeError(f"ope::Processor(backend {backend}): {lib().ope_dropin_last_error().decode()}")

    @property
    def backend(self) -> int:
        return int(lib().ope_dropin_backend(self.h))

    def process(self, raw: np.ndarray, timeout_ms: int = 120000) -> np.ndarray:
        p = self.p
        m = p.ascans_per_bscan * p.bscans_per_buffer
        raw = np.ascontiguousarray(raw)
        out = np.zeros((m, p.signal_length // 2), np.float32)
        rc = lib().ope_dropin_process(self.h, raw.ctypes.data, _fp(out), timeout_ms)
        if rc != 0:
            raise RuntimeError(f"process: {lib().ope_dropin_last_error().decode()}")
        return out

    def request_fpn(self) -> None:
        lib().ope_dropin_request_fpn(self.h)

    def set_fpn(self, prof: np.ndarray) -> None:
        prof = np.ascontiguousarray(prof, np.float32)
        if lib().ope_dropin_set_fpn(self.h, _fp(prof), prof.size // 2) != 0:
            raise RuntimeError(lib().ope_dropin_last_error().decode())

    def fpn_profile(self) -> np.ndarray:
        n = lib().ope_dropin_get_fpn(self.h, None, 0)
        out = np.zeros(n, np.float32)
        if n:
            lib().ope_dropin_get_fpn(self.h, _fp(out), n)
        return out

    def close(self) -> None:
        if self.h:
            lib().ope_dropin_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
