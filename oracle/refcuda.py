"""ctypes access to the reference CUDA backend built out of tree. COMPARISON ONLY.

``_ref/libope_cuda_ref.so`` is built by ``make -C oracle cuda`` from the
reference sources (src/backends/cuda/{cuda_backend,cuda_kernels}.cu with the
reference's default flags --use_fast_math and real sm_100 code, the three
src/core files) plus ``ref_cuda_driver.cpp``. Its DFT is cuFFT, a closed
library, so it is a baseline to compare speed and accuracy with, not an oracle.
Only tests and the reference arm of the benchmark use it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

from oracle.reflib import RefParams, REFERENCE_TREE, make_params  # noqa: F401  (re-exported)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libope_cuda_ref.so")

_lib: Optional[ctypes.CDLL] = None


def build(force: bool = False) -> bool:
    """Compile (or bring up to date) the reference CUDA backend when the
    reference tree is named by OPE_REFERENCE_TREE; otherwise use the prebuilt
    library."""
    if REFERENCE_TREE and os.path.isdir(REFERENCE_TREE):
        subprocess.run(["make", "-C", HERE, f"REF={REFERENCE_TREE}", "cuda"] + (["-B"] if force else []),
                       check=True, stdout=subprocess.DEVNULL)
    return os.path.exists(LIB_PATH)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(f"reference CUDA backend not built: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER(RefParams)
        fp = ctypes.POINTER(ctypes.c_float)
        L.ope_refcuda_last_error.restype = ctypes.c_char_p
        L.ope_refcuda_create.argtypes = [P, ctypes.c_int]
        L.ope_refcuda_create.restype = ctypes.c_void_p
        L.ope_refcuda_process.argtypes = [ctypes.c_void_p, ctypes.c_void_p, fp, ctypes.c_int]
        L.ope_refcuda_request_fpn.argtypes = [ctypes.c_void_p]
        L.ope_refcuda_set_fpn.argtypes = [ctypes.c_void_p, fp, ctypes.c_size_t]
        L.ope_refcuda_fill_inputs.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.ope_refcuda_stream.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_double)]
        L.ope_refcuda_destroy.argtypes = [ctypes.c_void_p]
        _lib = L
    return _lib


def _err() -> str:
    m = lib().ope_refcuda_last_error()
    return m.decode() if m else ""


class RefCudaBackend:
    """One reference CudaBackend with generated curves (device 0)."""

    def __init__(self, p: RefParams, num_input_buffers: int = 2):
        self.p = p
        self.h = lib().ope_refcuda_create(ctypes.byref(p), num_input_buffers)
        if not self.h:
            raise RuntimeError(f"reference CUDA backend creation failed: {_err()}")

    def process(self, raw: np.ndarray, timeout_ms: int = 120000) -> np.ndarray:
        """One frame through the ring, blocking until its output callback."""
        p = self.p
        out = np.zeros(p.signal_length * p.ascans_per_bscan * p.bscans_per_buffer // 2, np.float32)
        raw = np.ascontiguousarray(raw)
        rc = lib().ope_refcuda_process(self.h, raw.ctypes.data_as(ctypes.c_void_p),
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), timeout_ms)
        if rc != 0:
            raise RuntimeError(f"reference CUDA process failed ({rc}): {_err()}")
        return out.reshape(-1, p.signal_length // 2)

    def request_fpn(self) -> None:
        lib().ope_refcuda_request_fpn(self.h)

    def set_fpn(self, prof: np.ndarray) -> None:
        d = np.ascontiguousarray(prof, dtype=np.float32)
        rc = lib().ope_refcuda_set_fpn(self.h, d.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), d.size // 2)
        if rc != 0:
            raise RuntimeError(f"reference CUDA set_fpn failed ({rc}): {_err()}")

    def fill_inputs(self, raw: np.ndarray) -> None:
        raw = np.ascontiguousarray(raw)
        if lib().ope_refcuda_fill_inputs(self.h, raw.ctypes.data_as(ctypes.c_void_p)) != 0:
            raise RuntimeError(f"reference CUDA fill_inputs failed: {_err()}")

    def stream(self, frames: int, timeout_ms: int = 300000) -> float:
        """Pushes `frames` buffers back to back through the ring; wall seconds to the last callback."""
        sec = ctypes.c_double(0.0)
        rc = lib().ope_refcuda_stream(self.h, frames, timeout_ms, ctypes.byref(sec))
        if rc != 0:
            raise RuntimeError(f"reference CUDA stream failed ({rc}): {_err()}")
        return sec.value

    def close(self) -> None:
        if self.h:
            lib().ope_refcuda_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
