"""Test helpers: oracle settings from a ChainSpec, the CPU emulation harness,
GPU runs through the C ABI and error strata in dB."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from octproengine_b200 import capi
from octproengine_b200.chain import ChainSpec, open_context, NUMPY_DTYPE, FLOAT32
from oracle import restate as R

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
EMU_SRC = os.path.join(HERE, "emu", "chain_emu.cpp")
EMU_LIB = os.path.join(HERE, "emu", "_build", "libchain_emu.so")
CSRC = os.path.join(ROOT, "octproengine_b200", "csrc")

IN_KIND = {1: 0, 2: 1, 3: 2, 9: 3}  # ope::DataType -> kernel input kind


class EmuArgs(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("in_kind", ctypes.c_int), ("interp", ctypes.c_int),
                ("m", ctypes.c_longlong), ("inp", ctypes.c_void_p), ("curve", ctypes.c_void_p),
                ("window", ctypes.c_void_p), ("cos_sin", ctypes.c_void_p), ("fpn", ctypes.c_void_p),
                ("dc_window", ctypes.c_int), ("log_scaling", ctypes.c_int), ("gmin", ctypes.c_float),
                ("gmax", ctypes.c_float), ("addend", ctypes.c_float), ("mult", ctypes.c_float),
                ("flip", ctypes.c_int), ("ascans_per_bscan", ctypes.c_int), ("bscans", ctypes.c_int),
                ("dc_split", ctypes.c_int), ("dc_ref_order", ctypes.c_int)]


def emu_lib():
    deps = [EMU_SRC, os.path.join(CSRC, "tables.cpp")] + [os.path.join(CSRC, f) for f in os.listdir(CSRC)
                                                          if f.endswith((".cuh", ".h"))]
    if not os.path.exists(EMU_LIB) or any(os.path.getmtime(d) > os.path.getmtime(EMU_LIB) for d in deps):
        os.makedirs(os.path.dirname(EMU_LIB), exist_ok=True)
        subprocess.run(["g++", "-O1", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off",
                        "-I/usr/local/cuda/include", EMU_SRC, os.path.join(CSRC, "tables.cpp"),
                        "-o", EMU_LIB], check=True)
    L = ctypes.CDLL(EMU_LIB)
    L.emu_chain.argtypes = [ctypes.POINTER(EmuArgs), ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    return L


def _ptr(a):
    return None if a is None else a.ctypes.data


def emu_run(L, spec: ChainSpec, raw: np.ndarray, what: str = "image", fpn=None) -> np.ndarray:
    """Runs the kernel's code on the CPU. what: image | fft_input | bins."""
    n, m = spec.signal_length, spec.num_ascans
    r, w, cs = spec.curves()
    interp = (spec.interpolation + 1) if spec.resampling else 0
    kind = IN_KIND[spec.input_dtype] if not (spec.input_dtype == FLOAT32 and spec.float32_as_uint32) else 2
    fp = None if fpn is None else np.ascontiguousarray(fpn, np.float32)
    raw = np.ascontiguousarray(raw)
    e = EmuArgs(n, kind, interp, m, _ptr(raw), _ptr(r), _ptr(w) if spec.windowing else None,
                _ptr(cs) if spec.dispersion else None, _ptr(fp),
                spec.dc_window if spec.dc_removal else 0, int(spec.log_scaling), spec.grayscale_min,
                spec.grayscale_max, spec.addend, spec.multiplicator, int(spec.bscan_flip),
                spec.ascans_per_bscan, spec.bscans_per_buffer, int(spec.dc_split), int(spec.dc_reference_order))
    code = {"image": 0, "fft_input": 1, "bins": 2, "resampled": 3}[what]
    if what == "resampled":
        out = np.zeros((m, n), np.float32)
        assert L.emu_chain(ctypes.byref(e), code, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))) == 0
        return out
    if what == "image":
        out = np.zeros((m, n // 2), np.float32)
    elif what == "fft_input":
        out = np.zeros((m, n, 2), np.float32)
    else:
        out = np.zeros((m, n // 2, 2), np.float32)
    rc = L.emu_chain(ctypes.byref(e), code, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    assert rc == 0
    if what == "image":
        return out
    return out[..., 0] + 1j * out[..., 1]


def oracle_settings(spec: ChainSpec):
    st = R.ChainSettings(
        n=spec.signal_length, dtype=spec.input_dtype, resampling=spec.resampling,
        interpolation=spec.interpolation, windowing=spec.windowing, dispersion=spec.dispersion,
        dc_removal=spec.dc_removal, dc_window=spec.dc_window, log_scaling=spec.log_scaling,
        grayscale_min=spec.grayscale_min, grayscale_max=spec.grayscale_max, addend=spec.addend,
        multiplicator=spec.multiplicator, fpn_removal=spec.fpn_removal,
        fpn_bscan_count=spec.fpn_bscan_count, ascans_per_bscan=spec.ascans_per_bscan,
        float_as_float=(spec.input_dtype == FLOAT32 and not spec.float32_as_uint32))
    r, w, cs = spec.curves()
    cur = R.Curves(r, w, cs[0::2].copy(), cs[1::2].copy())
    return st, cur


def oracle_image(spec: ChainSpec, raw, mode="ref", **kw):
    st, cur = oracle_settings(spec)
    return R.process_buffer(raw, st, cur, mode=mode, **kw)


def fpn_kappa(spec: ChainSpec, X64: np.ndarray, fpn) -> np.ndarray:
    """Fixed-pattern cancellation factor kappa = |X| / |X - F| per kept bin (X the
    float64 DFT bin, F the FPN profile as interleaved pairs); 1 without FPN."""
    half = spec.signal_length // 2
    if fpn is None:
        return np.ones((X64.shape[0], half))
    F = fpn[0::2].astype(np.float64) + 1j * fpn[1::2].astype(np.float64)
    with np.errstate(divide="ignore", invalid="ignore"):
        k = np.abs(X64[:, :half]) / np.abs(X64[:, :half] - F[None, :half])
    return np.nan_to_num(np.maximum(k, 1.0), nan=1.0, posinf=1e30)


def to_db(out: np.ndarray, spec: ChainSpec) -> np.ndarray:
    """Output units back to dB (log mode): dB = (out/mult - addend)*range + min."""
    rng = np.float32(spec.grayscale_max) - np.float32(spec.grayscale_min)
    if rng < 1e-6:
        rng = 1.0
    return (out.astype(np.float64) / spec.multiplicator - spec.addend) * float(rng) + spec.grayscale_min


def random_raw(spec: ChainSpec, seed: int = 0, scale: float = 3000.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    n, m = spec.signal_length, spec.num_ascans
    dt = NUMPY_DTYPE[spec.input_dtype]
    if dt == np.uint8:
        return np.clip(128 + rng.normal(0, scale / 256, (m, n)), 0, 255).astype(np.uint8)
    if dt == np.float32:
        return (32768 + rng.normal(0, scale, (m, n))).astype(np.float32)
    v = np.clip(32768 + rng.normal(0, scale, (m, n)), 0, 65535)
    return v.astype(dt)


def gpu_run(spec: ChainSpec, raw: np.ndarray, what: str = "image", ctx=None, fpn_request=False,
            fpn_profile=None):
    """Runs the chain on cuda:0 through the C ABI with device-resident buffers."""
    import torch
    n, m = spec.signal_length, spec.num_ascans
    own = ctx is None
    if own:
        ctx = open_context(spec)
    try:
        if fpn_profile is not None:
            ctx.set_fpn_profile(fpn_profile)
        if fpn_request:
            ctx.request_fpn_determination()
        raw_b = np.ascontiguousarray(raw).view(np.uint8).reshape(-1)
        d_in = torch.from_numpy(raw_b.copy()).to("cuda:0")
        stream = torch.cuda.current_stream().cuda_stream
        if what == "image":
            d_out = torch.empty((m, n // 2), dtype=torch.float32, device="cuda:0")
            ctx.process_device(d_in.data_ptr(), d_out.data_ptr(), stream, num_ascans=m)
        else:
            d_out = torch.empty((m, n // 2, 2), dtype=torch.float32, device="cuda:0")
            ctx.process_bins_device(d_in.data_ptr(), d_out.data_ptr(), m, stream)
        torch.cuda.synchronize()
        assert ctx.synchronize() == 0
        out = d_out.cpu().numpy()
        if what != "image":
            out = out[..., 0] + 1j * out[..., 1]
        return out
    finally:
        if own:
            ctx.close()


# ---------------------------------------------------------------- golden --
GOLDEN_DIR = os.path.join(HERE, "golden")


def golden_cases():
    """(name, ChainSpec, data) for every fixture made by tests/golden/make_golden.py."""
    from oracle.reflib import RefParams
    out = []
    for f in sorted(os.listdir(GOLDEN_DIR)):
        if not f.endswith(".npz"):
            continue
        d = dict(np.load(os.path.join(GOLDEN_DIR, f)))
        p = RefParams.from_buffer_copy(d["params"].tobytes())
        spec = ChainSpec(
            signal_length=p.signal_length, ascans_per_bscan=p.ascans_per_bscan,
            bscans_per_buffer=p.bscans_per_buffer, input_dtype=p.input_dtype,
            resampling=bool(p.resampling_enabled), interpolation=p.interpolation,
            resampling_coeffs=tuple(p.resampling_coeffs), windowing=bool(p.windowing_enabled),
            window_type=p.window_type, window_center=p.window_center, window_fill=p.window_fill,
            dispersion=bool(p.dispersion_enabled), dispersion_coeffs=tuple(p.dispersion_coeffs),
            dc_removal=bool(p.dc_removal_enabled), dc_window=p.dc_window, log_scaling=bool(p.log_scaling),
            grayscale_min=p.grayscale_min, grayscale_max=p.grayscale_max, addend=p.addend,
            multiplicator=p.multiplicator, fpn_removal=bool(p.fpn_removal), fpn_bscan_count=p.fpn_bscan_count)
        out.append((f[:-4], spec, d))
    return out
