"""Numpy restatement of the reference per-A-scan chain. TEST INFRASTRUCTURE ONLY.

Every function names the reference code it restates (paths relative to the
reference project). Two precisions are offered for the chain:

* ``"ref"``  -- float32 arithmetic in the reference's own evaluation order for
  every stage before the inverse DFT (so the FFT input equals the reference's
  bit for bit), the unnormalised inverse DFT evaluated in float64 and rounded
  once to complex64 (what the FFTW-API shim computes in its default "f64"
  mode), then float32 magnitude / log10 / affine exactly as the reference.
* ``"f64"``  -- the same computation with all chain arithmetic in float64: the
  "truth" each float32 implementation is measured against. Curve tables
  (resampling positions, window, cos/sin of the phase) are the reference's
  float32 tables, treated as exact configuration data.

Parity pin: ``tests/test_oracle_pin.py`` checks this module against the
reference CPU backend compiled out of tree (``oracle/_ref``) and against the
golden fixtures in ``tests/golden``.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

F32 = np.float32

# C library float functions: the reference evaluates std::cos/std::sin/expf on
# float arguments, which resolve to libm's cosf/sinf/expf.
_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
for _name in ("cosf", "sinf", "expf", "log10f"):
    getattr(_libm, _name).restype = ctypes.c_float
    getattr(_libm, _name).argtypes = [ctypes.c_float]


def _cosf(x: float) -> F32:
    return F32(_libm.cosf(float(x)))


def _sinf(x: float) -> F32:
    return F32(_libm.sinf(float(x)))


def _expf(x: float) -> F32:
    return F32(_libm.expf(float(x)))


# reference enums (include/processorconfiguration.h:11-29, include/types.h:6-19)
LINEAR, CUBIC, LANCZOS = 0, 1, 2
HANN, GAUSS, SINE, LANCZOS_WIN, RECTANGULAR, FLAT_TOP = 0, 1, 2, 3, 4, 5
UINT8, UINT16, UINT32, FLOAT32 = 1, 2, 3, 9

_BITDEPTH = {1: 8, 2: 16, 3: 32, 4: 64, 5: 8, 6: 16, 7: 32, 8: 64, 9: 32, 10: 64, 11: 64, 12: 128}
_BYTES = {1: 1, 2: 2, 3: 4, 4: 8, 5: 1, 6: 2, 7: 4, 8: 8, 9: 4, 10: 8, 11: 8, 12: 16}


def bit_depth(dtype: int) -> int:
    """getDataTypeBitDepth (src/core/types.cpp:5-28)."""
    return _BITDEPTH.get(int(dtype), 0)


def byte_size(dtype: int) -> int:
    """getDataTypeByteSize (src/core/types.cpp:30-53)."""
    return _BYTES.get(int(dtype), 0)


# --------------------------------------------------------------------------
# curves (src/core/processorconfiguration.cpp:438-589, src/core/processor.cpp:77-99)
# --------------------------------------------------------------------------

def resampling_curve(n: int, coeffs) -> np.ndarray:
    """generateResamplingCurve (processorconfiguration.cpp:438-459).

    r(x) = c0 + x*(c1' + x*(c2' + x*c3')) in float32 with c_k' = c_k/(n-1)^k,
    clamped to [7, n-9] so a 16-tap Lanczos window stays inside the spectrum.
    """
    s1 = F32(F32(n) - F32(1.0))
    c0 = F32(coeffs[0])
    c1 = F32(F32(coeffs[1]) / s1)
    c2 = F32(F32(coeffs[2]) / F32(s1 * s1))
    c3 = F32(F32(coeffs[3]) / F32(F32(s1 * s1) * s1))
    x = np.arange(n, dtype=F32)
    val = c0 + x * (c1 + x * (c2 + x * c3))
    lo = F32(7.0)
    hi = F32(float((n - 9) % (1 << 64)))
    out = np.where(val < lo, lo, np.where(val > hi, hi, val)).astype(F32)
    return out


def dispersion_phase(n: int, coeffs) -> np.ndarray:
    """generateDispersionCurve (processorconfiguration.cpp:461-482).

    phase(i) = d0 + i*(d1' + i*(d2' + i*d3')) in float32, d_k' = d_k/(n-1)^k.
    The configured ``factor`` is never applied by the reference (processor.cpp:92-97).
    """
    den = F32(n - 1)
    d0 = F32(coeffs[0])
    d1 = F32(F32(coeffs[1]) / den)
    d2 = F32(F32(coeffs[2]) / F32(den * den))
    d3 = F32(F32(coeffs[3]) / F32(F32(den * den) * den))
    i = np.arange(n, dtype=F32)
    return (d0 + i * (d1 + i * (d2 + i * d3))).astype(F32)


def phase_to_cos_sin(phase: np.ndarray):
    """Processor::Impl::getDispersionCurve (processor.cpp:91-98): float cos/sin."""
    c = np.array([_cosf(p) for p in phase], dtype=F32)
    s = np.array([_sinf(p) for p in phase], dtype=F32)
    return c, s


def window_curve(n: int, wtype: int, center: float, fill: float) -> np.ndarray:
    """generateWindowCurve (processorconfiguration.cpp:484-589)."""
    size = n
    cpos = F32(center)
    if cpos > F32(1.0):
        cpos = F32(1.0)
    if cpos < F32(0.0):
        cpos = F32(0.0)
    fill32 = F32(fill)
    width = int(F32(fill32 * F32(size)))
    ctr = int(F32(cpos * F32(size)))
    min_pos = (ctr - width // 2) % (1 << 32)
    if min_pos >= (1 << 31):
        min_pos -= 1 << 32
    out = np.zeros(n, dtype=F32)
    wm1 = F32(F32(width) - F32(1.0))
    two_pi = 2.0 * math.pi
    for i in range(n):
        if wtype == GAUSS:
            xi = i - ctr
            xn = F32(F32(F32(xi) / F32(F32(size) - F32(1.0))) / fill32)
            out[i] = _expf(F32(F32(-10.0) * F32(xn * xn)))
            continue
        xi = i - min_pos
        xn = F32(F32(xi) / wm1)
        if xn > F32(0.999) or xn < F32(0.0001):
            out[i] = F32(0.0)
            continue
        if wtype == HANN:
            out[i] = F32(0.5 * (1.0 - math.cos(two_pi * float(xn))))
        elif wtype == SINE:
            out[i] = F32(math.sin(math.pi * float(xn)))
        elif wtype == LANCZOS_WIN:
            arg = F32(F32(F32(2.0) * xn) - F32(1.0))
            if arg == F32(0.0):
                out[i] = F32(1.0)
            else:
                out[i] = F32(math.sin(math.pi * float(arg)) / (math.pi * float(arg)))
        elif wtype == RECTANGULAR:
            out[i] = F32(1.0)
        elif wtype == FLAT_TOP:
            a0, a1, a2, a3, a4 = (F32(0.215578948), F32(0.416631580), F32(0.277263158),
                                  F32(0.083578947), F32(0.006947368))
            xd = float(xn)
            c1 = F32(math.cos(2.0 * math.pi * xd))
            c2 = F32(math.cos(4.0 * math.pi * xd))
            c3 = F32(math.cos(6.0 * math.pi * xd))
            c4 = F32(math.cos(8.0 * math.pi * xd))
            v = F32(a0 - F32(a1 * c1))
            v = F32(v + F32(a2 * c2))
            v = F32(v - F32(a3 * c3))
            v = F32(v + F32(a4 * c4))
            out[i] = v
        else:
            raise ValueError(f"unknown window type {wtype}")
    return out


# --------------------------------------------------------------------------
# per-A-scan stages (src/backends/cpu/cpu_kernels.tpp)
# --------------------------------------------------------------------------

def convert_input(raw: np.ndarray, dtype: int, n: int, float_as_float: bool = False) -> np.ndarray:
    """convertInputData (cpu_kernels.tpp:24-54): raw -> float32 rows (M, n).

    Bit depth <= 8 reads uint8, <= 16 reads uint16, otherwise uint32; so the
    reference reads FLOAT32 input as uint32 (a reference quirk). With
    ``float_as_float`` the bytes are read as float32 instead.
    """
    b = bit_depth(dtype)
    buf = np.ascontiguousarray(raw).view(np.uint8)
    if b <= 8:
        v = buf.view(np.uint8).astype(F32)
    elif b <= 16:
        v = buf.view(np.uint16).astype(F32)
    elif float_as_float and int(dtype) == FLOAT32:
        v = buf.view(np.float32).astype(F32)
    else:
        v = buf.view(np.uint32).astype(F32)
    return v.reshape(-1, n)


def dc_removal(x: np.ndarray, window: int, f64: bool = False) -> np.ndarray:
    """rollingAverageDCRemoval (cpu_kernels.tpp:56-82).

    Subtracts the mean of x[i-(W-1) .. min(i+W, n-1)]; the reference builds
    the window sums from a sequential float prefix sum, restated here with a
    sequential float32 accumulate (float64 in the truth mode).
    """
    dt = np.float64 if f64 else F32
    m, n = x.shape
    cs = np.zeros((m, n + 1), dtype=dt)
    cs[:, 1:] = np.cumsum(x.astype(dt), axis=1, dtype=dt)
    i = np.arange(n)
    start = np.where(i >= window - 1, i - (window - 1), 0)
    end = np.minimum(i + window, n - 1)
    s = cs[:, end + 1] - cs[:, start]
    cnt = (end - start + 1).astype(dt)
    return (x.astype(dt) - s / cnt).astype(dt)


def _clampi(v, n):
    return np.minimum(v, n - 1)


def klin_linear(x: np.ndarray, curve: np.ndarray, f64: bool = False) -> np.ndarray:
    """kLinearizationLinear (cpu_kernels.tpp:84-111): y1 + (y2-y1)*(nx-n1)."""
    dt = np.float64 if f64 else F32
    n = x.shape[1]
    nx = curve.astype(F32)
    n1 = _clampi(nx.astype(np.int32), n)
    n2 = _clampi(nx.astype(np.int32) + 1, n)
    t = (nx.astype(dt) - n1.astype(dt)).astype(dt)
    y1 = x[:, n1].astype(dt)
    y2 = x[:, n2].astype(dt)
    return (y1 + (y2 - y1) * t).astype(dt)


def klin_cubic(x: np.ndarray, curve: np.ndarray, f64: bool = False) -> np.ndarray:
    """kLinearizationCubic + cubicHermiteInterpolation (cpu_kernels.tpp:113-146,486-502)."""
    dt = np.float64 if f64 else F32
    n = x.shape[1]
    nx = curve.astype(F32)
    i1 = nx.astype(np.int32)
    n0 = _clampi(np.abs(i1 - 1), n)
    n1 = _clampi(i1, n)
    n2 = _clampi(i1 + 1, n)
    n3 = _clampi(i1 + 2, n)
    y0, y1, y2, y3 = (x[:, k].astype(dt) for k in (n0, n1, n2, n3))
    pos = (nx.astype(dt) - n1.astype(dt)).astype(dt)
    three, two, five, four, half = dt(3.0), dt(2.0), dt(5.0), dt(4.0), dt(0.5)
    a = (-y0 + three * (y1 - y2)) + y3
    b = ((two * y0 - five * y1) + four * y2) - y3
    c = -y0 + y2
    pos2 = pos * pos
    return ((half * pos) * ((a * pos2 + b * pos) + c) + y1).astype(dt)


def lanczos_taps(curve: np.ndarray, n: int, f64: bool = False):
    """Tap indices and weights of kLinearizationLanczos (cpu_kernels.tpp:148-196).

    Taps n0-7 .. n0+8 (n0 = (int)nx), clamped to [0, n-1]; weight
    lanczosKernel(nx - idx, 8) with |x| < 1e-5 -> 1 and |x| >= 8 -> 0.
    Returns (idx[16, n], w[16, n]).
    """
    nx = curve.astype(F32)
    n0 = nx.astype(np.int32)
    idx = np.empty((16, len(nx)), dtype=np.int64)
    w = np.empty((16, len(nx)), dtype=np.float64 if f64 else F32)
    pi32 = F32(math.pi)
    for t, i in enumerate(range(-7, 9)):
        k = np.clip(n0 + i, 0, n - 1)
        idx[t] = k
        for j in range(len(nx)):
            xv = F32(nx[j] - F32(k[j]))
            if f64:
                xd = float(xv)
                if abs(xd) < 1e-5:
                    w[t, j] = 1.0
                elif abs(xd) >= 8.0:
                    w[t, j] = 0.0
                else:
                    px = math.pi * xd
                    w[t, j] = (math.sin(px) / px) * (math.sin(px / 8.0) / (px / 8.0))
                continue
            if abs(xv) < F32(1e-5):
                w[t, j] = F32(1.0)
            elif abs(xv) >= F32(8.0):
                w[t, j] = F32(0.0)
            else:
                px = F32(pi32 * xv)
                pa = F32(px / F32(8.0))
                w[t, j] = F32(F32(_sinf(px) / px) * F32(_sinf(pa) / pa))
    return idx, w


def klin_lanczos(x: np.ndarray, curve: np.ndarray, taps=None, f64: bool = False) -> np.ndarray:
    """kLinearizationLanczos (cpu_kernels.tpp:165-196): sequential 16-tap sum."""
    dt = np.float64 if f64 else F32
    n = x.shape[1]
    idx, w = taps if taps is not None else lanczos_taps(curve, n, f64)
    acc = np.zeros((x.shape[0], len(curve)), dtype=dt)
    for t in range(16):
        acc = (acc + x[:, idx[t]].astype(dt) * w[t].astype(dt)).astype(dt)
    return acc


def inverse_dft(z: np.ndarray) -> np.ndarray:
    """computeIFFT (cpu_kernels.tpp:237-267): FFTW_BACKWARD, unnormalised.

    X[k] = sum_n z[n] exp(+2*pi*i*k*n/N), evaluated in float64.
    """
    n = z.shape[-1]
    return np.fft.ifft(z.astype(np.complex128), axis=-1) * n


def min_var_mean(X: np.ndarray, segments: int = 8, sequential: bool = True) -> np.ndarray:
    """getMinimumVarianceMean (cpu_kernels.tpp:402-458).

    X: (height, width) complex64 rows. Per column, over ``segments`` blocks of
    height//segments rows, pick the block mean with the smallest
    E|z|^2 - |E z|^2 (double accumulators, float results). Returns
    interleaved float32 (width*2).
    """
    height, width = X.shape
    seg_w = height // segments
    factor = F32(F32(1.0) / F32(seg_w))
    fd = float(factor)
    min_var = np.full(width, np.inf, dtype=F32)
    mx_best = np.zeros(width, dtype=F32)
    my_best = np.zeros(width, dtype=F32)
    for s in range(segments):
        rows = X[s * seg_w:(s + 1) * seg_w]
        dx = rows.real.astype(np.float64)
        dy = rows.imag.astype(np.float64)
        if sequential:
            sx = np.add.accumulate(dx, axis=0)[-1]
            sy = np.add.accumulate(dy, axis=0)[-1]
            sxx = np.add.accumulate(dx * dx + dy * dy, axis=0)[-1]
        else:
            sx, sy, sxx = dx.sum(0), dy.sum(0), (dx * dx + dy * dy).sum(0)
        mx = (sx * fd).astype(F32)
        my = (sy * fd).astype(F32)
        var = ((sxx * fd) - (mx.astype(np.float64) ** 2 + my.astype(np.float64) ** 2)).astype(F32)
        better = var < min_var
        min_var = np.where(better, var, min_var)
        mx_best = np.where(better, mx, mx_best)
        my_best = np.where(better, my, my_best)
    out = np.empty(2 * width, dtype=F32)
    out[0::2] = mx_best
    out[1::2] = my_best
    return out


def log_scale(X: np.ndarray, mult, gmin, gmax, addend, auto_minmax: bool, f64: bool = False) -> np.ndarray:
    """logScaleAndTruncate (cpu_kernels.tpp:301-341) on bins [0, N/2)."""
    dt = np.float64 if f64 else F32
    half = X.shape[1] // 2
    re = X[:, :half].real.astype(dt)
    im = X[:, :half].imag.astype(dt)
    mag2 = re * re + im * im
    with np.errstate(divide="ignore"):
        v = (dt(10.0) * np.log10(mag2 / dt(half))).astype(dt)
    if auto_minmax:
        lo = v.min(axis=1, keepdims=True)
        hi = v.max(axis=1, keepdims=True)
    else:
        lo = np.full((v.shape[0], 1), gmin, dtype=dt)
        hi = np.full((v.shape[0], 1), gmax, dtype=dt)
    rng = (hi - lo).astype(dt)
    rng = np.where(rng < dt(1e-6), dt(1.0), rng)
    return (dt(mult) * ((v - lo) / rng + dt(addend))).astype(dt)


def lin_scale(X: np.ndarray, mult, gmin, gmax, addend, f64: bool = False) -> np.ndarray:
    """linearScaleAndTruncate (cpu_kernels.tpp:343-378) on bins [0, N/2)."""
    dt = np.float64 if f64 else F32
    half = X.shape[1] // 2
    re = X[:, :half].real.astype(dt)
    im = X[:, :half].imag.astype(dt)
    mag = (np.sqrt(re * re + im * im) / dt(half)).astype(dt)
    rng = dt(gmax) - dt(gmin)
    if rng < dt(1e-6):
        rng = dt(1.0)
    return (dt(mult) * ((mag - dt(gmin)) / rng + dt(addend))).astype(dt)


# --------------------------------------------------------------------------
# the whole buffer (src/backends/cpu/cpu_backend.cpp:169-357)
# --------------------------------------------------------------------------

@dataclass
class Curves:
    """The three tables the backend receives (processor.cpp:102-125)."""
    resample: np.ndarray
    window: np.ndarray
    cos: np.ndarray
    sin: np.ndarray

    @staticmethod
    def generated(n, resampling_coeffs, window_type, window_center, window_fill, dispersion_coeffs):
        c, s = phase_to_cos_sin(dispersion_phase(n, dispersion_coeffs))
        return Curves(resampling_curve(n, resampling_coeffs),
                      window_curve(n, window_type, window_center, window_fill), c, s)


@dataclass
class ChainSettings:
    """The subset of ProcessorConfiguration (include/processorconfiguration.h:31-172)
    that the per-buffer chain reads."""
    n: int
    dtype: int = UINT16
    resampling: bool = False
    interpolation: int = LINEAR
    windowing: bool = False
    dispersion: bool = False
    dc_removal: bool = False
    dc_window: int = 64
    log_scaling: bool = True
    grayscale_min: float = 30.0
    grayscale_max: float = 100.0
    addend: float = 0.0
    multiplicator: float = 1.0
    fpn_removal: bool = False
    fpn_bscan_count: int = 1
    ascans_per_bscan: int = 512
    post_bg_removal: bool = False
    bg_weight: float = 1.0
    bg_offset: float = 0.0
    float_as_float: bool = False


@dataclass
class ChainResult:
    output: np.ndarray
    spectrum: Optional[np.ndarray] = None  # resampled, windowed, phase-multiplied (M, N) complex
    ifft: Optional[np.ndarray] = None      # (M, N) complex, before FPN subtraction
    fpn_profile: Optional[np.ndarray] = None
    bg_profile: Optional[np.ndarray] = None


def fft_input(raw, st: ChainSettings, curves: Curves, mode: str = "ref", lanczos=None) -> np.ndarray:
    """Stages 1-5 of processData (cpu_backend.cpp:184-230): the DFT input (M, N) complex."""
    f64 = mode == "f64"
    dt = np.float64 if f64 else F32
    x = convert_input(raw, st.dtype, st.n, st.float_as_float).astype(dt)
    if st.dc_removal:
        x = dc_removal(x, st.dc_window, f64)
    if st.resampling:
        if st.interpolation == LINEAR:
            x = klin_linear(x, curves.resample, f64)
        elif st.interpolation == CUBIC:
            x = klin_cubic(x, curves.resample, f64)
        else:
            x = klin_lanczos(x, curves.resample, lanczos, f64)
    if st.windowing:
        x = (x * curves.window.astype(dt)).astype(dt)
    if st.dispersion:
        re = (x * curves.cos.astype(dt)).astype(dt)
        im = (x * curves.sin.astype(dt)).astype(dt)
    else:
        re, im = x, np.zeros_like(x)
    ct = np.complex128 if f64 else np.complex64
    z = np.empty(x.shape, dtype=ct)
    z.real, z.imag = re, im
    return z


def process_buffer(raw, st: ChainSettings, curves: Curves, mode: str = "ref",
                   fpn_profile: Optional[np.ndarray] = None, determine_fpn: bool = False,
                   bg_profile: Optional[np.ndarray] = None, record_bg: bool = False,
                   lanczos=None, keep: bool = False) -> ChainResult:
    """CpuBackend::Impl::processData (cpu_backend.cpp:169-302), one buffer.

    FPN: when ``determine_fpn`` the profile is the minimum-variance mean over
    the first fpn_bscan_count*ascans_per_bscan A-scans of this buffer
    (computeFixedPatternNoiseIfRequested, cpu_backend.cpp:305-357, for the
    first buffer processed), and is then subtracted from this same buffer.
    """
    f64 = mode == "f64"
    z = fft_input(raw, st, curves, mode, lanczos)
    X = inverse_dft(z)
    if not f64:
        X = X.astype(np.complex64)
    res = ChainResult(output=None)
    if determine_fpn:
        req = st.fpn_bscan_count * st.ascans_per_bscan
        if X.shape[0] >= req:
            mv = min_var_mean(X[:req].astype(np.complex64) if not f64 else X[:req], 8)
            fpn_profile = mv[: 2 * (st.n // 2)]
            res.fpn_profile = fpn_profile
    Y = X
    if st.fpn_removal and fpn_profile is not None and len(fpn_profile) > 0:
        half = st.n // 2
        pairs = min(half, len(fpn_profile) // 2)
        dt = np.float64 if f64 else F32
        m = np.asarray(fpn_profile, dtype=F32)
        Y = X.copy()
        Y[:, :pairs] = ((X[:, :pairs].real - m[0:2 * pairs:2].astype(dt))
                        + 1j * (X[:, :pairs].imag - m[1:2 * pairs:2].astype(dt)))
    if st.log_scaling:
        auto = st.grayscale_min == st.grayscale_max
        out = log_scale(Y, st.multiplicator, st.grayscale_min, st.grayscale_max, st.addend, auto, f64)
    else:
        out = lin_scale(Y, st.multiplicator, st.grayscale_min, st.grayscale_max, st.addend, f64)
    if st.post_bg_removal:
        dt = np.float64 if f64 else F32
        if record_bg:
            acc = np.zeros(out.shape[1], dtype=dt)
            for a in range(out.shape[0]):
                acc = (acc + out[a]).astype(dt)
            bg_profile = (acc / dt(out.shape[0])).astype(dt)
            res.bg_profile = bg_profile
        if bg_profile is not None and len(bg_profile) > 0:
            bgv = (dt(st.bg_weight) * np.asarray(bg_profile, dtype=dt) + dt(st.bg_offset)).astype(dt)
            out = (out - bgv[None, :]).astype(dt)
    res.output = out
    if keep:
        res.spectrum = z
        res.ifft = X
    return res


# --------------------------------------------------------------------------
# sinusoidal scan correction: the reference CUDA backend only
# (cuda_kernels.cu:408-438, applied at cuda_backend.cu:696-706); the CPU
# backend has no such step, so this restates the CUDA kernels.
# --------------------------------------------------------------------------

def sinusoidal_curve(length: int) -> np.ndarray:
    """fillSinusoidalScanCorrectionCurve: (L/pi) acos(1 - 2k/L), float acos."""
    k = np.arange(length, dtype=np.float64)
    arg = (1.0 - (2.0 * k.astype(F32).astype(np.float64)) / float(F32(length))).astype(F32)
    ac = np.arccos(arg).astype(F32).astype(np.float64)
    return ((float(F32(length)) / math.pi) * ac).astype(F32)


def sinusoidal_correction(img: np.ndarray, ascans_per_bscan: int, curve: Optional[np.ndarray] = None) -> np.ndarray:
    """sinusoidalScanCorrection on a (A-scans, bins) float32 image: A-scan k of
    each B-scan interpolates between input A-scans (int)x and (int)x + 1 of the
    same flat buffer (x = curve[k]); the last A-scan of the buffer is kept. The
    interpolation is one fused multiply-add (f1 - f0) * frac + f0, rounded once
    (evaluated exactly in float64)."""
    m, width = img.shape
    h = ascans_per_bscan
    if curve is None:
        curve = sinusoidal_curve(h)
    flat = img.reshape(-1).astype(F32)
    out = flat.copy()
    idx = np.arange(m * width - width, dtype=np.int64)
    j = idx % width
    k = (idx // width) % h
    l = idx // (width * h)
    x = curve[k].astype(F32)
    xi = x.astype(np.int32).astype(np.int64)
    x0 = xi * width + j + l * width * h
    f0 = flat[x0]
    f1 = flat[x0 + width]
    frac = (x - xi.astype(F32)).astype(F32)
    d = (f1 - f0).astype(F32)
    out[idx] = (d.astype(np.float64) * frac.astype(np.float64) + f0.astype(np.float64)).astype(F32)
    return out.reshape(m, width)
