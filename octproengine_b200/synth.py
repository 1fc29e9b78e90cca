"""Seeded synthetic spectral-domain OCT buffers.

The reference ships no dataset; its own tests synthesise spectra
(tests/test_backend_output_comparison.cpp:52-85). The generator here follows
the benchmark workloads of this backend: each raw A-scan is

    DC + background_b(n) + G(k~) * sum_j a_j cos(2 pi z_j k(n)/N + psi(k~)) + noise

with DC = 32768 counts, k(n) = n + 2e-5 n^2 - 1e-8 n^3 (a cubic non-linear
wavenumber map, in samples), k~ = k(n)/(N-1), a Gaussian source envelope G of
sigma 0.25 band centred on the band, five reflectors with depths uniform on
[20, 900] bins (undulating slowly across the B-scan) and amplitudes
log-uniform over 40 dB, dispersion psi = d2 (k~-1/2)^2 + d3 (k~-1/2)^3,
Gaussian noise of sigma 30 counts, clipped to [0, 65535] and rounded to the
requested sample type. An optional per-B-scan background row adds a fixed
pattern ripple of 0.5 % of DC amplitude.

:func:`linearising_coeffs` and :func:`compensating_coeffs` return the
reference-convention resampling and dispersion coefficients
(processorconfiguration.cpp:438-482, t = i/(N-1)) that undo k(n) and psi.
Generation runs in torch on any device so large buffers are made on the GPU.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np
import torch

K_COEFFS = (0.0, 1.0, 2e-5, -1e-8)


@dataclass
class SynthParams:
    n: int = 2048
    ascans: int = 512
    bscans: int = 1
    seed: int = 0
    dtype: str = "uint16"  # uint8 | uint16 | float32
    d2: float = 0.0
    d3: float = 0.0
    k_coeffs: tuple = K_COEFFS
    reflectors: int = 5
    amp_max: float = 6000.0
    noise_sigma: float = 30.0
    dc: float = 32768.0
    background_ripple: bool = False
    # When set, the wavenumber map is defined by its resampling curve instead of
    # k_coeffs: raw sample n carries wavenumber index k(n) = r^-1(n) with
    # r(t) = sum_m c_m t^m, t = j/(n-1) (the reference's resampling polynomial),
    # so resampling with exactly these coefficients linearises the spectrum.
    resampling_truth: Optional[tuple] = None


def k_map(n: int, coeffs=K_COEFFS) -> np.ndarray:
    x = np.arange(n, dtype=np.float64)
    return coeffs[0] + coeffs[1] * x + coeffs[2] * x ** 2 + coeffs[3] * x ** 3


def k_map_from_resampling(n: int, coeffs) -> np.ndarray:
    """Wavenumber index of each raw sample for a monotone resampling polynomial.

    r(j) = sum_m c_m (j/(n-1))^m gives the raw position at which wavenumber j
    is sampled; its inverse, evaluated on a 16x oversampled grid and linearly
    interpolated, gives k(n).
    """
    j = np.linspace(0.0, n - 1.0, 16 * (n - 1) + 1)
    t = j / (n - 1)
    r = sum(float(coeffs[m]) * t ** m for m in range(4))
    if np.any(np.diff(r) <= 0):
        raise ValueError("resampling polynomial is not monotone on [0, n-1]")
    return np.interp(np.arange(n, dtype=np.float64), r, j)


def linearising_coeffs(n: int, coeffs=K_COEFFS) -> tuple:
    """Resampling coefficients (c0..c3, over t = j/(n-1)) with k(r(j)) = j."""
    k = k_map(n, coeffs)
    j = np.arange(n, dtype=np.float64)
    r = np.interp(j, k, np.arange(n, dtype=np.float64))  # k is monotone on [0, n)
    t = j / (n - 1)
    A = np.stack([t ** p for p in range(4)], 1)
    sol, *_ = np.linalg.lstsq(A, r, rcond=None)
    return tuple(float(v) for v in sol)


class KmapFamily:
    """The resampling coefficients c0..c3 that linearise the wavenumber map
    k(n) = K0 + K1 n + K2 n^2 + K3 s n^3, as a function of the scale s of its
    cubic coefficient (the perturbation of the autofocus workload): one free
    physical parameter instead of four raw coefficients. Tabulated once on a
    fine grid of s and interpolated with cubic splines, so an evaluation costs
    microseconds on the host."""

    def __init__(self, n: int, coeffs=K_COEFFS, s_range=(0.5, 1.5), points: int = 401):
        from scipy.interpolate import CubicSpline
        self.n = n
        self.coeffs = tuple(coeffs)
        self.s = np.linspace(s_range[0], s_range[1], points)
        tab = np.array([linearising_coeffs(n, self.k_coeffs(s)) for s in self.s])
        self._spline = CubicSpline(self.s, tab, axis=0)

    def k_coeffs(self, s: float) -> tuple:
        c = list(self.coeffs)
        c[3] = c[3] * float(s)
        return tuple(c)

    def __call__(self, kappa) -> np.ndarray:
        return self._spline(float(np.asarray(kappa).reshape(-1)[0]))


def compensating_coeffs(d2: float, d3: float) -> tuple:
    """Dispersion coefficients (d0..d3 over t) whose phase equals psi(t).

    The reference multiplies the spectrum by exp(+i phase) and keeps bins
    [0, N/2) of an exp(+i) inverse DFT; those bins carry the exp(-i psi)
    component of a real fringe, so the compensating phase is +psi.
    psi(t) = d2 (t-1/2)^2 + d3 (t-1/2)^3 expanded in powers of t.
    """
    return (0.25 * d2 - 0.125 * d3, -d2 + 0.75 * d3, d2 - 1.5 * d3, d3)


def generate(p: SynthParams, device="cpu") -> torch.Tensor:
    """Returns a (bscans*ascans, n) tensor of the requested dtype on `device`."""
    rng = np.random.default_rng(p.seed)
    n, A, B = p.n, p.ascans, p.bscans
    M = A * B
    dev = torch.device(device)
    kn = k_map(n, p.k_coeffs) if p.resampling_truth is None else k_map_from_resampling(n, p.resampling_truth)
    k = torch.tensor(kn, dtype=torch.float64, device=dev)
    kt = k / (n - 1)
    env = torch.exp(-0.5 * ((kt - 0.5) / 0.25) ** 2)
    psi = p.d2 * (kt - 0.5) ** 2 + p.d3 * (kt - 0.5) ** 3
    z0 = rng.uniform(20.0, 900.0, size=(B, p.reflectors))
    amp = p.amp_max * 10.0 ** (-rng.uniform(0.0, 40.0, size=(B, p.reflectors)) / 20.0)
    ph0 = rng.uniform(0.0, 2 * np.pi, size=(B, p.reflectors))
    und = rng.uniform(0.0, 2 * np.pi, size=(B, p.reflectors))
    a_idx = np.arange(A)
    out = torch.empty((M, n), dtype={"uint8": torch.uint8, "uint16": torch.int32,
                                     "float32": torch.float32}[p.dtype], device=dev)
    gen = torch.Generator(device=dev)
    gen.manual_seed(p.seed * 7919 + 17)
    chunk = max(1, min(A, (1 << 24) // n))
    for b in range(B):
        bg = None
        if p.background_ripple:
            f = rng.uniform(50.0, 400.0)
            phi = rng.uniform(0, 2 * np.pi)
            bg = 0.005 * p.dc * torch.cos(2 * np.pi * f * torch.arange(n, device=dev, dtype=torch.float64) / n + phi)
        for a0 in range(0, A, chunk):
            a1 = min(A, a0 + chunk)
            aa = torch.tensor(a_idx[a0:a1], dtype=torch.float64, device=dev)[:, None]
            sig = torch.zeros((a1 - a0, n), dtype=torch.float64, device=dev)
            for j in range(p.reflectors):
                z = z0[b, j] + 8.0 * torch.sin(2 * np.pi * aa / A + und[b, j])
                sig += amp[b, j] * torch.cos(2 * np.pi * z * k[None, :] / n + psi[None, :] + ph0[b, j])
            x = p.dc + env[None, :] * sig
            if bg is not None:
                x = x + bg[None, :]
            x = x + p.noise_sigma * torch.randn((a1 - a0, n), generator=gen, device=dev, dtype=torch.float64)
            rows = slice(b * A + a0, b * A + a1)
            if p.dtype == "uint8":
                out[rows] = torch.clamp(torch.round(x / 256.0), 0, 255).to(torch.uint8)
            elif p.dtype == "uint16":
                out[rows] = torch.clamp(torch.round(x), 0, 65535).to(torch.int32)
            else:
                out[rows] = x.to(torch.float32)
    if p.dtype == "uint16":
        # torch has no unsigned 16-bit arithmetic on all devices: pack via int16 bits
        out = out.to(torch.int32)
        out = torch.where(out >= 32768, out - 65536, out).to(torch.int16)
    return out


def as_numpy(t: torch.Tensor, dtype: str) -> np.ndarray:
    a = t.cpu().numpy()
    if dtype == "uint16":
        return a.view(np.uint16)
    return a
