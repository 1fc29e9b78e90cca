"""Float64 reference of the differentiable chain. TEST INFRASTRUCTURE ONLY.

Restates, in float64 torch with autograd, the chain that the autofocus kernels
differentiate (octproengine_b200/csrc/autofocus.cuh), following the reference
CPU backend stage by stage:

* resampling position r(j) = sum_m c_m t^m, t = j/(N-1), clamped to [7, N-9]
  (ProcessorConfiguration::generateResamplingCurve, processorconfiguration.cpp:438-459);
* the integer mean of each A-scan subtracted (the exact DC split of the chain,
  with nothing added back);
* kLinearizationLinear / kLinearizationCubic (with n0 = |n1 - 1|) /
  kLinearizationLanczos with the a = 8 kernel (cpu_kernels.tpp:84-196);
* window, then exp(i phi), phi(j) = sum_m d_m t^m
  (generateDispersionCurve, processorconfiguration.cpp:461-482;
  applyWindow + dispersionCompensation, cpu_kernels.tpp:198-235);
* the unnormalised exp(+i) inverse DFT, bins [0, N/2) (cpu_kernels.tpp:237-267);
* intensity |X|^2, 10 log10(|X|^2/(N/2)), or the Shannon entropy of the
  normalised intensity.

Torch's autograd of this float64 code is the reference gradient the GPU
adjoint is checked against; it is never used by the product path.
"""
from __future__ import annotations

import numpy as np
import torch

F64 = torch.float64
LINEAR, CUBIC, LANCZOS = 0, 1, 2


def _lanczos8(x: torch.Tensor) -> torch.Tensor:
    """lanczosKernel(x, 8) (cpu_kernels.tpp:148-162): sinc(x) sinc(x/8) on |x| < 8, 1 near 0."""
    v = torch.sinc(x) * torch.sinc(x / 8.0)
    v = torch.where(x.abs() < 1e-5, torch.ones_like(v), v)
    return torch.where(x.abs() >= 8.0, torch.zeros_like(v), v)


def centred_mean_removed(raw: np.ndarray) -> torch.Tensor:
    """x - c with c the A-scan mean rounded to an integer (exact for integer samples)."""
    x = torch.as_tensor(np.asarray(raw, dtype=np.float64))
    if np.issubdtype(np.asarray(raw).dtype, np.integer):
        c = torch.round(x.sum(1, keepdim=True) / x.shape[1])
    else:
        c = x.mean(1, keepdim=True)
    return x - c


def _f32_horner(coeffs: torch.Tensor, n: int) -> torch.Tensor:
    """The polynomial as the reference evaluates it: float32 Horner in j with
    coefficients divided by (n-1)^m (processorconfiguration.cpp:438-482)."""
    c = coeffs.detach().numpy().astype(np.float32)
    s1 = np.float32(np.float32(n) - np.float32(1.0))
    k1 = np.float32(c[1] / s1)
    k2 = np.float32(c[2] / np.float32(s1 * s1))
    k3 = np.float32(c[3] / np.float32(np.float32(s1 * s1) * s1))
    x = np.arange(n, dtype=np.float32)
    v = (np.float32(c[0]) + x * (k1 + x * (k2 + x * k3))).astype(np.float32)
    return torch.as_tensor(v.astype(np.float64))


def chain_bins(x: torch.Tensor, params: torch.Tensor, window: torch.Tensor, interp: int,
               f32_curves: bool = True) -> torch.Tensor:
    """Complex bins [0, N/2) of every A-scan of x (float64, mean removed).

    With f32_curves the resampling positions and the phase take the
    reference's float32 values (configuration data), with float64 derivatives
    for autograd; without, everything is float64 (smooth in the parameters,
    for finite-difference checks of this module).
    """
    M, N = x.shape
    t = torch.arange(N, dtype=F64) / (N - 1)
    d, c = params[:4], params[4:]
    r = c[0] + t * (c[1] + t * (c[2] + t * c[3]))
    if f32_curves:
        r = r + (_f32_horner(c, N) - r).detach()
    r = r.clamp(7.0, N - 9.0)
    n1 = torch.floor(r.detach()).long()
    if interp == LINEAR:
        y1, y2 = x[:, n1], x[:, (n1 + 1).clamp(max=N - 1)]
        y = y1 + (y2 - y1) * (r - n1)
    elif interp == CUBIC:
        y0 = x[:, (n1 - 1).abs().clamp(max=N - 1)]
        y1, y2, y3 = x[:, n1], x[:, (n1 + 1).clamp(max=N - 1)], x[:, (n1 + 2).clamp(max=N - 1)]
        pos = r - n1
        a = -y0 + 3.0 * (y1 - y2) + y3
        b = 2.0 * y0 - 5.0 * y1 + 4.0 * y2 - y3
        cc = y2 - y0
        y = 0.5 * pos * (a * pos * pos + b * pos + cc) + y1
    else:
        y = 0.0
        for k in range(16):
            idx = (n1 - 7 + k).clamp(0, N - 1)
            y = y + x[:, idx] * _lanczos8(r - idx.to(F64))
    phi = d[0] + t * (d[1] + t * (d[2] + t * d[3]))
    if f32_curves:
        phi = phi + (_f32_horner(d, N) - phi).detach()
    z = (y * window) * torch.exp(1j * phi)
    return torch.fft.ifft(z, dim=1)[:, : N // 2] * N


def intensity(raw: np.ndarray, params, window, interp: int, requires_grad: bool = False, f32_curves: bool = True):
    p = torch.as_tensor(np.asarray(params, np.float64)).clone().requires_grad_(requires_grad)
    w = torch.as_tensor(np.asarray(window, np.float64))
    X = chain_bins(centred_mean_removed(raw), p, w, interp, f32_curves)
    return X.real ** 2 + X.imag ** 2, p


def entropy_of(I: torch.Tensor) -> torch.Tensor:
    S = I.sum()
    p = I / S
    return -(torch.where(p > 0, p * torch.log(p), torch.zeros_like(p))).sum()


def entropy_and_grad(raw: np.ndarray, params, window, interp: int, f32_curves: bool = True):
    """(H, dH/dparams) in float64."""
    I, p = intensity(raw, params, window, interp, requires_grad=True, f32_curves=f32_curves)
    H = entropy_of(I)
    (g,) = torch.autograd.grad(H, p)
    return float(H), g.numpy()


def image_grad(raw: np.ndarray, params, window, interp: int, grad_out: np.ndarray, db: bool = False):
    """d/dparams of sum(grad_out * image), image = I or 10 log10(I/(N/2))."""
    I, p = intensity(raw, params, window, interp, requires_grad=True)
    img = 10.0 * torch.log10(I / (I.shape[1])) if db else I
    L = (img * torch.as_tensor(np.asarray(grad_out, np.float64))).sum()
    (g,) = torch.autograd.grad(L, p)
    return g.numpy()
