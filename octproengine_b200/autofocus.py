"""Differentiable OCT chain and gradient autofocus on B200.

The reference sets dispersion and k-linearisation coefficients by hand
(Processor::setDispersionCoefficients / setResamplingCoefficients,
src/core/processor.cpp:371-470); the usual way to find them is a parameter
sweep of the whole chain. Here the chain is differentiable: the hand-written
adjoint kernels behind ``ope_b200_af_backward`` (octproengine_b200/csrc/
autofocus.cuh) give the gradient of an image objective with respect to the
8 chain parameters

    params = (d0, d1, d2, d3, c0, c1, c2, c3)

-- the dispersion polynomial and the resampling polynomial in the reference's
convention (processorconfiguration.cpp:438-482, t = j/(N-1)) -- so autofocus
becomes a gradient fit.

* :class:`Autofocus` -- one ``ope_b200_af`` handle (signal length, input type,
  interpolation, window) with raw forward / adjoint calls on device tensors;
* :class:`ChainImage` and :class:`ChainEntropy` -- ``torch.autograd.Function``
  wrappers: the image (intensity or dB) or the Shannon entropy of the
  normalised intensity, differentiable with respect to ``params``;
* :func:`fit_dispersion` -- BFGS on (d2, d3) of the centred dispersion phase
  psi(t) = d2 (t-1/2)^2 + d3 (t-1/2)^3, entropy objective;
* :func:`fit_dispersion_kmap` -- BFGS on (d2, d3) and the parameters of a
  k-map family (the resampling coefficients as a function of a few physical
  parameters), with the full adjoint's k-map gradient;
* :func:`grid_sweep` -- the parameter sweep it replaces, every grid point one
  launch of the same forward chain, all enqueued back to back.

Everything runs on the GPU through the C ABI; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np
import torch

from . import capi

OUT_INTENSITY = 1
OUT_DB = 2
LINEAR, CUBIC, LANCZOS = 0, 1, 2  # ope::InterpolationMethod

_DTYPES = {"uint8": 1, "uint16": 2, "float32": 9}  # ope::DataType
_TORCH_DTYPES = {"uint8": torch.uint8, "uint16": torch.int16, "float32": torch.float32}

# psi(t) = d2 (t-1/2)^2 + d3 (t-1/2)^3 expanded in powers of t: d = M @ (d2, d3)
CENTRED_TO_POLY = np.array([[0.25, -0.125], [-1.0, 0.75], [1.0, -1.5], [0.0, 1.0]])


def dispersion_poly(d2: float, d3: float) -> np.ndarray:
    """Reference-convention dispersion coefficients of the centred (d2, d3)."""
    return CENTRED_TO_POLY @ np.array([d2, d3], dtype=np.float64)


def _ptr(t: Optional[torch.Tensor]):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


_CAI_TYPES = {torch.uint8: "|u1", torch.int16: "<i2", torch.float32: "<f4"}


class _DeviceMemory:
    """Device memory owned elsewhere, described by the CUDA array interface."""

    def __init__(self, ptr: int, shape, dtype: torch.dtype):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": _CAI_TYPES[dtype],
                                         "data": (int(ptr), False), "version": 2, "strides": None}


def frame_input_view(ctx, ticket: int, ascans: int, stream=None) -> torch.Tensor:
    """The first `ascans` raw A-scans of a submitted ring frame, as a device
    tensor over the ring slot's own copy (no transfer). `stream` (default: the
    current one) waits for the frame's input copy. The view is valid until
    the frame is released; work reading it must have finished by then."""
    if stream is None:
        stream = torch.cuda.current_stream()
    ptr = ctx.frame_device_input(ticket, stream.cuda_stream)
    dtype = {1: torch.uint8, 2: torch.int16, 9: torch.float32}[ctx.cfg.input_dtype]
    return torch.as_tensor(_DeviceMemory(ptr, (ascans, ctx.cfg.signal_length), dtype),
                           device=torch.device("cuda", ctx.cfg.device))


def _stream(stream) -> ctypes.c_void_p:
    if stream is None:
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Autofocus:
    """The differentiable chain for one geometry: N samples per A-scan, one
    input type, one interpolation, one window. One handle serves one stream
    at a time (its device tables and partial sums are shared by its calls)."""

    def __init__(self, n: int, input_dtype: str = "uint16", interpolation: int = LANCZOS,
                 window: Optional[np.ndarray] = None, device: int = 0, bitshift: bool = False):
        if input_dtype not in _DTYPES:
            raise ValueError(f"input_dtype must be one of {sorted(_DTYPES)}")
        self.n = int(n)
        self.input_dtype = input_dtype
        self.interpolation = int(interpolation)
        self.device = torch.device("cuda", device)
        h = ctypes.c_void_p()
        w = None
        if window is not None:
            self._window = np.ascontiguousarray(window, np.float32)
            if self._window.size != self.n:
                raise ValueError("window must have N values")
            w = capi.fptr(self._window)
        rc = capi.lib().ope_b200_af_create(self.n, _DTYPES[input_dtype], self.interpolation, w, device,
                                           ctypes.byref(h))
        if rc != capi.OK:
            raise capi.B200Error(rc, f"autofocus handle for N={n}, {input_dtype}, interpolation {interpolation}")
        self.h = h
        if bitshift:  # DataParameters::bitshift: 8/16-bit samples >> 4, as the chain applies it
            self._check(capi.lib().ope_b200_af_set_bitshift(self.h, 1))

    def close(self) -> None:
        if getattr(self, "h", None):
            capi.lib().ope_b200_af_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int) -> None:
        if rc != capi.OK:
            raise capi.B200Error(rc, capi.lib().ope_b200_af_last_error(self.h).decode())

    def _check_raw(self, raw: torch.Tensor) -> int:
        if raw.device.type != "cuda" or raw.dtype != _TORCH_DTYPES[self.input_dtype]:
            raise TypeError(f"raw must be a CUDA tensor of {_TORCH_DTYPES[self.input_dtype]}")
        if raw.dim() != 2 or raw.shape[1] != self.n or not raw.is_contiguous():
            raise ValueError(f"raw must be a contiguous (A-scans, {self.n}) tensor")
        return raw.shape[0]

    @staticmethod
    def _check_params(params: torch.Tensor) -> None:
        if params.device.type != "cuda" or params.dtype != torch.float32 or params.numel() != 8:
            raise TypeError("params must be a CUDA float32 tensor of 8 values (d0..d3, c0..c3)")

    def forward(self, raw: torch.Tensor, params: torch.Tensor, output: int = OUT_INTENSITY,
                out: Optional[torch.Tensor] = None, hs: Optional[torch.Tensor] = None, stream=None) -> None:
        """Image (``out``, A-scans x N/2 float32) and/or (H, S) (``hs``, 2 float64)."""
        m = self._check_raw(raw)
        self._check_params(params)
        self._check(capi.lib().ope_b200_af_forward(self.h, _ptr(raw), m, _ptr(params), output, _ptr(out), _ptr(hs),
                                                   _stream(stream)))

    def backward(self, raw: torch.Tensor, params: torch.Tensor, grad: torch.Tensor,
                 grad_out: Optional[torch.Tensor] = None, hs: Optional[torch.Tensor] = None,
                 output: int = OUT_INTENSITY, stream=None, dispersion_only: bool = False) -> None:
        """dL/dparams into ``grad`` (8 float32): L = sum(grad_out * image) or L = H.
        ``dispersion_only``: d0..d3 only (the k-map entries are 0), a cheaper adjoint."""
        m = self._check_raw(raw)
        self._check_params(params)
        if grad_out is not None and (grad_out.dtype != torch.float32 or not grad_out.is_contiguous()
                                     or grad_out.shape != (m, self.n // 2)):
            raise ValueError("grad_out must be a contiguous float32 (A-scans, N/2) tensor")
        f = capi.lib().ope_b200_af_backward_dispersion if dispersion_only else capi.lib().ope_b200_af_backward
        self._check(f(self.h, _ptr(raw), m, _ptr(params), output, _ptr(grad_out), _ptr(hs), _ptr(grad),
                      _stream(stream)))


class ChainImage(torch.autograd.Function):
    """image = chain(raw; params): intensity |X|^2 or 10 log10(|X|^2/(N/2))."""

    @staticmethod
    def forward(ctx, raw, params, af: Autofocus, output: int = OUT_INTENSITY):
        p = params.detach().contiguous()
        out = torch.empty((raw.shape[0], af.n // 2), dtype=torch.float32, device=raw.device)
        af.forward(raw, p, output=output, out=out)
        ctx.save_for_backward(raw, p)
        ctx.af, ctx.output = af, output
        return out

    @staticmethod
    def backward(ctx, g):
        raw, p = ctx.saved_tensors
        grad = torch.empty(8, dtype=torch.float32, device=raw.device)
        ctx.af.backward(raw, p, grad, grad_out=g.contiguous().float(), output=ctx.output)
        return None, grad, None, None


class ChainEntropy(torch.autograd.Function):
    """H(params) = -sum p ln p, p = I / sum I over every bin of every A-scan."""

    @staticmethod
    def forward(ctx, raw, params, af: Autofocus):
        p = params.detach().contiguous()
        hs = torch.empty(2, dtype=torch.float64, device=raw.device)
        af.forward(raw, p, hs=hs)
        ctx.save_for_backward(raw, p, hs)
        ctx.af = af
        return hs[0].clone()

    @staticmethod
    def backward(ctx, g):
        raw, p, hs = ctx.saved_tensors
        grad = torch.empty(8, dtype=torch.float32, device=raw.device)
        ctx.af.backward(raw, p, grad, hs=hs)
        return None, grad * g.to(torch.float32), None


@dataclass
class FitResult:
    d2: float
    d3: float
    entropy: float
    iterations: int
    evaluations: int
    seconds: float
    history: list = field(default_factory=list)  # (d2, d3, H, seconds since start) per iteration


class FitEvaluator:
    """H and dH/d(d2, d3) at a point, one host round trip per evaluation.

    With ``graph`` the whole evaluation (parameter upload from pinned host
    memory, forward, adjoint, result download) is captured once in a CUDA
    graph and replayed, so an evaluation costs one graph launch and one
    synchronisation on the host. One evaluator serves any number of fits on
    the same device tensor (new data copied into it between fits), so the graph
    capture, and the device-wide synchronisation that torch performs when a
    capture begins, happen once rather than once per fit. The 80 bytes of
    parameters and results move
    by a small kernel (ope_b200_af_small_copy) rather than by copy-engine DMA,
    so an evaluation does not wait behind bulk transfers that other streams
    have queued on the copy engines (frames streaming through a ring).
    """

    def __init__(self, af: Autofocus, raw: torch.Tensor, kmap: Sequence[float], graph: bool = True):
        self.af, self.raw = af, raw
        dev = raw.device
        self.kmap = np.asarray(kmap, np.float32)
        self.h_params = torch.empty(8, dtype=torch.float32, pin_memory=True)
        self.d_params = torch.empty(8, dtype=torch.float32, device=dev)
        self.d_hs = torch.empty(2, dtype=torch.float64, device=dev)
        self.d_grad = torch.empty(8, dtype=torch.float32, device=dev)
        self.h_hs = torch.empty(2, dtype=torch.float64, pin_memory=True)
        self.h_grad = torch.empty(8, dtype=torch.float32, pin_memory=True)
        self.count = 0
        self.graph = None
        L = capi.lib()
        self.sm_copies = all(L.ope_b200_af_kernel_accessible(_ptr(t)) == 1 for t in
                             (self.h_params, self.d_params, self.h_hs, self.d_hs, self.h_grad, self.d_grad))
        self._set(np.zeros(2))
        if graph:
            side = torch.cuda.Stream(dev)
            side.wait_stream(torch.cuda.current_stream(dev))
            with torch.cuda.stream(side):
                self._enqueue(side)  # warm-up outside the capture
            side.synchronize()
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph, stream=side):
                self._enqueue(side)
        self.stream = torch.cuda.current_stream(dev)

    def _set(self, theta) -> None:
        hp = self.h_params.numpy()
        hp[:4] = dispersion_poly(theta[0], theta[1])
        hp[4:] = self.kmap

    def _copy(self, dst: torch.Tensor, src: torch.Tensor, stream) -> None:
        if not self.sm_copies:
            dst.copy_(src, non_blocking=True)
            return
        rc = capi.lib().ope_b200_af_small_copy(_ptr(dst), _ptr(src), src.numel() * src.element_size(),
                                               _stream(stream))
        if rc != capi.OK:
            raise capi.B200Error(rc, "small copy failed")

    def _enqueue(self, stream) -> None:
        self._copy(self.d_params, self.h_params, stream)
        self.af.forward(self.raw, self.d_params, hs=self.d_hs, stream=stream)
        # the gradient's finalize kernel writes straight into page-locked host memory
        grad = self.h_grad if self.sm_copies else self.d_grad
        self.af.backward(self.raw, self.d_params, grad, hs=self.d_hs, stream=stream, dispersion_only=True)
        self._copy(self.h_hs, self.d_hs, stream)
        if not self.sm_copies:
            self._copy(self.h_grad, self.d_grad, stream)

    def __call__(self, theta: np.ndarray):
        self._set(theta)
        if self.graph is not None:
            self.graph.replay()
        else:
            self._enqueue(self.stream)
        torch.cuda.current_stream(self.raw.device).synchronize()
        self.count += 1
        g = CENTRED_TO_POLY.T @ self.h_grad.numpy()[:4].astype(np.float64)
        return float(self.h_hs[0]), g


class KmapFitEvaluator(FitEvaluator):
    """H and its gradient with respect to (d2, d3, kappa_1 .. kappa_K), where the
    resampling coefficients are ``kmap_of(kappa)`` -> (c0..c3), a k-map family
    given by the caller (for example the inverse of a physical wavenumber map
    with a few free coefficients). Per evaluation: forward and the FULL adjoint
    (dH/dc0..c3 as well as dH/dd0..d3), replayed from one CUDA graph; the chain
    rule through ``kmap_of`` runs on the host with a central-difference
    Jacobian (``dkappa``)."""

    def __init__(self, af: Autofocus, raw: torch.Tensor, kmap_of, k0: Sequence[float], dkappa: float = 1e-4,
                 graph: bool = True):
        self.kmap_of = kmap_of
        self.dkappa = float(dkappa)
        self.nk = len(k0)
        super().__init__(af, raw, kmap_of(np.asarray(k0, np.float64)), graph=graph)

    def _set(self, theta) -> None:
        theta = np.asarray(theta, np.float64)
        hp = self.h_params.numpy()
        hp[:4] = dispersion_poly(theta[0], theta[1])
        if theta.size > 2:
            hp[4:] = np.asarray(self.kmap_of(theta[2:]), np.float32)
        else:
            hp[4:] = self.kmap

    def _enqueue(self, stream) -> None:
        self._copy(self.d_params, self.h_params, stream)
        self.af.forward(self.raw, self.d_params, hs=self.d_hs, stream=stream)
        grad = self.h_grad if self.sm_copies else self.d_grad
        self.af.backward(self.raw, self.d_params, grad, hs=self.d_hs, stream=stream, dispersion_only=False)
        self._copy(self.h_hs, self.d_hs, stream)
        if not self.sm_copies:
            self._copy(self.h_grad, self.d_grad, stream)

    def jacobian(self, kappa: np.ndarray) -> np.ndarray:
        """d(c0..c3)/d(kappa), 4 x K, central differences."""
        J = np.empty((4, self.nk))
        for i in range(self.nk):
            e = np.zeros(self.nk)
            e[i] = self.dkappa
            J[:, i] = (np.asarray(self.kmap_of(kappa + e), np.float64) -
                       np.asarray(self.kmap_of(kappa - e), np.float64)) / (2 * self.dkappa)
        return J

    def __call__(self, theta: np.ndarray):
        theta = np.asarray(theta, np.float64)
        self._set(theta)
        if self.graph is not None:
            self.graph.replay()
        else:
            self._enqueue(self.stream)
        torch.cuda.current_stream(self.raw.device).synchronize()
        self.count += 1
        g8 = self.h_grad.numpy().astype(np.float64)
        gd = CENTRED_TO_POLY.T @ g8[:4]
        gk = self.jacobian(theta[2:]).T @ g8[4:]
        return float(self.h_hs[0]), np.concatenate([gd, gk])


def _allreduce_sum(values: np.ndarray, group=None) -> np.ndarray:
    """Sum over the ranks of `group` in float64 (on the device under NCCL, on the host under gloo)."""
    import torch.distributed as dist
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    t = torch.as_tensor(np.asarray(values, np.float64)).to(dev)
    dist.all_reduce(t, group=group)
    return t.cpu().numpy()


def entropy_parts(h_local: float, s_local: float) -> np.ndarray:
    """(S_r, sum I ln I over this rank's bins) from its own entropy: S_r (ln S_r - H_r).
    A rank without data contributes (0, 0)."""
    return np.array([s_local, s_local * (np.log(s_local) - h_local) if s_local > 0 else 0.0])


def entropy_from_parts(parts: np.ndarray) -> tuple:
    """(H, S) from the summed parts: H = ln S - (sum I ln I) / S."""
    S, IlnI = float(parts[0]), float(parts[1])
    return float(np.log(S) - IlnI / S), S


def combine_entropy(h_local: float, s_local: float, group=None) -> tuple:
    """Global (H, S) of the normalised intensity over every rank's bins from each
    rank's own (H_r, S_r): one all-reduce of the two parts."""
    return entropy_from_parts(_allreduce_sum(entropy_parts(h_local, s_local), group))


class DistributedFitEvaluator:
    """H and dH/d(d2, d3) of the entropy over the A-scans of every rank of a
    process group (one volume split across GPUs, each rank holding its own
    B-scans). Per evaluation: the forward on this rank's A-scans gives (H_r,
    S_r); one all-reduce of 2 values gives the global (H, S); the adjoint on
    this rank's A-scans with the global (H, S) gives this rank's share of the
    gradient; one all-reduce of 8 values sums the shares. Every rank gets the
    same (H, g), so BFGS takes the same steps everywhere and the ranks issue
    the same collectives. ``local_forward(p8) -> (H_r, S_r)`` and
    ``local_backward(p8, H, S) -> g8`` run the chain on this rank's data
    (by default the GPU kernels of ``af`` on ``raw``)."""

    def __init__(self, kmap: Sequence[float], af: Optional[Autofocus] = None, raw: Optional[torch.Tensor] = None,
                 group=None, local_forward=None, local_backward=None):
        self.kmap = np.asarray(kmap, np.float32)
        self.group = group
        self.count = 0
        if local_forward is None:
            dev = raw.device
            d_params = torch.empty(8, dtype=torch.float32, device=dev)
            d_hs = torch.empty(2, dtype=torch.float64, device=dev)
            d_grad = torch.empty(8, dtype=torch.float32, device=dev)

            empty = raw.shape[0] == 0  # a rank without A-scans still joins every collective

            def local_forward(p8):
                if empty:
                    return 0.0, 0.0
                d_params.copy_(torch.from_numpy(p8.astype(np.float32)))
                af.forward(raw, d_params, hs=d_hs)
                h = d_hs.cpu().numpy()
                return float(h[0]), float(h[1])

            def local_backward(p8, H, S):
                if empty:
                    return np.zeros(8)
                d_hs.copy_(torch.tensor([H, S], dtype=torch.float64))
                af.backward(raw, d_params, d_grad, hs=d_hs, dispersion_only=True)
                return d_grad.cpu().numpy().astype(np.float64)
        self.local_forward, self.local_backward = local_forward, local_backward

    def __call__(self, theta: np.ndarray):
        p8 = np.zeros(8, np.float64)
        p8[:4] = dispersion_poly(theta[0], theta[1]).astype(np.float32)
        p8[4:] = self.kmap
        h_r, s_r = self.local_forward(p8)
        H, S = combine_entropy(h_r, s_r, self.group)
        g8 = _allreduce_sum(self.local_backward(p8, H, S), self.group)
        self.count += 1
        return H, CENTRED_TO_POLY.T @ g8[:4]


def fit_dispersion(af: Autofocus, raw: torch.Tensor, kmap: Sequence[float], init=(0.0, 0.0),
                   max_iter: int = 60, step_tol: float = 1e-3, first_step: float = 2.0,
                   graph: bool = True, evaluator=None) -> FitResult:
    """Minimises the image entropy over the centred dispersion (d2, d3).

    BFGS with an Armijo backtracking line search on the host (2 x 2 inverse
    Hessian); each evaluation is one forward (entropy) and one adjoint pass on
    the device, replayed from a CUDA graph when ``graph`` is set (the capture
    happens before the clock starts). ``kmap`` holds the resampling
    coefficients c0..c3. Stops when a step moves less than ``step_tol`` (rad).
    ``evaluator``: a FitEvaluator built earlier for this handle, this tensor
    and this k-map, reused instead of building (and capturing) a new one; or a
    DistributedFitEvaluator, which fits one dispersion to the A-scans of every
    rank of its process group.
    """
    if evaluator is None:
        ev = FitEvaluator(af, raw, kmap, graph=graph)
    else:
        ev = evaluator
        if not np.array_equal(ev.kmap, np.asarray(kmap, np.float32)):
            raise ValueError("evaluator was built for another k-map")
        if isinstance(ev, FitEvaluator) and (ev.af is not af or ev.raw.data_ptr() != raw.data_ptr()
                                             or ev.raw.shape != raw.shape):
            raise ValueError("evaluator was built for another handle or tensor")
    count0 = ev.count
    t0 = time.perf_counter()
    x = np.asarray(init, np.float64)
    f, g = ev(x)
    gmax = float(np.abs(g).max())
    hinv = np.eye(2) * (first_step / gmax if gmax > 0 else 1.0)
    hist = [(float(x[0]), float(x[1]), f, time.perf_counter() - t0)]
    it = 0
    for it in range(1, max_iter + 1):
        d = -hinv @ g
        if g @ d >= 0:  # not a descent direction: restart from steepest descent
            hinv = np.eye(2) * (first_step / max(float(np.abs(g).max()), 1e-30))
            d = -hinv @ g
        step = 1.0
        while True:
            xn = x + step * d
            fn, gn = ev(xn)
            if fn <= f + 1e-4 * step * float(g @ d) or step < 1e-6:
                break
            step *= 0.5
        s, yv = xn - x, gn - g
        sy = float(s @ yv)
        if sy > 1e-30:
            rho = 1.0 / sy
            eye = np.eye(2)
            hinv = (eye - rho * np.outer(s, yv)) @ hinv @ (eye - rho * np.outer(yv, s)) + rho * np.outer(s, s)
        x, f, g = xn, fn, gn
        hist.append((float(x[0]), float(x[1]), f, time.perf_counter() - t0))
        if float(np.linalg.norm(s)) < step_tol:
            break
    secs = time.perf_counter() - t0
    return FitResult(float(x[0]), float(x[1]), f, it, ev.count - count0, secs, hist)


@dataclass
class JointFitResult:
    d2: float
    d3: float
    kappa: np.ndarray  # the fitted k-map family parameters
    kmap: np.ndarray  # the resampling coefficients c0..c3 they give
    entropy: float
    iterations: int
    evaluations: int
    seconds: float
    history: list = field(default_factory=list)  # (theta, H, seconds since start) per iteration


def _bfgs(ev, x0: np.ndarray, scale: np.ndarray, max_iter: int, step_tol: float, first_step: float):
    """BFGS with Armijo backtracking in the scaled coordinates y = x / scale."""
    t0 = time.perf_counter()
    n = x0.size

    def fy(y):
        f, g = ev(y * scale)
        return f, g * scale

    y = x0 / scale
    f, g = fy(y)
    gmax = float(np.abs(g).max())
    hinv = np.eye(n) * (first_step / gmax if gmax > 0 else 1.0)
    hist = [(y * scale, f, time.perf_counter() - t0)]
    it = 0
    for it in range(1, max_iter + 1):
        d = -hinv @ g
        if g @ d >= 0:
            hinv = np.eye(n) * (first_step / max(float(np.abs(g).max()), 1e-30))
            d = -hinv @ g
        step = 1.0
        while True:
            yn = y + step * d
            fn, gn = fy(yn)
            if fn <= f + 1e-4 * step * float(g @ d) or step < 1e-6:
                break
            step *= 0.5
        s, yv = yn - y, gn - g
        sy = float(s @ yv)
        if sy > 1e-30:
            rho = 1.0 / sy
            eye = np.eye(n)
            hinv = (eye - rho * np.outer(s, yv)) @ hinv @ (eye - rho * np.outer(yv, s)) + rho * np.outer(s, s)
        y, f, g = yn, fn, gn
        hist.append((y * scale, f, time.perf_counter() - t0))
        if float(np.linalg.norm(s)) < step_tol:  # a step below step_tol in the scaled coordinates
            break
    return y * scale, f, it, time.perf_counter() - t0, hist


def fit_dispersion_kmap(af: Autofocus, raw: torch.Tensor, kmap_of, k0: Sequence[float], init=(0.0, 0.0),
                        kappa_scale: Optional[Sequence[float]] = None, max_iter: int = 120, step_tol: float = 1e-3,
                        first_step: float = 2.0, graph: bool = True, evaluator=None) -> JointFitResult:
    """Minimises the image entropy jointly over the centred dispersion (d2, d3)
    and the parameters kappa of a k-map family: the resampling coefficients
    are ``kmap_of(kappa)``, starting from ``k0`` (the nominal k-map).

    A fit over the four raw resampling coefficients is ill-posed: on scenes of
    a few reflectors the entropy cannot tell a cubic k-map error from cubic
    dispersion. A k-map family with the physics' own few free parameters (for
    instance the cubic coefficient of the wavenumber map) is not: a k-map
    error shifts the phase of each reflector in proportion to its depth,
    dispersion does not, so the joint optimum separates them.
    ``kappa_scale``: typical size of one unit of each kappa relative to a
    radian of (d2, d3) for the optimiser's coordinates (default 0.01).
    """
    k0 = np.asarray(k0, np.float64)
    ev = evaluator if evaluator is not None else KmapFitEvaluator(af, raw, kmap_of, k0, graph=graph)
    count0 = ev.count
    x0 = np.concatenate([np.asarray(init, np.float64), k0])
    ks = np.full(k0.size, 0.01) if kappa_scale is None else np.asarray(kappa_scale, np.float64)
    scale = np.concatenate([[1.0, 1.0], ks])
    x, f, it, secs, hist = _bfgs(ev, x0, scale, max_iter, step_tol, first_step)
    return JointFitResult(float(x[0]), float(x[1]), x[2:].copy(), np.asarray(kmap_of(x[2:]), np.float64), f, it,
                          ev.count - count0, secs, hist)


@dataclass
class SweepResult:
    d2: float
    d3: float
    entropy: float
    seconds: float
    grid: np.ndarray  # (n2, n3) entropies
    capture_seconds: float = 0.0


def fit_dispersion_distributed(af: Autofocus, raw: torch.Tensor, kmap: Sequence[float], group=None,
                               **kw) -> FitResult:
    """fit_dispersion over the A-scans of every rank of `group` (torch.distributed
    process group, NCCL between GPUs): `raw` holds this rank's A-scans; every rank
    returns the same result."""
    ev = DistributedFitEvaluator(kmap, af=af, raw=raw, group=group)
    return fit_dispersion(af, raw, kmap, evaluator=ev, **kw)


def grid_sweep(af: Autofocus, raw: torch.Tensor, kmap: Sequence[float], d2_range=(-40.0, 40.0),
               d3_range=(-20.0, 20.0), n2: int = 64, n3: int = 64, graph: bool = True) -> SweepResult:
    """Entropy of the forward chain at every point of an n2 x n3 (d2, d3) grid.

    All parameter vectors are uploaded once; the n2*n3 forward passes run back
    to back on one stream -- replayed from one CUDA graph when ``graph`` is set
    (captured before the clock starts, its capture time reported apart) --
    with one synchronisation at the end.
    """
    dev = raw.device
    g2 = np.linspace(d2_range[0], d2_range[1], n2)
    g3 = np.linspace(d3_range[0], d3_range[1], n3)
    P = np.empty((n2 * n3, 8), np.float32)
    k = 0
    for a in g2:
        for b in g3:
            P[k, :4] = dispersion_poly(a, b)
            P[k, 4:] = kmap
            k += 1
    d_params = torch.from_numpy(P).to(dev)
    hs = torch.empty((n2 * n3, 2), dtype=torch.float64, device=dev)

    def enqueue(stream):
        for k in range(n2 * n3):
            af.forward(raw, d_params[k], hs=hs[k], stream=stream)

    g = None
    cap = 0.0
    if graph:
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            af.forward(raw, d_params[0], hs=hs[0], stream=side)  # warm-up outside the capture
        side.synchronize()
        t_c = time.perf_counter()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=side):
            enqueue(side)
        torch.cuda.synchronize(dev)
        cap = time.perf_counter() - t_c
    stream = torch.cuda.current_stream(dev)
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    if g is not None:
        g.replay()
    else:
        enqueue(stream)
    best = int(torch.argmin(hs[:, 0]).item())  # synchronises
    secs = time.perf_counter() - t0
    H = hs[:, 0].cpu().numpy().reshape(n2, n3)
    return SweepResult(float(g2[best // n3]), float(g3[best % n3]), float(H.flat[best]), secs, H, cap)
