"""Host-side description of one chain configuration and its context set-up.

:class:`ChainSpec` carries the fields of ``ope::ProcessorConfiguration``
(include/processorconfiguration.h:31-180) the chain reads, with the reference
defaults. :func:`open_context` creates a C-ABI context and hands it the
generated curves the way ``Processor::Impl::initialize`` /
``updateAllBackendCurves`` do (src/core/processor.cpp:135-156,102-125): the
resampling curve, the window curve and the dispersion phase converted to
interleaved (cos, sin).
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace
from typing import Optional, Sequence

import numpy as np

from . import capi

# ope::DataType (include/types.h:6-19)
UINT8, UINT16, UINT32, FLOAT32 = 1, 2, 3, 9
DTYPE_BYTES = {UINT8: 1, UINT16: 2, UINT32: 4, FLOAT32: 4}
NUMPY_DTYPE = {UINT8: np.uint8, UINT16: np.uint16, UINT32: np.uint32, FLOAT32: np.float32}
# ope::InterpolationMethod / ope::WindowType
LINEAR, CUBIC, LANCZOS = 0, 1, 2
HANN, GAUSS, SINE, LANCZOS_WINDOW, RECTANGULAR, FLAT_TOP = 0, 1, 2, 3, 4, 5


@dataclass
class ChainSpec:
    signal_length: int = 1024
    ascans_per_bscan: int = 512
    bscans_per_buffer: int = 1
    input_dtype: int = UINT16
    resampling: bool = False
    interpolation: int = LINEAR
    resampling_coeffs: Sequence[float] = (0.0, 1.0, 0.0, 0.0)
    windowing: bool = False
    window_type: int = HANN
    window_center: float = 0.5
    window_fill: float = 0.95
    dispersion: bool = False
    dispersion_coeffs: Sequence[float] = (0.0, 0.0, 0.0, 0.0)
    dc_removal: bool = False
    dc_window: int = 64
    log_scaling: bool = True
    grayscale_min: float = 30.0
    grayscale_max: float = 100.0
    addend: float = 0.0
    multiplicator: float = 1.0
    fpn_removal: bool = False
    fpn_bscan_count: int = 1
    fpn_continuous: bool = False
    bscan_flip: bool = False
    float32_as_uint32: bool = False
    bitshift: bool = False  # 8/16-bit samples >> 4 before the chain
    dc_split: bool = True
    # rolling-average DC removal in the reference CPU backend's order (its
    # sequential float prefix sum) instead of exact integer window sums
    dc_reference_order: bool = False
    device: int = 0
    num_input_buffers: int = 2  # depth of the host frame ring
    # custom curves (used instead of the generated ones when given)
    resampling_curve: Optional[np.ndarray] = field(default=None, repr=False)
    window_curve: Optional[np.ndarray] = field(default=None, repr=False)
    dispersion_phase: Optional[np.ndarray] = field(default=None, repr=False)

    @property
    def num_ascans(self) -> int:
        return self.ascans_per_bscan * self.bscans_per_buffer

    @property
    def bytes_per_sample(self) -> int:
        return DTYPE_BYTES[self.input_dtype]

    def with_(self, **kw) -> "ChainSpec":
        return replace(self, **kw)

    def to_config(self) -> capi.Config:
        c = capi.default_config()
        c.signal_length = self.signal_length
        c.ascans_per_bscan = self.ascans_per_bscan
        c.bscans_per_buffer = self.bscans_per_buffer
        c.input_dtype = self.input_dtype
        c.resampling_enabled = int(self.resampling)
        c.interpolation = int(self.interpolation)
        c.windowing_enabled = int(self.windowing)
        c.dispersion_enabled = int(self.dispersion)
        c.dc_removal_enabled = int(self.dc_removal)
        c.dc_window = int(self.dc_window)
        c.log_scaling = int(self.log_scaling)
        c.grayscale_min = self.grayscale_min
        c.grayscale_max = self.grayscale_max
        c.addend = self.addend
        c.multiplicator = self.multiplicator
        c.fpn_removal = int(self.fpn_removal)
        c.fpn_bscan_count = int(self.fpn_bscan_count)
        c.fpn_continuous = int(self.fpn_continuous)
        c.bscan_flip = int(self.bscan_flip)
        c.float32_as_uint32 = int(self.float32_as_uint32)
        c.bitshift = int(self.bitshift)
        c.dc_split = int(self.dc_split)
        c.dc_reference_order = int(self.dc_reference_order)
        c.device = int(self.device)
        c.num_input_buffers = int(self.num_input_buffers)
        return c

    # curves as the reference Processor hands them to its backend
    def curves(self):
        n = self.signal_length
        r = self.resampling_curve if self.resampling_curve is not None else \
            capi.generate_resampling_curve(n, self.resampling_coeffs)
        w = self.window_curve if self.window_curve is not None else \
            capi.generate_window_curve(n, self.window_type, self.window_center, self.window_fill)
        ph = self.dispersion_phase if self.dispersion_phase is not None else \
            capi.generate_dispersion_phase(n, self.dispersion_coeffs)
        return (np.ascontiguousarray(r, np.float32), np.ascontiguousarray(w, np.float32),
                capi.phase_to_cos_sin(np.ascontiguousarray(ph, np.float32)))


def open_context(spec: ChainSpec) -> capi.Context:
    ctx = capi.Context(spec.to_config())
    r, w, cs = spec.curves()
    ctx.set_resampling_curve(r)
    ctx.set_window_curve(w)
    ctx.set_dispersion_curve(cs)
    return ctx
