"""Generates the golden fixtures in tests/golden/ from the REFERENCE itself.

Runs the reference CPU backend (ope::CpuBackend from the reference sources,
compiled out of tree by oracle/Makefile into oracle/_ref/libope_cpu_ref.so;
FFT = project shim, not FFTW) on small seeded inputs and stores inputs,
curves and outputs as .npz: ``out`` with the shim's DFT evaluated in float64,
``out_f32fft`` with it evaluated in float32. The oracle restatement and the GPU
kernels are then checked against these files on machines without the
reference tree.

    python tests/golden/make_golden.py [name ...]   # all cases, or the named ones
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import reflib  # noqa: E402
from octproengine_b200 import synth  # noqa: E402  (the benchmark's seeded generator; numpy + torch)

_LIN2048 = synth.linearising_coeffs(2048)
_DISP = synth.compensating_coeffs(12.0, -6.0)

# (name, params for reflib.make_params, dtype, seed)
# The first case is the reference's own comparison-test configuration
# (tests/test_backend_output_comparison.cpp:18-45) at fewer A-scans.
CASES = [
    ("refcmp_cubic_hann_dc", dict(n=2048, ascans=16, dtype=2, resampling=True, interpolation=1,
                                  resampling_coeffs=(0.5, 2048.0, -100.0, 50.0), windowing=True, window_type=0,
                                  window_center=0.9, window_fill=0.85, dispersion=True,
                                  dispersion_coeffs=(0.0, 0.0, 1.0, -3.0), dc_removal=True,
                                  grayscale_min=0.0, grayscale_max=80.0), 11),
    ("lin_hann_disp_n1024", dict(n=1024, ascans=12, dtype=2, resampling=True, interpolation=0,
                                 resampling_coeffs=(0.3, 1010.0, 30.0, -12.0), windowing=True, window_type=0,
                                 window_center=0.5, window_fill=0.95, dispersion=True,
                                 dispersion_coeffs=(0.2, -1.0, 4.0, -2.0), grayscale_min=30.0,
                                 grayscale_max=100.0), 12),
    ("lanczos_gauss_n512", dict(n=512, ascans=9, dtype=2, resampling=True, interpolation=2,
                                resampling_coeffs=(1.0, 500.0, 10.0, -5.0), windowing=True, window_type=1,
                                window_center=0.45, window_fill=0.8, dispersion=True,
                                dispersion_coeffs=(0.0, 0.5, -3.0, 1.5), grayscale_min=0.0,
                                grayscale_max=90.0), 13),
    ("u8_sine_lin_scale", dict(n=512, ascans=8, dtype=1, resampling=True, interpolation=0,
                               resampling_coeffs=(0.0, 511.0, 0.0, 0.0), windowing=True, window_type=2,
                               window_center=0.5, window_fill=0.9, log_scaling=False,
                               grayscale_min=0.0, grayscale_max=2.0), 14),
    ("flattop_auto_minmax_n2048", dict(n=2048, ascans=6, dtype=2, windowing=True, window_type=5,
                                       window_center=0.5, window_fill=0.9, grayscale_min=50.0,
                                       grayscale_max=50.0, multiplicator=2.0, addend=0.1), 15),
    ("fpn_cubic_n1024", dict(n=1024, ascans=32, dtype=2, resampling=True, interpolation=1,
                             resampling_coeffs=(0.5, 1020.0, -20.0, 10.0), windowing=True, window_type=0,
                             window_center=0.5, window_fill=0.95, fpn_removal=True, fpn_bscan_count=1,
                             grayscale_min=20.0, grayscale_max=110.0), 16),
    # the benchmark workload's shape: 2048 samples, cubic, Gaussian window,
    # dispersion compensation, FPN determined from the frame, spectra from the
    # benchmark generator with a fixed-pattern background ripple
    ("headline_cubic_gauss_fpn_n2048", dict(n=2048, ascans=64, dtype=2, resampling=True, interpolation=1,
                                            resampling_coeffs=_LIN2048, windowing=True, window_type=1,
                                            window_center=0.5, window_fill=0.9, dispersion=True,
                                            dispersion_coeffs=_DISP, fpn_removal=True, fpn_bscan_count=1,
                                            grayscale_min=30.0, grayscale_max=110.0, gen="bench"), 17),
    # rolling-average DC removal where the reference's float prefix sums round (N = 4096)
    ("dc_lanczos_n4096", dict(n=4096, ascans=8, dtype=2, resampling=True, interpolation=2,
                              resampling_coeffs=(0.5, 4090.0, -40.0, 20.0), windowing=True, window_type=0,
                              window_center=0.5, window_fill=0.95, dispersion=True,
                              dispersion_coeffs=(0.0, 0.0, 2.0, -1.0), dc_removal=True, dc_window=64,
                              grayscale_min=20.0, grayscale_max=110.0), 18),
]


def raw_for(n, m, dtype, seed):
    rng = np.random.default_rng(seed)
    if dtype == 1:
        return np.clip(128 + rng.normal(0, 20, (m, n)), 0, 255).astype(np.uint8)
    x = np.arange(n)
    base = 2000 + 1000 * np.sin(0.3 * x)[None, :]
    peaks = sum(a * np.exp(-((x - c * n) / w) ** 2)[None, :] for a, c, w in ((8000, 0.2, 50), (5000, 0.5, 30)))
    v = base + peaks + rng.normal(0, 120, (m, n)) + rng.normal(0, 2000, (m, 1))
    return np.clip(v + 20000, 0, 65535).astype(np.uint16)


def main(names=()):
    if not reflib.available():
        reflib.build()
    reflib.set_fft_precision("f64")
    for name, kw, seed in CASES:
        if names and name not in names:
            continue
        kw = dict(kw)
        n, m = kw.pop("n"), kw.pop("ascans")
        dtype = kw.pop("dtype")
        gen = kw.pop("gen", None)
        p = reflib.make_params(n, m, 1, dtype, **kw)
        if gen == "bench":
            raw = synth.as_numpy(synth.generate(synth.SynthParams(n=n, ascans=m, seed=seed, d2=12.0, d3=-6.0,
                                                                  background_ripple=True)), "uint16")
        else:
            raw = raw_for(n, m, dtype, seed)
        r, w, ph, cs = reflib.generate_curves(p)
        be = reflib.RefBackend(p)
        if kw.get("fpn_removal"):
            be.request_fpn()
        out = be.process(raw)
        fpn = be.fpn_profile()
        be.close()
        # the same run with the shim evaluating the DFT in float32 (radix-2),
        # i.e. the accuracy class of a float32 library FFT such as FFTW's
        reflib.set_fft_precision("f32")
        be = reflib.RefBackend(p)
        if kw.get("fpn_removal"):
            be.request_fpn()
        out_f32fft = be.process(raw)
        be.close()
        reflib.set_fft_precision("f64")
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), raw=raw, out=out, out_f32fft=out_f32fft, resample=r, window=w, phase=ph,
                            cos_sin=cs, fpn=fpn, n=n, m=m, dtype=dtype,
                            params=np.frombuffer(bytes(p), dtype=np.uint8))
        print(name, raw.shape, out.shape, float(out.min()), float(out.max()), "fpn pairs", fpn.size // 2)


if __name__ == "__main__":
    main(tuple(sys.argv[1:]))
