"""Three-way parity per stratum: GPU vs float64, reference CPU backend vs float64,
GPU vs reference CPU backend, on the benchmark workloads (seeded synthetic
spectra).

GPU = this backend through the C ABI; CPU = the reference CpuBackend compiled
out of tree (oracle/_ref) with its FFT served by the project's float32 radix-2
shim (FFTW is absent on both machines); float64 = the oracle restatement with
every chain operation in float64. Errors are in dB (the log output mapped back
through the grayscale affine), as max-abs over all bins, over the display range
(float64 >= grayscale min), over displayed bins where the FPN subtraction
cancels at most 20 dB, over bins >= 40 dB, and as the 99.9th percentile of all
bins; plus the cancellation-normalised error: each bin's dB error divided by
its cancellation factor kappa = |X| / |X - F| (X the float64 DFT bin, F the FPN
profile; kappa = 1 without FPN removal), i.e. the error the bin carries before
the subtraction amplifies it.

With FPN removal on, the FPN profile matches the fixed pattern (the background
ripple) to 60-80 dB on a few bins per A-scan. Any float32 path's rounding there
is multiplied by kappa (up to ~1e4), so the raw all-bins, display and p99.9
maxima of both float32 paths are set by a handful of such bins (0.5-1 dB on
displayed bins, 25-30 dB on bins that end near zero) and say nothing about
which path is more accurate; they are printed, not ordered. The claims:
* every case: the GPU is no less accurate than the reference's own float32 path
  on bins >= 40 dB, on displayed bins with kappa <= 10, and in the
  cancellation-normalised error; and within 1e-3 dB of float64 on bins >= 40 dB
  and on displayed bins with kappa <= 10;
* without FPN removal (kappa = 1): no less accurate on every stratum.
"""
import numpy as np
import pytest

import helpers as H
from octproengine_b200 import synth
from octproengine_b200.chain import ChainSpec, LINEAR, CUBIC, LANCZOS, HANN, GAUSS

pytestmark = pytest.mark.gpu


def _cases():
    n = 2048
    lin = synth.linearising_coeffs(n)
    disp = synth.compensating_coeffs(12.0, -6.0)
    c1 = ChainSpec(signal_length=n, ascans_per_bscan=512, bscans_per_buffer=1, resampling=True, interpolation=LINEAR,
                   resampling_coeffs=lin, windowing=True, window_type=HANN, window_center=0.5, window_fill=0.95,
                   dispersion=True, dispersion_coeffs=disp, grayscale_min=35.0, grayscale_max=115.0)
    out = [("config1 linear hann", c1, synth.SynthParams(n=n, ascans=512, seed=1, d2=12.0, d3=-6.0))]
    for interp, name in ((CUBIC, "cubic"), (LANCZOS, "lanczos8")):
        c2 = ChainSpec(signal_length=n, ascans_per_bscan=1024, bscans_per_buffer=2, resampling=True,
                       interpolation=interp, resampling_coeffs=lin, windowing=True, window_type=GAUSS,
                       window_center=0.5, window_fill=0.9, dispersion=True, dispersion_coeffs=disp,
                       fpn_removal=True, fpn_bscan_count=1, grayscale_min=35.0, grayscale_max=115.0)
        out.append((f"config2 {name} gauss fpn", c2,
                    synth.SynthParams(n=n, ascans=1024, bscans=2, seed=2, d2=12.0, d3=-6.0, background_ripple=True)))
    return out


STRATA = ("all", "display", "display k<=10", ">=40dB", "p99.9", "normalised")
ORDERED = ("display k<=10", ">=40dB", "normalised")  # GPU <= CPU in every case


def _strata(err, ref_db, kappa, gmin):
    disp = ref_db >= gmin
    return {"all": float(err.max()), "display": float(err[disp].max()),
            "display k<=10": float(err[disp & (kappa <= 10.0)].max()),
            ">=40dB": float(err[ref_db >= 40.0].max()), "p99.9": float(np.percentile(err, 99.9)),
            "normalised": float((err / kappa).max())}


def _cancellation(spec, X64, ref_db):
    """kappa = |X| / |Y|, |Y| recovered from the float64 output in dB."""
    half = spec.signal_length // 2
    if not spec.fpn_removal:
        return np.ones_like(ref_db)
    amp = np.sqrt(half * 10.0 ** (ref_db / 10.0))
    with np.errstate(divide="ignore"):
        return np.maximum(np.abs(X64[:, :half]) / amp, 1.0)


@pytest.mark.parametrize("name,spec,sp", _cases(), ids=lambda v: v if isinstance(v, str) else "")
def test_three_way_parity_per_stratum(cuda, reflib, name, spec, sp):
    raw = synth.as_numpy(synth.generate(sp), "uint16")
    gpu = H.gpu_run(spec, raw, fpn_request=spec.fpn_removal)
    res64 = H.oracle_image(spec, raw, mode="f64", determine_fpn=spec.fpn_removal, keep=True)
    reflib.set_fft_precision("f32")
    p = reflib.make_params(spec.signal_length, spec.ascans_per_bscan, spec.bscans_per_buffer, 2, resampling=True,
                           interpolation=spec.interpolation, resampling_coeffs=spec.resampling_coeffs,
                           windowing=True, window_type=spec.window_type, window_center=spec.window_center,
                           window_fill=spec.window_fill, dispersion=True, dispersion_coeffs=spec.dispersion_coeffs,
                           fpn_removal=spec.fpn_removal, fpn_bscan_count=spec.fpn_bscan_count,
                           grayscale_min=spec.grayscale_min, grayscale_max=spec.grayscale_max)
    be = reflib.RefBackend(p)
    if spec.fpn_removal:
        be.request_fpn()
    cpu = be.process(raw)
    be.close()
    g, c, t = (H.to_db(x, spec) for x in (gpu, cpu, res64.output))
    kappa = _cancellation(spec, res64.ifft, t)
    gmin = spec.grayscale_min
    rows = {"GPU vs FP64": _strata(np.abs(g - t), t, kappa, gmin),
            "CPU vs FP64": _strata(np.abs(c - t), t, kappa, gmin),
            "GPU vs CPU": _strata(np.abs(g - c), t, kappa, gmin)}
    disp = t >= gmin
    print(f"\n{name} ({spec.num_ascans} A-scans of {spec.signal_length}; displayed bins with kappa <= 10: "
          f"{(disp & (kappa <= 10)).sum() / disp.sum():.2%}), dB max-abs per stratum:")
    for k, v in rows.items():
        print(f"  {k:12s} " + "  ".join(f"{s} {x:.2e}" for s, x in v.items()))
    gpu_e, cpu_e = rows["GPU vs FP64"], rows["CPU vs FP64"]
    for s in (STRATA if not spec.fpn_removal else ORDERED):
        assert gpu_e[s] <= 1.05 * cpu_e[s] + 1e-6, (s, rows)
    assert gpu_e[">=40dB"] < 1e-3 and gpu_e["display k<=10"] < 1e-3, rows
