"""The chain against the reference CPU backend's own output, at the 1e-3 dB bar.

Every golden fixture holds ``out``: the reference CpuBackend (compiled from the
reference sources, tests/golden/make_golden.py) run on the fixture's input with
its DFT evaluated exactly by the FFT shim and rounded once. Every stage before
the DFT is the reference's own float32 arithmetic; this chain reproduces those
stages bit for bit (rolling-average DC removal in the reference's order), so
the remaining difference is this chain's float32 DFT.

Claims, per fixture, in output dB (the log output mapped back through the
grayscale affine; for auto min/max the per-A-scan range; for linear output the
amplitude in dB), with X the float64 DFT bin, F the FPN profile and
kappa = |X| / |X - F| the fixed-pattern cancellation factor (1 without FPN
removal):
  * max |chain - reference| <= 1e-3 dB on bins >= 40 dB (every fixture);
  * <= 1e-3 dB on displayed bins (reference >= grayscale min) with kappa <= 10
    that lie within 70 dB of their A-scan's strongest float64 bin (every
    fixture but the auto min/max one, below);
  * on all displayed bins with kappa <= 10 the chain is no further from the
    reference's exact-DFT output than the reference's own float32-DFT path is.
Where the 1e-3 dB bar does not hold, and why:
  * displayed bins more than 70 dB below their A-scan's strongest bin (the
    grayscale floor sits 85-130 dB below the DC bin in these fixtures): any
    float32 DFT's rounding, relative to the strongest bin, is above 1e-3 dB
    there; measured up to 2.4e-3 dB for this chain and up to 1.9e-2 dB for the
    reference's own float32 path;
  * auto min/max (grayscale min == max): every bin of an A-scan is mapped
    through that A-scan's minimum, its weakest bin, which carries the float32
    error floor; measured 1.03e-3 dB (the reference's float32 path: 5.5e-3);
  * bins where the FPN subtraction cancels 60-80 dB (kappa up to ~1e4), which
    multiplies any float32 rounding by kappa, and the weakest bins below the
    display floor: printed, not claimed.
"""
import numpy as np
import pytest

import helpers as H

DB_BAR = 1e-3


def _cases():
    return [(name, spec.with_(dc_reference_order=spec.dc_removal), d) for name, spec, d in H.golden_cases()]


def _db_pair(img, ref, spec, X64):
    """Both outputs in dB, per the fixture's output mode."""
    half = spec.signal_length // 2
    if not spec.log_scaling:
        rng = np.float32(spec.grayscale_max) - np.float32(spec.grayscale_min)
        rng = 1.0 if rng < 1e-6 else float(rng)

        def amp_db(o):
            amp = (o.astype(np.float64) / spec.multiplicator - spec.addend) * rng + spec.grayscale_min
            return 20.0 * np.log10(np.maximum(np.abs(amp), 1e-30))
        return amp_db(img), amp_db(ref)
    if spec.grayscale_min == spec.grayscale_max:
        # auto min/max per A-scan (cpu_kernels.tpp:327-335): out = mult * ((v - mn)/range + addend)
        v = 10.0 * np.log10(np.maximum(np.abs(X64[:, :half]) ** 2 / half, 1e-300))
        rng = np.maximum(v.max(axis=1, keepdims=True) - v.min(axis=1, keepdims=True), 1e-6)

        def db(o):
            return (o.astype(np.float64) / spec.multiplicator - spec.addend) * rng
        return db(img), db(ref)
    return H.to_db(img, spec), H.to_db(ref, spec)


def _strata(spec, d, img, res64, fpn):
    g, r = _db_pair(img, d["out"], spec, res64.ifft)
    err = np.abs(g - r)
    kappa = H.fpn_kappa(spec, res64.ifft, fpn)
    half = spec.signal_length // 2
    p2 = np.abs(res64.ifft[:, :half]) ** 2
    rel = 10.0 * np.log10(np.maximum(p2, 1e-300) / p2.max(axis=1, keepdims=True))
    if spec.log_scaling and spec.grayscale_min != spec.grayscale_max:
        shown = r >= spec.grayscale_min
        strong = r >= 40.0
    else:  # auto range and linear output: relative to each A-scan's strongest bin
        peak = r.max(axis=1, keepdims=True)
        shown = r >= peak - 60.0
        strong = r >= peak - 40.0
    sel = shown & (kappa <= 10.0)
    return {"all": err.max(), ">=40dB": err[strong].max(), "displayed k<=10": err[sel].max(),
            "displayed k<=10 within 70 dB": err[sel & (rel >= -70.0)].max()}


def _check(name, spec, d, img):
    fpn = d["fpn"] if spec.fpn_removal else None
    res64 = H.oracle_image(spec, d["raw"], mode="f64", fpn_profile=fpn, keep=True)
    mine = _strata(spec, d, img, res64, fpn)
    ref32 = _strata(spec, d, d["out_f32fft"], res64, fpn)
    print(f"\n{name}, dB max-abs against the reference CpuBackend (exact DFT):")
    for label, e in (("this chain", mine), ("reference, float32 DFT", ref32)):
        print(f"  {label:24s} " + "  ".join(f"{k} {v:.2e}" for k, v in e.items()))
    assert mine[">=40dB"] <= DB_BAR, (name, mine)
    if not (spec.log_scaling and spec.grayscale_min == spec.grayscale_max):
        assert mine["displayed k<=10 within 70 dB"] <= DB_BAR, (name, mine)
    assert mine["displayed k<=10"] <= ref32["displayed k<=10"], (name, mine, ref32)


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_emulated_chain_vs_reference_cpu_backend(emu, case):
    name, spec, d = case
    fpn = d["fpn"] if spec.fpn_removal else None
    img = H.emu_run(emu, spec, d["raw"], "image", fpn=fpn)
    _check(name, spec, d, img)


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_gpu_chain_vs_reference_cpu_backend(cuda, case):
    name, spec, d = case
    fpn = d["fpn"] if spec.fpn_removal else None
    img = H.gpu_run(spec, d["raw"], fpn_profile=fpn)
    _check(name, spec, d, img)
