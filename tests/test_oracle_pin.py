"""Pins the numpy restatement (oracle/restate.py) to the reference itself:
the committed golden fixtures (made by the reference CPU backend) and, where
the reference tree is present, the reference library live."""
import numpy as np
import pytest

import helpers as H
from oracle import restate as R


@pytest.mark.parametrize("case", H.golden_cases(), ids=lambda c: c[0])
def test_restatement_matches_golden(case):
    name, spec, d = case
    st, cur = H.oracle_settings(spec)
    # curves: bit-exact
    assert np.array_equal(cur.resample, d["resample"])
    assert np.array_equal(cur.window, d["window"])
    assert np.array_equal(R.dispersion_phase(spec.signal_length, spec.dispersion_coeffs), d["phase"])
    assert np.array_equal(cur.cos, d["cos_sin"][0::2]) and np.array_equal(cur.sin, d["cos_sin"][1::2])
    res = R.process_buffer(d["raw"], st, cur, determine_fpn=spec.fpn_removal)
    # every stage before the DFT is float32-exact; the DFT is float64 in both
    # (shim "f64" mode vs numpy), then rounded: a few ulp on the output
    scale = max(1.0, float(np.abs(d["out"]).max()))
    assert np.abs(res.output - d["out"]).max() <= 4e-7 * scale
    if spec.fpn_removal:
        assert d["fpn"].size == spec.signal_length
        np.testing.assert_allclose(res.fpn_profile, d["fpn"], rtol=2e-6, atol=1e-3)


def test_golden_includes_reference_comparison_config():
    names = [c[0] for c in H.golden_cases()]
    assert "refcmp_cubic_hann_dc" in names


@pytest.mark.parametrize("method", [0, 1, 2])
@pytest.mark.parametrize("n", [256, 1024, 2048])
def test_klinearization_bit_exact_live(reflib, method, n):
    rng = np.random.default_rng(n + method)
    x = (32768 + rng.normal(0, 4000, n)).astype(np.float32)
    # generated (clamped) and custom, unclamped curves incl. edges
    curves = [R.resampling_curve(n, (0.5, n, -100, 50)),
              np.clip(np.linspace(-0.4, n - 0.6, n) + rng.normal(0, 0.3, n), 0, n - 1).astype(np.float32)]
    for curve in curves:
        ref = reflib.klinearization(x, curve, method)
        mine = {0: R.klin_linear, 1: R.klin_cubic, 2: R.klin_lanczos}[method](x[None], curve)[0]
        assert np.array_equal(ref, mine)


@pytest.mark.parametrize("wtype", range(6))
@pytest.mark.parametrize("n,center,fill", [(512, 0.5, 0.95), (2048, 0.9, 0.85), (1000, 0.1, 0.5), (4096, 1.3, 1.2)])
def test_curves_bit_exact_live(reflib, wtype, n, center, fill):
    p = reflib.make_params(n, 4, 1, 2, window_type=wtype, window_center=center, window_fill=fill,
                           resampling_coeffs=(1.5, n * 0.97, -33.0, 12.0), dispersion_coeffs=(0.1, -2.0, 7.0, -3.0))
    r, w, ph, cs = reflib.generate_curves(p)
    assert np.array_equal(r, R.resampling_curve(n, (1.5, n * 0.97, -33.0, 12.0)))
    assert np.array_equal(w, R.window_curve(n, wtype, center, fill))
    assert np.array_equal(ph, R.dispersion_phase(n, (0.1, -2.0, 7.0, -3.0)))
    c, s = R.phase_to_cos_sin(ph)
    assert np.array_equal(cs[0::2], c) and np.array_equal(cs[1::2], s)


def test_min_var_mean_bit_exact_live(reflib):
    rng = np.random.default_rng(7)
    X = (rng.normal(0, 1000, (64, 128)) + 1j * rng.normal(0, 1000, (64, 128))).astype(np.complex64)
    ref = reflib.min_var_mean(X, 8)
    mine = R.min_var_mean(X, 8)
    assert np.array_equal(ref, mine)


@pytest.mark.parametrize("dc", [False, True])
@pytest.mark.parametrize("interp", [0, 1, 2])
def test_full_chain_live(reflib, interp, dc):
    n, m = 1024, 10
    reflib.set_fft_precision("f64")
    p = reflib.make_params(n, m, 1, 2, resampling=True, interpolation=interp,
                           resampling_coeffs=(0.5, n, -40, 20), windowing=True, window_type=0, window_center=0.5,
                           window_fill=0.9, dispersion=True, dispersion_coeffs=(0, 0, 2, -1), dc_removal=dc,
                           grayscale_min=0, grayscale_max=80)
    raw = np.clip(32768 + np.random.default_rng(interp).normal(0, 3000, (m, n)), 0, 65535).astype(np.uint16)
    be = reflib.RefBackend(p)
    out = be.process(raw)
    be.close()
    st = R.ChainSettings(n=n, resampling=True, interpolation=interp, windowing=True, dispersion=True,
                         dc_removal=dc, grayscale_min=0, grayscale_max=80, ascans_per_bscan=m)
    cur = R.Curves.generated(n, (0.5, n, -40, 20), 0, 0.5, 0.9, (0, 0, 2, -1))
    mine = R.process_buffer(raw, st, cur).output
    assert np.abs(mine - out).max() <= 4e-7 * max(1.0, np.abs(out).max())
