"""The chain kernel's own phase functions, run on the CPU by tests/emu, against
the oracle: the pre-FFT stages bit for bit, the FFT to float32 accuracy, the
output within the stated tolerances. Every shared-memory index is
bounds-checked by the emulation."""
import numpy as np
import pytest

import helpers as H
from octproengine_b200.chain import ChainSpec, UINT8, UINT16, UINT32, FLOAT32, LINEAR, CUBIC, LANCZOS
from oracle import restate as R

NS = [512, 1024, 2048, 4096, 8192]
INTERPS = [None, LINEAR, CUBIC, LANCZOS]


def spec_for(n, interp, dtype=UINT16, m=5, **kw):
    base = dict(signal_length=n, ascans_per_bscan=m, input_dtype=dtype, resampling=interp is not None,
                interpolation=interp or 0, resampling_coeffs=(0.5, n, -100.0, 50.0), windowing=True,
                window_type=0, window_center=0.5, window_fill=0.9, dispersion=True,
                dispersion_coeffs=(0.0, 0.0, 1.0, -3.0), grayscale_min=0.0, grayscale_max=80.0)
    base.update(kw)
    return ChainSpec(**base)


def oracle_resampled(spec, raw):
    """The oracle's spectrum after unpack, DC removal and k-linearisation."""
    st, cur = H.oracle_settings(spec.with_(windowing=False, dispersion=False))
    return R.fft_input(raw, st, cur).real


def assert_fft_input_close(spec, z, raw):
    """Window x phase is applied as one folded factor (w cos, w sin), so the
    DFT input differs from the reference's (y w) cos by at most a few ulp."""
    st, cur = H.oracle_settings(spec)
    zr = R.fft_input(raw, st, cur)
    scale = np.maximum(np.abs(zr), 1e-30)
    assert (np.abs(z - zr) / scale).max() < 4e-7


@pytest.mark.parametrize("interp", INTERPS)
@pytest.mark.parametrize("n", NS)
def test_resampled_bit_exact(emu, n, interp):
    """Unpack, indexing and the interpolation arithmetic equal the reference bit for bit."""
    spec = spec_for(n, interp, dc_split=False)
    raw = H.random_raw(spec, seed=n)
    y = H.emu_run(emu, spec, raw, "resampled")
    assert np.array_equal(y, oracle_resampled(spec, raw))
    assert_fft_input_close(spec, H.emu_run(emu, spec, raw, "fft_input"), raw)


@pytest.mark.parametrize("dtype", [UINT8, UINT16, UINT32, FLOAT32])
def test_resampled_dtypes_bit_exact(emu, dtype):
    spec = spec_for(1024, CUBIC, dtype=dtype, m=3, dc_split=False)
    raw = H.random_raw(spec, seed=dtype)
    assert np.array_equal(H.emu_run(emu, spec, raw, "resampled"), oracle_resampled(spec, raw))


def test_float32_as_uint32_quirk(emu):
    """With float32_as_uint32 the bytes are read as uint32 (cpu_kernels.tpp:47-52)."""
    spec = spec_for(512, LINEAR, dtype=FLOAT32, m=2, float32_as_uint32=True, dc_split=False)
    raw = H.random_raw(spec, seed=3)
    assert np.array_equal(H.emu_run(emu, spec, raw, "resampled"), oracle_resampled(spec, raw))


@pytest.mark.parametrize("n", NS)
def test_fft_accuracy(emu, n):
    spec = spec_for(n, LINEAR, m=4, dc_split=False)
    raw = H.random_raw(spec, seed=1)
    z = H.emu_run(emu, spec, raw, "fft_input")
    X = H.emu_run(emu, spec, raw, "bins")
    X64 = R.inverse_dft(z)[:, : n // 2]
    rel = np.abs(X - X64).max() / np.abs(X64).max()
    assert rel < 4e-7, rel


@pytest.mark.parametrize("n", [512, 2048, 8192])
def test_dc_removal_exact_rolling_mean(emu, n):
    """Rolling-average DC removal uses exact integer window sums: the spectrum
    matches the float64 evaluation of the reference formula to float32
    rounding (the reference's own float prefix sum is less accurate)."""
    spec = spec_for(n, CUBIC, m=4, dc_removal=True, dc_window=64)
    raw = H.random_raw(spec, seed=2)
    y = H.emu_run(emu, spec, raw, "resampled")
    st, cur = H.oracle_settings(spec.with_(windowing=False, dispersion=False))
    y64 = R.fft_input(raw, st, cur, mode="f64").real
    yref = R.fft_input(raw, st, cur).real
    err_gpu = np.abs(y - y64).max()
    err_ref = np.abs(yref - y64).max()
    assert err_gpu < 4e-3
    assert err_gpu <= err_ref


@pytest.mark.parametrize("window", [32, 50, 7])
def test_dc_removal_small_sums_bit_exact(emu, window):
    """While the reference's float prefix sum stays below 2^24 it is exact and
    both agree bit for bit (uint8 input). Windows of 2W = 64 (a power of two:
    the interior mean is a multiplication by the exact reciprocal), 100 and 14
    (divisions)."""
    spec = spec_for(1024, LINEAR, dtype=UINT8, m=4, dc_removal=True, dc_window=window)
    raw = H.random_raw(spec, seed=9)
    assert np.array_equal(H.emu_run(emu, spec, raw, "resampled"), oracle_resampled(spec, raw))


@pytest.mark.parametrize("n", [512, 2048, 4096])
@pytest.mark.parametrize("interp", INTERPS)
def test_image_vs_oracle(emu, n, interp):
    spec = spec_for(n, interp, m=6)
    raw = H.random_raw(spec, seed=5)
    img = H.emu_run(emu, spec, raw, "image")
    ref = H.oracle_image(spec, raw).output
    db = np.abs(H.to_db(img, spec) - H.to_db(ref, spec))
    assert db.max() < 5e-3, db.max()


def test_odd_count_single_row_last_pair(emu):
    spec = spec_for(1024, LINEAR, m=7)
    raw = H.random_raw(spec, seed=4)
    img = H.emu_run(emu, spec, raw, "image")
    ref = H.oracle_image(spec, raw).output
    assert np.abs(H.to_db(img, spec) - H.to_db(ref, spec)).max() < 5e-3


def test_linear_scaling(emu):
    spec = spec_for(1024, CUBIC, m=4, log_scaling=False, grayscale_min=0.0, grayscale_max=3.0, multiplicator=2.0,
                    addend=0.25)
    raw = H.random_raw(spec, seed=6)
    img = H.emu_run(emu, spec, raw, "image")
    ref = H.oracle_image(spec, raw).output
    # FFT rounding is relative to the strongest bin of the A-scan
    assert np.abs(img - ref).max() <= 2e-6 * np.abs(ref).max()


def test_auto_minmax(emu):
    spec = spec_for(2048, None, m=4, grayscale_min=40.0, grayscale_max=40.0, multiplicator=1.5, addend=0.1)
    raw = H.random_raw(spec, seed=8)
    img = H.emu_run(emu, spec, raw, "image")
    ref = H.oracle_image(spec, raw).output
    np.testing.assert_allclose(img, ref, rtol=0, atol=2e-5)


def test_fpn_profile_subtraction(emu):
    spec = spec_for(1024, LINEAR, m=4, fpn_removal=True)
    raw = H.random_raw(spec, seed=10)
    rng = np.random.default_rng(1)
    prof = (rng.normal(0, 2000, 1024)).astype(np.float32)  # 512 complex pairs
    img = H.emu_run(emu, spec, raw, "image", fpn=prof)
    ref = H.oracle_image(spec, raw, fpn_profile=prof).output
    assert np.abs(H.to_db(img, spec) - H.to_db(ref, spec)).max() < 5e-3


def test_bscan_flip_row_mapping(emu):
    """Flip mirrors B-scan b laterally when b is even and b+1 exists
    (cuda_kernels.cu:553-573): B-scans 0 and 2 of 3 -> only 0 is flipped."""
    base = spec_for(512, LINEAR, m=4, ascans_per_bscan=4, bscans_per_buffer=3)
    raw = H.random_raw(base, seed=11)
    a = H.emu_run(emu, base, raw, "image")
    b = H.emu_run(emu, base.with_(bscan_flip=True), raw, "image")
    assert np.array_equal(b[0:4], a[0:4][::-1])
    assert np.array_equal(b[4:12], a[4:12])


@pytest.mark.parametrize("case", H.golden_cases(), ids=lambda c: c[0])
def test_emulated_kernel_vs_golden(emu, case):
    """Kernel error against float64 is no larger than the reference's own error
    when its DFT runs in float32 (``out_f32fft``), and small on the display
    range [grayscale_min, inf) in dB."""
    name, spec, d = case
    fpn = d["fpn"] if spec.fpn_removal else None
    img = H.emu_run(emu, spec, d["raw"], "image", fpn=fpn)
    st, cur = H.oracle_settings(spec)
    res64 = R.process_buffer(d["raw"], st, cur, mode="f64", fpn_profile=fpn, keep=True)
    f64 = res64.output
    ref32 = d["out_f32fft"]
    if spec.log_scaling and spec.grayscale_min != spec.grayscale_max:
        k_db, r_db, t_db = H.to_db(img, spec), H.to_db(ref32, spec), H.to_db(f64, spec)
        err_kernel = np.abs(k_db - t_db)
        err_ref = np.abs(r_db - t_db)
        assert err_kernel.max() <= max(2.0 * err_ref.max(), 5e-3)
        # displayed bins, leaving out those where the FPN subtraction cancels
        # more than 20 dB (kappa > 10), which multiplies any float32 rounding
        display = (t_db >= spec.grayscale_min) & (H.fpn_kappa(spec, res64.ifft, fpn) <= 10.0)
        assert err_kernel[display].max() < 1e-2
    else:
        # linear scaling, or log scaling with the automatic per-A-scan range
        # (normalised by the weakest bin, whose float32 error is largest)
        err_kernel = np.abs(img.astype(np.float64) - f64).max()
        err_ref = np.abs(ref32.astype(np.float64) - f64).max()
        assert err_kernel <= max(2.0 * err_ref, 1e-5 * np.abs(f64).max())


@pytest.mark.parametrize("interp", [LINEAR, CUBIC, LANCZOS])
def test_exact_dc_split_accuracy(emu, interp):
    """On spectra with the real DC offset (32768 counts) the float32 DFT error
    floor is set by the DC term; the exact DC split removes it: error against
    float64 drops by an order of magnitude on every bin."""
    from octproengine_b200 import synth
    n, m = 2048, 16
    spec = ChainSpec(signal_length=n, ascans_per_bscan=m, resampling=True, interpolation=interp,
                     resampling_coeffs=synth.linearising_coeffs(n), windowing=True, window_type=0,
                     window_center=0.5, window_fill=0.95, dispersion=True,
                     dispersion_coeffs=synth.compensating_coeffs(10.0, -5.0), grayscale_min=0.0,
                     grayscale_max=100.0)
    raw = synth.as_numpy(synth.generate(synth.SynthParams(n=n, ascans=m, seed=3, d2=10.0, d3=-5.0)), "uint16")
    f64 = H.to_db(H.oracle_image(spec, raw, mode="f64").output, spec)
    on = H.to_db(H.emu_run(emu, spec, raw, "image"), spec)
    off = H.to_db(H.emu_run(emu, spec.with_(dc_split=False), raw, "image"), spec)
    ref = H.to_db(H.oracle_image(spec, raw).output, spec)  # reference arithmetic, float64 DFT
    e_on, e_off, e_ref = np.abs(on - f64), np.abs(off - f64), np.abs(ref - f64)
    hi = f64 >= 0
    assert e_on[hi].max() < 0.4 * e_off[hi].max()
    # no worse than the reference's own float32 stages even with an exact DFT
    assert e_on[hi].max() <= e_ref[hi].max()
    assert e_on[f64 >= 30].max() < 2e-3


@pytest.mark.parametrize("dtype", [UINT16, UINT8, UINT32, FLOAT32])
@pytest.mark.parametrize("n", [1024, 4096])
def test_dc_reference_order_bit_exact_vs_reference_library(emu, reflib, n, dtype):
    """With dc_reference_order the rolling-average DC removal follows the
    reference's sequential float prefix sum: the k-linearised spectrum equals
    the reference library's own convertInput -> rollingAverageDCRemoval ->
    kLinearization bit for bit (cpu_kernels.tpp:56-82,113-146), where the
    prefix sums pass 2^24 and round (the default exact-sum mode differs there)."""
    spec = spec_for(n, CUBIC, dtype=dtype, m=4, dc_removal=True, dc_window=64, dc_reference_order=True,
                    dc_split=False)
    raw = H.random_raw(spec, seed=n + dtype)
    y = H.emu_run(emu, spec, raw, "resampled")
    r, _, _ = spec.curves()
    x = np.stack([reflib.convert_input(row, dtype) for row in raw]) if dtype != FLOAT32 else raw.astype(np.float32)
    ref = np.stack([reflib.klinearization(row, r, CUBIC) for row in reflib.rolling_dc(x, 64)])
    assert np.array_equal(y, ref)
    if dtype == UINT16:  # the prefix sums reach ~1.3e8 > 2^24: the exact-sum mode is not the reference's
        y_exact = H.emu_run(emu, spec.with_(dc_reference_order=False), raw, "resampled")
        assert not np.array_equal(y_exact, ref)


@pytest.mark.parametrize("bits,dtype", [(12, UINT16), (8, UINT8), (16, UINT16)])
def test_dc_reference_order_exact_prefix_shortcut(emu, reflib, bits, dtype):
    """Integer samples whose row totals stay below 2^24 (12-bit samples at
    N = 2048, any 8-bit ones) take the kernel's exact-prefix shortcut in
    reference order; the k-linearised spectrum still equals the reference
    library's bit for bit. One pair mixes a low row with a full-range 16-bit
    row (totals above 2^24), which takes the serial float prefix instead."""
    n = 2048
    spec = spec_for(n, CUBIC, dtype=dtype, m=4, dc_removal=True, dc_window=64, dc_reference_order=True,
                    dc_split=False)
    rng = np.random.default_rng(bits)
    raw = rng.integers(0, 1 << bits, size=(4, n)).astype(np.uint16 if dtype == UINT16 else np.uint8)
    if dtype == UINT16:
        raw[3] = rng.integers(30000, 65536, size=n).astype(np.uint16)  # pair (2, 3): one row above 2^24
    assert (raw[:2].astype(np.int64).sum(axis=1) < (1 << 24)).all() == (bits <= 12)
    y = H.emu_run(emu, spec, raw, "resampled")
    r, _, _ = spec.curves()
    x = np.stack([reflib.convert_input(row, dtype) for row in raw])
    ref = np.stack([reflib.klinearization(row, r, CUBIC) for row in reflib.rolling_dc(x, 64)])
    assert np.array_equal(y, ref)


@pytest.mark.parametrize("n", [2048, 8192])
def test_dc_reference_order_segments_bit_exact_on_structured_rows(emu, reflib, n):
    """16-bit samples in reference order take the kernel's segment form of the
    float prefix (per-binade parity steps, float additions across 2^24 and the
    binade boundaries). Rows built to stress it: constant 65535 (the sum ends
    in the 2^28 binade at N = 8192), constant 32769 (an odd sample: every
    addition in the 2-ulp binade is a tie), alternating 65535 / 1, values
    2 mod 4 near the top (ties in the 4-ulp binade), a full-range random row
    and a high-range one. The k-linearised spectrum equals the reference
    library's convertInput -> rollingAverageDCRemoval -> kLinearization bit
    for bit (cpu_kernels.tpp:24-82,113-146)."""
    rng = np.random.default_rng(n)
    i = np.arange(n)
    raw = np.stack([np.full(n, 65535), np.full(n, 32769), np.where(i % 2 == 1, 65535, 1),
                    65530 - 4 * rng.integers(0, 8, size=n), rng.integers(0, 65536, size=n),
                    rng.integers(30000, 65536, size=n)]).astype(np.uint16)
    spec = spec_for(n, CUBIC, dtype=UINT16, m=raw.shape[0], dc_removal=True, dc_window=64,
                    dc_reference_order=True, dc_split=False)
    y = H.emu_run(emu, spec, raw, "resampled")
    r, _, _ = spec.curves()
    x = np.stack([reflib.convert_input(row, UINT16) for row in raw])
    ref = np.stack([reflib.klinearization(row, r, CUBIC) for row in reflib.rolling_dc(x, 64)])
    assert np.array_equal(y, ref)


@pytest.mark.parametrize("window", [64, 50])
def test_dc_reference_order_matches_restatement(emu, window):
    """The oracle restatement's rolling mean is the reference's float prefix
    sum; the kernel in reference order equals it bit for bit (odd window counts
    use the correctly rounded division)."""
    spec = spec_for(2048, LINEAR, m=4, dc_removal=True, dc_window=window, dc_reference_order=True, dc_split=False)
    raw = H.random_raw(spec, seed=window)
    assert np.array_equal(H.emu_run(emu, spec, raw, "resampled"), oracle_resampled(spec, raw))
