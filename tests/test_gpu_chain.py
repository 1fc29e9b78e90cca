"""GPU parity of the fused chain, called through the C ABI (include/ope_b200.h).

* complex bins: bit-identical to the CPU emulation of the same kernel code
  (whose pre-FFT stages are bit-identical to the oracle restatement, itself
  pinned to the reference);
* images: against the oracle and the golden fixtures with the tolerances of
  tests/test_emulator.py;
* full-size buffers: size-independent properties (A-scan permutation and
  buffer splitting leave every output bit unchanged; repeated runs are
  identical);
* error paths: misaligned buffers and a bounded wait that runs out.
"""
import numpy as np
import pytest

import helpers as H
from octproengine_b200 import capi
from octproengine_b200.chain import (ChainSpec, open_context, UINT8, UINT16, UINT32, FLOAT32, LINEAR, CUBIC,
                                     LANCZOS, GAUSS, HANN)
from oracle import restate as R

pytestmark = pytest.mark.gpu

NS = [512, 1024, 2048, 4096, 8192]
INTERPS = [None, LINEAR, CUBIC, LANCZOS]


def spec_for(n, interp, dtype=UINT16, m=5, **kw):
    base = dict(signal_length=n, ascans_per_bscan=m, input_dtype=dtype, resampling=interp is not None,
                interpolation=interp or 0, resampling_coeffs=(0.5, n, -100.0, 50.0), windowing=True,
                window_type=HANN, window_center=0.5, window_fill=0.9, dispersion=True,
                dispersion_coeffs=(0.0, 0.0, 1.0, -3.0), grayscale_min=0.0, grayscale_max=80.0)
    base.update(kw)
    return ChainSpec(**base)


@pytest.mark.parametrize("interp", INTERPS)
@pytest.mark.parametrize("n", NS)
def test_bins_bit_identical_to_emulation(cuda, emu, n, interp):
    spec = spec_for(n, interp, m=7)
    raw = H.random_raw(spec, seed=n + 1)
    g = H.gpu_run(spec, raw, "bins")
    e = H.emu_run(emu, spec, raw, "bins")
    assert np.array_equal(g.astype(np.complex64), e.astype(np.complex64))


@pytest.mark.parametrize("dtype", [UINT8, UINT16, UINT32, FLOAT32])
@pytest.mark.parametrize("dc", ["off", "exact", "reference"])
def test_dtypes_and_dc_bit_identical_to_emulation(cuda, emu, dtype, dc):
    """Every input type, with rolling-average DC removal off, in exact-sum mode
    and in the reference's float prefix-sum order (whose k-linearised spectrum
    the emulation shows equal to the reference library's, bit for bit)."""
    spec = spec_for(2048, CUBIC, dtype=dtype, m=6, dc_removal=dc != "off", dc_window=64,
                    dc_reference_order=dc == "reference")
    raw = H.random_raw(spec, seed=dtype)
    g = H.gpu_run(spec, raw, "bins")
    e = H.emu_run(emu, spec, raw, "bins")
    assert np.array_equal(g.astype(np.complex64), e.astype(np.complex64))


def test_reference_order_exact_prefix_shortcut_bit_identical_to_emulation(cuda, emu):
    """12-bit samples in reference order: pairs whose row totals stay below
    2^24 take the exact-prefix shortcut, the pair that mixes in a full-range
    16-bit row takes the serial float prefix; both equal the emulation (and so
    the reference library) bit for bit."""
    spec = spec_for(2048, CUBIC, dtype=UINT16, m=6, dc_removal=True, dc_window=64, dc_reference_order=True)
    rng = np.random.default_rng(12)
    raw = rng.integers(0, 4096, size=(6, 2048)).astype(np.uint16)
    raw[5] = rng.integers(30000, 65536, size=2048).astype(np.uint16)
    g = H.gpu_run(spec, raw, "bins")
    e = H.emu_run(emu, spec, raw, "bins")
    assert np.array_equal(g.astype(np.complex64), e.astype(np.complex64))


@pytest.mark.parametrize("n", [512, 1024, 4096, 8192])
def test_reference_order_segments_bit_identical_to_emulation(cuda, emu, n):
    """Full-range 16-bit samples in reference order at every segment count of
    the kernel's segment form of the float prefix (8 segments per row at
    N = 512, where one warp walks both rows, to 128 at N = 8192, four records
    per lane): the GPU's complex bins equal the emulation's (whose k-linearised
    spectrum equals the reference library's) bit for bit. Rows as in the
    emulator's structured-row test: constant 65535, constant 32769 (ties),
    alternating 65535 / 1, values 2 mod 4 near the top, random."""
    rng = np.random.default_rng(n + 7)
    i = np.arange(n)
    raw = np.stack([np.full(n, 65535), np.full(n, 32769), np.where(i % 2 == 1, 65535, 1),
                    65530 - 4 * rng.integers(0, 8, size=n), rng.integers(0, 65536, size=n),
                    rng.integers(30000, 65536, size=n)]).astype(np.uint16)
    spec = spec_for(n, CUBIC, dtype=UINT16, m=raw.shape[0], dc_removal=True, dc_window=64, dc_reference_order=True)
    g = H.gpu_run(spec, raw, "bins")
    e = H.emu_run(emu, spec, raw, "bins")
    assert np.array_equal(g.astype(np.complex64), e.astype(np.complex64))


@pytest.mark.parametrize("dtype", [UINT8, UINT16, FLOAT32])
@pytest.mark.parametrize("n", [512, 1024, 4096, 8192])
def test_exact_sum_dc_removal_bit_identical_to_emulation(cuda, emu, n, dtype):
    """Rolling-average DC removal with exact window sums at every length: the
    interior chunks' window means come from paired prefix entries (and, for 8-
    and 16-bit samples, sums converted as (2^23 + S) - 2^23), the edge chunks'
    from single entries with the correctly rounded division; the GPU's complex
    bins equal the emulation's bit for bit."""
    spec = spec_for(n, CUBIC, dtype=dtype, m=5, dc_removal=True, dc_window=64)
    raw = H.random_raw(spec, seed=n + 11 * dtype)
    g = H.gpu_run(spec, raw, "bins")
    e = H.emu_run(emu, spec, raw, "bins")
    assert np.array_equal(g.astype(np.complex64), e.astype(np.complex64))


@pytest.mark.parametrize("interp", INTERPS)
@pytest.mark.parametrize("n", [512, 2048, 8192])
def test_image_vs_oracle(cuda, n, interp):
    spec = spec_for(n, interp, m=9)
    raw = H.random_raw(spec, seed=3)
    img = H.gpu_run(spec, raw)
    ref = H.oracle_image(spec, raw).output
    f64 = H.oracle_image(spec, raw, mode="f64").output
    err_gpu = np.abs(H.to_db(img, spec) - H.to_db(f64, spec)).max()
    err_cpu = np.abs(H.to_db(ref, spec) - H.to_db(f64, spec)).max()
    # the GPU (float32 DFT, exact DC split) is no further from float64 than the
    # reference arithmetic evaluated with an exact DFT, plus 1e-2 dB
    assert err_gpu <= err_cpu + 1e-2, (err_gpu, err_cpu)


@pytest.mark.parametrize("case", H.golden_cases(), ids=lambda c: c[0])
def test_golden_fixtures(cuda, case):
    name, spec, d = case
    fpn = d["fpn"] if spec.fpn_removal else None
    img = H.gpu_run(spec, d["raw"], fpn_profile=fpn)
    st, cur = H.oracle_settings(spec)
    res64 = R.process_buffer(d["raw"], st, cur, mode="f64", fpn_profile=fpn, keep=True)
    f64 = res64.output
    ref32 = d["out_f32fft"]
    if spec.log_scaling and spec.grayscale_min != spec.grayscale_max:
        k_db, r_db, t_db = H.to_db(img, spec), H.to_db(ref32, spec), H.to_db(f64, spec)
        err_kernel = np.abs(k_db - t_db)
        assert err_kernel.max() <= max(2.0 * np.abs(r_db - t_db).max(), 5e-3)
        # displayed bins, leaving out those where the FPN subtraction cancels
        # more than 20 dB (kappa > 10), which multiplies any float32 rounding
        display = (t_db >= spec.grayscale_min) & (H.fpn_kappa(spec, res64.ifft, fpn) <= 10.0)
        assert err_kernel[display].max() < 1e-2
    else:
        err_kernel = np.abs(img.astype(np.float64) - f64).max()
        err_ref = np.abs(ref32.astype(np.float64) - f64).max()
        assert err_kernel <= max(2.0 * err_ref, 1e-5 * np.abs(f64).max())


def test_fpn_determination_matches_oracle(cuda):
    """requestFixedPatternNoiseDetermination + removal in one frame, as
    computeFixedPatternNoiseIfRequested (cpu_backend.cpp:305-357) does for the
    first frame: profile from the first fpn_bscan_count*A A-scans."""
    spec = spec_for(1024, CUBIC, m=64, ascans_per_bscan=64, bscans_per_buffer=2, fpn_removal=True,
                    grayscale_min=20.0, grayscale_max=110.0)
    raw = H.random_raw(spec, seed=21)
    ctx = open_context(spec)
    try:
        img = H.gpu_run(spec, raw, ctx=ctx, fpn_request=True)
        prof = ctx.fpn_profile()
    finally:
        ctx.close()
    res = H.oracle_image(spec, raw, determine_fpn=True)
    assert prof.size == spec.signal_length  # N/2 complex pairs
    scale = np.abs(res.fpn_profile).max()
    assert np.abs(prof - res.fpn_profile).max() <= 1e-5 * scale
    f64 = H.oracle_image(spec, raw, mode="f64", fpn_profile=res.fpn_profile).output
    err = np.abs(H.to_db(img, spec) - H.to_db(f64, spec))
    assert err[H.to_db(f64, spec) >= spec.grayscale_min].max() < 1e-2


def test_fpn_accumulates_across_buffers(cuda):
    """fpn_bscan_count larger than one buffer: the determination completes on
    the buffer that brings the count to fpn_bscan_count*A A-scans."""
    spec = spec_for(512, LINEAR, m=32, ascans_per_bscan=32, bscans_per_buffer=1, fpn_removal=True,
                    fpn_bscan_count=2)
    r1 = H.random_raw(spec, seed=31)
    r2 = H.random_raw(spec, seed=32)
    ctx = open_context(spec)
    try:
        ctx.request_fpn_determination()
        H.gpu_run(spec, r1, ctx=ctx)
        assert ctx.fpn_profile().size == 0
        H.gpu_run(spec, r2, ctx=ctx)
        prof = ctx.fpn_profile()
    finally:
        ctx.close()
    st, cur = H.oracle_settings(spec)
    X = R.inverse_dft(R.fft_input(np.concatenate([r1, r2]), st, cur)).astype(np.complex64)
    want = R.min_var_mean(X, 8)[:512]
    assert np.abs(prof - want).max() <= 1e-5 * np.abs(want).max()


def test_full_size_properties(cuda):
    """2048 x 1024 x 8 uint16: A-scans are independent, so permuting the input
    rows permutes the output rows and splitting the buffer changes nothing,
    bit for bit; a sample of rows matches the oracle."""
    import torch
    spec = spec_for(2048, LANCZOS, m=1024, ascans_per_bscan=1024, bscans_per_buffer=8, window_type=GAUSS)
    m = spec.num_ascans
    from octproengine_b200 import synth
    x = synth.generate(synth.SynthParams(n=2048, ascans=1024, bscans=8, seed=5), device="cuda:0")
    ctx = open_context(spec)
    try:
        out = torch.empty((m, 1024), dtype=torch.float32, device="cuda:0")
        s = torch.cuda.current_stream().cuda_stream
        ctx.process_device(x.data_ptr(), out.data_ptr(), s)
        out2 = torch.empty_like(out)
        ctx.process_device(x.data_ptr(), out2.data_ptr(), s)
        perm = torch.randperm(m, generator=torch.Generator().manual_seed(0)).to("cuda:0")
        xp = x[perm].contiguous()
        outp = torch.empty_like(out)
        ctx.process_device(xp.data_ptr(), outp.data_ptr(), s)
        half = m // 2 + 1
        outs = torch.empty_like(out)
        ctx.process_device(x.data_ptr(), outs.data_ptr(), s, num_ascans=half)
        ctx.process_device(x[half:].contiguous().data_ptr(), outs[half:].data_ptr(), s, num_ascans=m - half)
        torch.cuda.synchronize()
        assert ctx.synchronize() == 0
    finally:
        ctx.close()
    assert torch.equal(out, out2)
    assert torch.equal(outp, out[perm])
    assert torch.equal(outs, out)
    rows = np.array([0, 1, 777, 4096, m - 1])
    raw = x[torch.from_numpy(rows).to("cuda:0")].cpu().numpy().view(np.uint16)
    ref = H.oracle_image(spec.with_(ascans_per_bscan=len(rows), bscans_per_buffer=1), raw).output
    got = out[torch.from_numpy(rows).to("cuda:0")].cpu().numpy()
    assert np.abs(H.to_db(got, spec) - H.to_db(ref, spec)).max() < 1e-2


def test_misaligned_input_rejected(cuda):
    import torch
    spec = spec_for(512, LINEAR, m=4)
    ctx = open_context(spec)
    try:
        buf = torch.zeros(512 * 4 * 2 + 64, dtype=torch.uint8, device="cuda:0")
        out = torch.empty((4, 256), dtype=torch.float32, device="cuda:0")
        with pytest.raises(capi.B200Error) as ei:
            ctx.process_device(buf.data_ptr() + 2, out.data_ptr())
        assert ei.value.code == capi.E_INVALID
        for bad_out in (out.data_ptr() + 2, 0):  # output not float-aligned; null output
            with pytest.raises(capi.B200Error) as ei:
                ctx.process_device(buf.data_ptr(), bad_out)
            assert ei.value.code == capi.E_INVALID
        with pytest.raises(capi.B200Error) as ei:  # an empty buffer is an error, as in the reference
            ctx.process_device(buf.data_ptr(), out.data_ptr(), num_ascans=0)
        assert ei.value.code == capi.E_INVALID
        with pytest.raises(capi.B200Error):
            ctx.process_device(0, out.data_ptr())  # null input
    finally:
        ctx.close()


def test_bounded_wait_reports_timeout_and_context_recovers(cuda):
    """The first input copy is withheld: the kernel's bounded wait runs out,
    it records a status and returns; the next frame on the same context is
    correct."""
    spec = spec_for(1024, LINEAR, m=6)
    raw = H.random_raw(spec, seed=2)
    ctx = open_context(spec)
    try:
        ctx.inject_copy_stall(2000)  # 2 ms
        with pytest.raises(AssertionError):
            H.gpu_run(spec, raw, ctx=ctx)  # synchronize() reports the status
        img = H.gpu_run(spec, raw, ctx=ctx)
    finally:
        ctx.close()
    ref = H.oracle_image(spec, raw).output
    assert np.abs(H.to_db(img, spec) - H.to_db(ref, spec)).max() < 1e-2


def test_timeout_with_copy_in_flight_waits_it_out(cuda):
    """Every CTA's first wait is treated as run out while its input copy is in
    flight: the CTA waits that copy out (a second bound) before it returns, so
    the status holds the timeout bit alone, never 'copy pending', and the next
    frame on the same context is correct."""
    import torch
    spec = spec_for(2048, CUBIC, m=40)
    raw = H.random_raw(spec, seed=12)
    ctx = open_context(spec)
    try:
        d_in = torch.from_numpy(np.ascontiguousarray(raw).view(np.uint8).reshape(-1).copy()).to("cuda:0")
        d_out = torch.empty((spec.num_ascans, 1024), dtype=torch.float32, device="cuda:0")
        ctx.inject_wait_abort()
        ctx.process_device(d_in.data_ptr(), d_out.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert ctx.synchronize() == 1  # STATUS_MBAR_TIMEOUT, no STATUS_COPY_PENDING
        img = H.gpu_run(spec, raw, ctx=ctx)
    finally:
        ctx.close()
    assert np.array_equal(img, H.gpu_run(spec, raw))


def test_process_host_roundtrip(cuda):
    spec = spec_for(2048, CUBIC, m=12)
    raw = H.random_raw(spec, seed=4)
    ctx = open_context(spec)
    try:
        a = ctx.process_host(raw)
    finally:
        ctx.close()
    b = H.gpu_run(spec, raw)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("bscans,flip", [(7, True), (20, False), (4, True)])
def test_pipelined_process_host_matches_device_path(cuda, bscans, flip):
    # process_host splits buffers of >= 4 B-scans into chunks of B-scan pairs
    # whose copies overlap the chain; every output bit must match one launch
    spec = spec_for(1024, LANCZOS, m=16).with_(bscans_per_buffer=bscans, bscan_flip=flip, fpn_removal=True)
    raw = H.random_raw(spec, seed=bscans)
    prof = np.random.default_rng(2).normal(0, 500, 1024).astype(np.float32)
    ctx = open_context(spec)
    try:
        ctx.set_fpn_profile(prof)
        a = ctx.process_host(raw)
        assert ctx.synchronize() == 0
    finally:
        ctx.close()
    b = H.gpu_run(spec, raw, fpn_profile=prof)
    assert np.array_equal(a, b)


def _bg_spec(**kw):
    return spec_for(2048, CUBIC, m=40).with_(grayscale_min=10.0, grayscale_max=90.0, **kw)


def test_post_process_background_subtraction_is_exact(cuda):
    # applyPostProcessBackgroundSubtraction (cpu_kernels.tpp:381-400):
    # out - (weight * profile + offset), the last operation on each value
    import ctypes
    base = _bg_spec()
    spec = base.with_()
    raw = H.random_raw(spec, seed=31)
    plain = H.gpu_run(base, raw)
    prof = np.random.default_rng(5).uniform(0.0, 0.5, 1024).astype(np.float32)
    cfg = spec.to_config()
    cfg.post_bg_removal = 1
    cfg.bg_weight = 0.75
    cfg.bg_offset = -0.125
    ctx = capi.Context(cfg)
    r, w, cs = spec.curves()
    ctx.set_resampling_curve(r)
    ctx.set_window_curve(w)
    ctx.set_dispersion_curve(cs)
    try:
        capi._check(ctx.h, capi.lib().ope_b200_set_bg_profile(ctx.h, capi.fptr(prof), prof.size))
        got = H.gpu_run(spec, raw, ctx=ctx)
    finally:
        ctx.close()
    bgv = (np.float32(0.75) * prof + np.float32(-0.125)).astype(np.float32)
    assert np.array_equal(got, (plain - bgv[None, :]).astype(np.float32))
    st = R.ChainSettings(n=2048, resampling=True, interpolation=CUBIC, windowing=True, dispersion=True,
                         grayscale_min=10.0, grayscale_max=90.0, ascans_per_bscan=40, post_bg_removal=True,
                         bg_weight=0.75, bg_offset=-0.125)
    ref = R.process_buffer(raw, st, R.Curves(r, w, cs[0::2].copy(), cs[1::2].copy()), bg_profile=prof).output
    assert np.abs(got - ref).max() * 80.0 < 1e-2


def test_post_process_background_recording(cuda):
    # recordPostProcessBackground (cpu_backend.cpp:105-118): float sum over the
    # frame's A-scans in order, divided by their count; then subtracted from
    # the same frame (cpu_backend.cpp:283-301)
    import ctypes
    spec = _bg_spec()
    raw = H.random_raw(spec, seed=32)
    plain = H.gpu_run(spec, raw)
    acc = np.zeros(1024, np.float32)
    for row in plain:
        acc = (acc + row).astype(np.float32)
    want_prof = (acc / np.float32(plain.shape[0])).astype(np.float32)
    cfg = spec.to_config()
    cfg.post_bg_removal = 1
    cfg.bg_weight = 1.0
    cfg.bg_offset = 0.0
    ctx = capi.Context(cfg)
    r, w, cs = spec.curves()
    ctx.set_resampling_curve(r)
    ctx.set_window_curve(w)
    ctx.set_dispersion_curve(cs)
    try:
        capi._check(ctx.h, capi.lib().ope_b200_request_bg_recording(ctx.h))
        first = H.gpu_run(spec, raw, ctx=ctx)
        prof = np.zeros(1024, np.float32)
        n = ctypes.c_size_t(0)
        capi._check(ctx.h, capi.lib().ope_b200_get_bg_profile(ctx.h, capi.fptr(prof), 1024, ctypes.byref(n)))
        raw2 = H.random_raw(spec, seed=33)
        second = H.gpu_run(spec, raw2, ctx=ctx)  # subtracts the recorded profile
        assert ctx.synchronize() == 0
    finally:
        ctx.close()
    assert n.value == 1024 and np.array_equal(prof, want_prof)
    assert np.array_equal(first, (plain - want_prof[None, :]).astype(np.float32))
    plain2 = H.gpu_run(spec, raw2)
    assert np.array_equal(second, (plain2 - want_prof[None, :]).astype(np.float32))


@pytest.mark.parametrize("with_bg", [False, True])
def test_sinusoidal_scan_correction(cuda, with_bg):
    # sinusoidalScanCorrection of the reference CUDA backend (cuda_kernels.cu:
    # 408-438): lateral resampling after the flip, before the background
    spec = spec_for(1024, CUBIC, m=64).with_(bscans_per_buffer=3, bscan_flip=True)
    raw = H.random_raw(spec, seed=41)
    plain = H.gpu_run(spec, raw)
    cfg = spec.to_config()
    cfg.sinusoidal_correction = 1
    prof = np.random.default_rng(9).uniform(0, 0.3, 512).astype(np.float32)
    if with_bg:
        cfg.post_bg_removal = 1
        cfg.bg_weight = 2.0
        cfg.bg_offset = 0.25
    ctx = capi.Context(cfg)
    r, w, cs = spec.curves()
    ctx.set_resampling_curve(r)
    ctx.set_window_curve(w)
    ctx.set_dispersion_curve(cs)
    try:
        if with_bg:
            capi._check(ctx.h, capi.lib().ope_b200_set_bg_profile(ctx.h, capi.fptr(prof), prof.size))
        got = H.gpu_run(spec, raw, ctx=ctx)
        assert ctx.synchronize() == 0
    finally:
        ctx.close()
    want = R.sinusoidal_correction(plain, 64)
    if with_bg:
        want = (want - (np.float32(2.0) * prof + np.float32(0.25))[None, :]).astype(np.float32)
    assert np.array_equal(got[-1], want[-1])  # last A-scan passes through
    # the curve comes from the device acosf, the restatement from numpy's: a
    # last-bit difference in x (ulp up to 4e-6 for x < 64) moves the fraction,
    # so outputs agree to |f1 - f0| * 4e-6 rather than to the last bit
    assert np.allclose(got, want, rtol=0, atol=1e-5), np.abs(got - want).max()


@pytest.mark.parametrize("dtype", [UINT8, UINT16])
@pytest.mark.parametrize("dc", [False, True])
def test_bitshift_equals_the_pre_shifted_input(cuda, dtype, dc):
    """DataParameters::bitshift (the reference GPU path's rule: 8/16-bit samples
    >> 4) gives every bit of the image of the input shifted on the host;
    32-bit samples ignore the flag."""
    spec = spec_for(1024, CUBIC, dtype=dtype, m=7, dc_removal=dc, dc_window=32)
    raw = H.random_raw(spec, seed=4)
    got = H.gpu_run(spec.with_(bitshift=True), raw)
    want = H.gpu_run(spec, (raw >> 4).astype(raw.dtype))
    assert np.array_equal(got, want)
    assert not np.array_equal(got, H.gpu_run(spec, raw))


def test_bitshift_ignored_for_32_bit_samples(cuda):
    spec = spec_for(512, LINEAR, dtype=UINT32, m=4)
    raw = H.random_raw(spec, seed=5)
    assert np.array_equal(H.gpu_run(spec.with_(bitshift=True), raw), H.gpu_run(spec, raw))
