"""The streaming paths on the device: the C ABI's frame ring and the
reference-facing Processor API (Python module and C++ library) over it.

Every frame delivered through the ring or a Processor callback must be
bit-identical to ope_b200_process_host on the same input with the same
configuration (the same kernels run; only the buffering differs), and frames
arrive in submission order (src/core/processor.cpp:279-282 of the reference:
process() is asynchronous, outputs come back through the callbacks).
"""
import os
import subprocess
import threading

import numpy as np
import pytest

import helpers as H
import octproengine_b200 as pkg
from octproengine_b200 import build as B
from octproengine_b200 import capi
from octproengine_b200.chain import ChainSpec, open_context, CUBIC, GAUSS, HANN

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _spec(n=2048, a=256, b=2, **kw):
    base = dict(signal_length=n, ascans_per_bscan=a, bscans_per_buffer=b, resampling=True, interpolation=CUBIC,
                resampling_coeffs=(0.5, float(n - 1) - 40.0, 60.0, -20.0), windowing=True, window_type=GAUSS,
                window_center=0.5, window_fill=0.9, dispersion=True, dispersion_coeffs=(0.0, 0.0, 2.0, -1.0),
                grayscale_min=20.0, grayscale_max=90.0)
    base.update(kw)
    return ChainSpec(**base)


def _frames(spec, count, seed=5):
    return [H.random_raw(spec, seed=seed + i) for i in range(count)]


def _reference_outputs(spec, frames):
    with open_context(spec) as ctx:
        return [ctx.process_host(f).copy() for f in frames]


# ---------------------------------------------------------------- C ABI ring


def test_ring_submit_wait_release(cuda):
    import torch
    spec = _spec()
    frames = _frames(spec, 7)
    want = _reference_outputs(spec, frames)
    with open_context(spec) as ctx:
        depth = capi.lib().ope_b200_ring_depth(ctx.h)
        assert depth >= 2
        pinned = [torch.from_numpy(f.view(np.uint8).reshape(-1).copy()).pin_memory() for f in frames]
        tickets = []
        for k in range(depth):
            tickets.append(ctx.submit(pinned[k].data_ptr()))
        with pytest.raises(capi.B200Error) as ei:  # every slot holds an unreleased frame
            ctx.submit(pinned[depth].data_ptr())
        assert ei.value.code == capi.E_STATE
        nxt = depth
        done = 0
        while done < len(frames):
            t = tickets[done]
            ctx.input_released(t, 20000)
            out = ctx.wait(t, 20000)
            np.testing.assert_array_equal(out, want[done])
            ctx.release(t)
            with pytest.raises(capi.B200Error):
                ctx.release(t)  # released twice
            done += 1
            if nxt < len(frames):
                tickets.append(ctx.submit(pinned[nxt].data_ptr()))
                nxt += 1
        assert tickets == list(range(1, len(frames) + 1))


def test_ring_submit_to_caller_buffers(cuda):
    import torch
    spec = _spec(n=1024, a=512, b=1)
    frames = _frames(spec, 4, seed=40)
    want = _reference_outputs(spec, frames)
    m, half = spec.num_ascans, spec.signal_length // 2
    with open_context(spec) as ctx:
        ins = [torch.from_numpy(f.view(np.uint8).reshape(-1).copy()).pin_memory() for f in frames]
        outs = [torch.empty((m, half), dtype=torch.float32).pin_memory() for _ in frames]
        for i in range(0, len(frames), 2):
            ts = [ctx.submit_to(ins[j].data_ptr(), outs[j].data_ptr()) for j in (i, i + 1)]
            for t, j in zip(ts, (i, i + 1)):
                view = ctx.wait(t, 20000)
                assert view.ctypes.data == outs[j].data_ptr()  # the output went where it was asked to
                ctx.release(t)
                np.testing.assert_array_equal(outs[j].numpy(), want[j])


def test_frame_device_input_is_the_submitted_frame(cuda):
    import torch
    from octproengine_b200.autofocus import frame_input_view
    spec = _spec(n=1024, a=256, b=2)
    frames = _frames(spec, 3, seed=41)
    want = _reference_outputs(spec, frames)
    side = torch.cuda.Stream()
    with open_context(spec) as ctx:
        pinned = [torch.from_numpy(f.view(np.uint8).reshape(-1).copy()).pin_memory() for f in frames]
        tickets = [ctx.submit(p.data_ptr()) for p in pinned[:2]]
        for k, t in enumerate(tickets):
            view = frame_input_view(ctx, t, spec.num_ascans, side)  # side waits for the input copy
            with torch.cuda.stream(side):
                got = view.clone()
            side.synchronize()
            assert np.array_equal(got.cpu().numpy().view(np.uint16), frames[k].reshape(spec.num_ascans, -1))
            np.testing.assert_array_equal(ctx.wait(t, 20000), want[k])
            ctx.release(t)
        with pytest.raises(capi.B200Error):
            ctx.frame_device_input(tickets[0], side.cuda_stream)  # released


# ------------------------------------------------------- Python Processor API


@pytest.fixture(scope="module")
def ope():
    B.build()
    return pkg.reference_api()


def _configure(ope, proc, spec):
    proc.set_input_parameters(spec.signal_length, spec.ascans_per_bscan, spec.bscans_per_buffer,
                              ope.DataType.UINT16)
    proc.set_resampling_coefficients(list(spec.resampling_coeffs))
    proc.enable_resampling(True)
    proc.set_interpolation_method(ope.InterpolationMethod.CUBIC)
    proc.set_window_parameters(ope.WindowType.GAUSS, spec.window_center, spec.window_fill)
    proc.enable_windowing(True)
    proc.set_dispersion_coefficients(list(spec.dispersion_coeffs), 1.0)
    proc.enable_dispersion_compensation(True)
    proc.set_grayscale_range(spec.grayscale_min, spec.grayscale_max)


class _Collector:
    def __init__(self):
        self.frames = []
        self.cv = threading.Condition()

    def __call__(self, arr):
        with self.cv:
            self.frames.append(np.array(arr, copy=True))
            self.cv.notify_all()

    def wait(self, count, timeout=60.0):
        with self.cv:
            ok = self.cv.wait_for(lambda: len(self.frames) >= count, timeout)
        assert ok, f"{len(self.frames)}/{count} frames delivered"
        return self.frames


def _stream(proc, frames):
    for f in frames:
        buf = proc.get_next_available_buffer()
        buf[:] = f.reshape(-1)
        proc.process(buf)


def test_processor_stream_matches_c_abi(ope, cuda):
    spec = _spec()
    frames = _frames(spec, 6, seed=11)
    want = _reference_outputs(spec, frames)
    with ope.Processor(ope.Backend.B200) as proc:
        _configure(ope, proc, spec)
        proc.initialize()
        c1, c2 = _Collector(), _Collector()
        proc.add_output_callback(c1)
        proc.add_output_callback(c2)
        _stream(proc, frames)
        got1, got2 = c1.wait(len(frames)), c2.wait(len(frames))
    assert len(got1) == len(got2) == len(frames)
    for g1, g2, w in zip(got1, got2, want):
        assert g1.dtype == np.float32 and g1.size == w.size
        np.testing.assert_array_equal(g1.reshape(w.shape), w)
        np.testing.assert_array_equal(g2.reshape(w.shape), w)


def test_processor_output_matches_oracle(ope, cuda):
    """One frame of the Processor path against the oracle (the reference CPU
    chain restated), at the same tolerance as the C ABI's image tests."""
    spec = _spec(n=1024, a=128, b=1)
    frame = _frames(spec, 1, seed=3)[0]
    col = _Collector()
    with ope.Processor(ope.Backend.B200) as proc:
        _configure(ope, proc, spec)
        proc.set_callback(col)
        proc.initialize()
        _stream(proc, [frame])
        out = col.wait(1)[0].reshape(spec.num_ascans, spec.signal_length // 2)
    ref = H.oracle_image(spec, frame, mode="f64").output
    err = np.abs(H.to_db(out, spec) - H.to_db(ref, spec))
    assert err.max() < 0.05, err.max()


def test_processor_hot_swap_takes_effect(ope, cuda):
    spec = _spec(n=1024, a=256, b=2)
    frames = _frames(spec, 3, seed=21)
    col = _Collector()
    with ope.Processor(ope.Backend.B200) as proc:
        _configure(ope, proc, spec)
        proc.set_callback(col)
        proc.initialize()
        _stream(proc, frames[:1])
        col.wait(1)
        proc.enable_log_scaling(False)
        proc.set_signal_multiplicator_and_addend(0.5, 0.25)
        _stream(proc, frames[1:2])
        col.wait(2)
        proc.enable_log_scaling(True)
        proc.enable_bscan_flip(True)
        proc.set_window_parameters(ope.WindowType.HANN, 0.5, 0.95)
        _stream(proc, frames[2:3])
        got = col.wait(3)
    want0 = _reference_outputs(spec, frames[:1])[0]
    want1 = _reference_outputs(spec.with_(log_scaling=False, multiplicator=0.5, addend=0.25), frames[1:2])[0]
    want2 = _reference_outputs(spec.with_(bscan_flip=True, window_type=HANN, window_fill=0.95, multiplicator=0.5,
                                          addend=0.25), frames[2:3])[0]
    for g, w in zip(got, [want0, want1, want2]):
        np.testing.assert_array_equal(g.reshape(w.shape), w)


def test_processor_fpn_determination_and_files(ope, cuda, tmp_path):
    spec = _spec(n=1024, a=256, b=2, fpn_removal=True, fpn_bscan_count=1)
    frames = _frames(spec, 2, seed=31)
    col = _Collector()
    with ope.Processor(ope.Backend.B200) as proc:
        _configure(ope, proc, spec)
        proc.enable_fixed_pattern_noise_removal(True)
        proc.set_fixed_pattern_noise_bscan_count(1)
        proc.set_callback(col)
        proc.initialize()
        assert not proc.has_fixed_pattern_noise_profile()
        proc.request_fixed_pattern_noise_determination()
        _stream(proc, frames)
        got = col.wait(2)
        assert proc.has_fixed_pattern_noise_profile()
        assert proc.get_fixed_pattern_noise_profile_size() == spec.signal_length // 2
        prof = proc.get_fixed_pattern_noise_profile()
        path = str(tmp_path / "fpn.csv")
        proc.save_fixed_pattern_noise_profile_to_file(path)
        proc.set_fixed_pattern_noise_profile(np.zeros_like(prof))
        np.testing.assert_array_equal(proc.get_fixed_pattern_noise_profile(), 0.0)
        proc.load_fixed_pattern_noise_profile_from_file(path)
        np.testing.assert_allclose(proc.get_fixed_pattern_noise_profile(), prof, rtol=1e-5, atol=1e-6)
    with open_context(spec) as ctx:
        ctx.request_fpn_determination()
        want = [ctx.process_host(f).copy() for f in frames]
        want_prof = ctx.fpn_profile()
    np.testing.assert_array_equal(prof, want_prof)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g.reshape(w.shape), w)


def test_processor_reinitializes_on_new_dimensions(ope, cuda):
    spec_a = _spec(n=1024, a=128, b=1)
    spec_b = _spec(n=2048, a=64, b=2)
    fa, fb = _frames(spec_a, 1, seed=50)[0], _frames(spec_b, 1, seed=51)[0]
    col = _Collector()
    with ope.Processor(ope.Backend.B200) as proc:
        _configure(ope, proc, spec_a)
        proc.set_callback(col)
        proc.initialize()
        _stream(proc, [fa])
        col.wait(1)
        _configure(ope, proc, spec_b)  # new signal length: the next buffer request re-initializes
        buf = proc.get_next_available_buffer()
        assert buf.size == spec_b.signal_length * spec_b.num_ascans
        buf[:] = fb.reshape(-1)
        proc.process(buf)
        got = col.wait(2)
    np.testing.assert_array_equal(got[0].reshape(spec_a.num_ascans, -1), _reference_outputs(spec_a, [fa])[0])
    np.testing.assert_array_equal(got[1].reshape(spec_b.num_ascans, -1), _reference_outputs(spec_b, [fb])[0])


# --------------------------------------------------------- C++ Processor API


def test_cpp_processor_stream(cuda, tmp_path):
    B.build()
    exe = str(tmp_path / "processor_stream")
    src = os.path.join(ROOT, "tests", "cpp", "processor_stream.cpp")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "include", "ope"), src,
                        "-o", exe, "-L", B.LIBDIR, "-lope_host", "-lope_b200", "-Wl,-rpath," + B.LIBDIR],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    spec = _spec(n=2048, a=256, b=2)
    frames = _frames(spec, 5, seed=61)
    raw_path, out_path = str(tmp_path / "in.raw"), str(tmp_path / "out.f32")
    np.concatenate([f.reshape(-1) for f in frames]).astype(np.uint16).tofile(raw_path)
    r = subprocess.run([exe, raw_path, out_path, str(spec.signal_length), str(spec.ascans_per_bscan),
                        str(spec.bscans_per_buffer), str(len(frames))], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-3000:]
    got = np.fromfile(out_path, dtype=np.float32).reshape(len(frames), spec.num_ascans, -1)
    want = _reference_outputs(spec, frames)
    for g, w in zip(got, want):
        np.testing.assert_array_equal(g, w)


def test_ring_with_sinusoidal_correction_and_background(cuda):
    # the sinusoidal scratch image is shared by the context: frames that overlap
    # on the ring's streams must still come out as one-at-a-time processing
    import torch
    spec = _spec(n=1024, a=64, b=2)
    cfg = spec.to_config()
    cfg.sinusoidal_correction = 1
    cfg.post_bg_removal = 1
    cfg.bg_weight = 0.5
    cfg.bg_offset = 0.1
    frames = _frames(spec, 6, seed=60)
    prof = np.linspace(0.0, 0.2, 512, dtype=np.float32)

    def make():
        ctx = capi.Context(cfg)
        r, w, cs = spec.curves()
        ctx.set_resampling_curve(r)
        ctx.set_window_curve(w)
        ctx.set_dispersion_curve(cs)
        capi._check(ctx.h, capi.lib().ope_b200_set_bg_profile(ctx.h, capi.fptr(prof), prof.size))
        return ctx

    ref = make()
    try:
        want = [ref.process_host(f).copy() for f in frames]
    finally:
        ref.close()
    ctx = make()
    try:
        pinned = [torch.from_numpy(f.view(np.uint8).reshape(-1).copy()).pin_memory() for f in frames]
        depth = capi.lib().ope_b200_ring_depth(ctx.h)
        tickets = [ctx.submit(pinned[k].data_ptr()) for k in range(depth)]
        nxt, done = depth, 0
        while done < len(frames):
            out = ctx.wait(tickets[done], 20000)
            np.testing.assert_array_equal(out, want[done])
            ctx.release(tickets[done])
            done += 1
            if nxt < len(frames):
                tickets.append(ctx.submit(pinned[nxt].data_ptr()))
                nxt += 1
        assert ctx.synchronize() == 0
    finally:
        ctx.close()
