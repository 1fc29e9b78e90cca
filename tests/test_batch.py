"""Batched chain: uneven buffers in one persistent launch (ope_b200_batch_*).

Every buffer of a batch must get exactly the chain a single-buffer call of
its context runs: with the default radix schedule the outputs are compared
bit for bit with ope_b200_process_device_n; with the other schedule (a
different FFT evaluation order) against the oracle in dB. Also: CUDA-graph
replay on new data, every tuning candidate, the autotuner, ragged A-scan
counts, FPN subtraction and argument errors.
"""
import numpy as np
import pytest

import helpers as H
from octproengine_b200 import capi
from octproengine_b200.chain import ChainSpec, open_context, UINT8, UINT16, FLOAT32, LINEAR, CUBIC, LANCZOS, \
    GAUSS, HANN, SINE, RECTANGULAR
from oracle import restate as R

pytestmark = pytest.mark.gpu


def _spec(n, m, dtype, interp, window, seed):
    rng = np.random.default_rng(seed)
    return ChainSpec(signal_length=n, ascans_per_bscan=m, bscans_per_buffer=1, input_dtype=dtype,
                     resampling=interp is not None, interpolation=interp or 0,
                     resampling_coeffs=(0.5, n - 1.0, float(rng.uniform(-120, 120)), float(rng.uniform(-60, 60))),
                     windowing=True, window_type=window, window_center=0.5, window_fill=0.9, dispersion=True,
                     dispersion_coeffs=(0.0, 0.0, float(rng.uniform(-20, 20)), float(rng.uniform(-10, 10))),
                     grayscale_min=0.0, grayscale_max=90.0)


def _case(count=9, seed=1):
    rng = np.random.default_rng(seed)
    lens = [1024, 2048, 4096]
    dtypes = [UINT8, UINT16, FLOAT32]
    interps = [None, LINEAR, CUBIC, LANCZOS]
    windows = [HANN, GAUSS, SINE, RECTANGULAR]
    specs = []
    for k in range(count):
        n = lens[k % 3]
        m = int(rng.integers(1, 300))
        specs.append(_spec(n, m, dtypes[(k // 3) % 3], interps[k % 4], windows[k % 4], seed * 100 + k))
    return specs


class _Bufs:
    def __init__(self, specs, cuda, seed=0):
        import torch
        self.specs = specs
        self.ctxs = [open_context(s) for s in specs]
        self.raw = [H.random_raw(s, seed=seed + k) for k, s in enumerate(specs)]
        self.d_in = [torch.from_numpy(np.ascontiguousarray(r).view(np.uint8).reshape(-1).copy()).to(cuda)
                     for r in self.raw]
        self.d_out = [torch.full((s.num_ascans, s.signal_length // 2), np.nan, dtype=torch.float32, device=cuda)
                      for s in specs]

    def items(self):
        return [(c, i.data_ptr(), o.data_ptr(), s.num_ascans)
                for c, i, o, s in zip(self.ctxs, self.d_in, self.d_out, self.specs)]

    def single(self):
        import torch
        outs = []
        for c, i, s in zip(self.ctxs, self.d_in, self.specs):
            o = torch.empty((s.num_ascans, s.signal_length // 2), dtype=torch.float32, device=i.device)
            c.process_device(i.data_ptr(), o.data_ptr(), torch.cuda.current_stream().cuda_stream,
                             num_ascans=s.num_ascans)
            outs.append(o)
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in outs]

    def outputs(self):
        import torch
        torch.cuda.synchronize()
        return [o.cpu().numpy() for o in self.d_out]


def _stream():
    import torch
    return torch.cuda.current_stream().cuda_stream


def test_batch_bit_identical_to_single_buffer_calls(cuda):
    from octproengine_b200.batch import Batch
    bufs = _Bufs(_case(), cuda)
    ref = bufs.single()
    with Batch(bufs.items()) as b:
        b.run(_stream())
        got = bufs.outputs()
    for k, (g, r) in enumerate(zip(got, ref)):
        assert np.array_equal(g, r), f"buffer {k}: {bufs.specs[k]}"
    for c in bufs.ctxs:
        assert c.synchronize() == 0


@pytest.mark.parametrize("pairs", [1, 3, 32])
def test_every_unit_size_gives_the_same_bits(cuda, pairs):
    from octproengine_b200.batch import Batch
    bufs = _Bufs(_case(count=6, seed=2), cuda, seed=10)
    ref = bufs.single()
    with Batch(bufs.items()) as b:
        for n in (1024, 2048, 4096):
            b.set_tuning(n, pairs, 0)
        b.run(_stream())
        got = bufs.outputs()
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)


@pytest.mark.parametrize("sched", [1, 2])
def test_other_radix_schedules_match_oracle(cuda, sched):
    """Radix plans with the short pass first (4*16*16, 8*16*16) or second
    (16*4*16, 16*8*16): a different evaluation order, as accurate."""
    from octproengine_b200.batch import Batch
    specs = [_spec(n, 37, UINT16, CUBIC, HANN, 5 + n) for n in (1024, 2048)]
    bufs = _Bufs(specs, cuda, seed=20)
    ref = bufs.single()
    with Batch(bufs.items()) as b:
        b.set_tuning(1024, 2, sched)
        b.set_tuning(2048, 2, sched)
        b.run(_stream())
        got = bufs.outputs()
    for s, g, r, raw in zip(specs, got, ref, bufs.raw):
        assert not np.array_equal(g, r)  # a different evaluation order really ran
        rr, w, cs = s.curves()
        st = R.ChainSettings(n=s.signal_length, resampling=True, interpolation=CUBIC, windowing=True,
                             dispersion=True, grayscale_min=0.0, grayscale_max=90.0,
                             ascans_per_bscan=s.ascans_per_bscan)
        o64 = R.process_buffer(raw, st, R.Curves(rr, w, cs[0::2].copy(), cs[1::2].copy()), mode="f64").output
        shown = o64 * 90.0 >= 30.0
        e_new = np.abs(g - o64)[shown].max() * 90.0
        e_old = np.abs(r - o64)[shown].max() * 90.0
        assert e_new < 2e-3 and e_new < 4 * e_old + 1e-4, (e_new, e_old)


def test_graph_replay_sees_new_data(cuda):
    import torch
    from octproengine_b200.batch import Batch
    bufs = _Bufs(_case(count=5, seed=3), cuda, seed=30)
    with Batch(bufs.items()) as b:
        b.run_graph(_stream())
        first = bufs.outputs()
        assert all(np.array_equal(g, r) for g, r in zip(first, bufs.single()))
        for k, s in enumerate(bufs.specs):  # new input in the same device buffers
            new = H.random_raw(s, seed=99 + k)
            bufs.d_in[k].copy_(torch.from_numpy(np.ascontiguousarray(new).view(np.uint8).reshape(-1).copy()))
        b.run_graph(_stream())
        b.run_graph(_stream())
        second = bufs.outputs()
        ref = bufs.single()
    for g, r, f in zip(second, ref, first):
        assert np.array_equal(g, r) and not np.array_equal(g, f)


def test_autotune_picks_a_candidate_and_keeps_results(cuda):
    from octproengine_b200.batch import Batch
    specs = [_spec(n, m, UINT16, CUBIC, HANN, n + m) for n, m in ((1024, 500), (2048, 300), (4096, 120))]
    bufs = _Bufs(specs, cuda, seed=40)
    ref = bufs.single()
    with Batch(bufs.items()) as b:
        b.autotune(reps=2)
        for n in (1024, 2048, 4096):
            pp, sc, us = b.tuning(n)
            assert pp in (1, 2, 4, 8, 16, 32) and sc in (0, 1, 2) and us > 0
            if n == 4096:
                assert sc == 0
        b.run(_stream())
        got = bufs.outputs()
        scheds = {n: b.tuning(n)[1] for n in (1024, 2048, 4096)}
    for s, g, r in zip(specs, got, ref):
        if scheds[s.signal_length] == 0:
            assert np.array_equal(g, r)
        else:
            assert np.abs(g - r).max() * 90.0 < 0.05


def test_fpn_subtraction_in_a_batch(cuda):
    from octproengine_b200.batch import Batch
    specs = [_spec(2048, 64, UINT16, LINEAR, HANN, 7).with_(fpn_removal=True),
             _spec(1024, 33, UINT8, CUBIC, GAUSS, 8)]
    bufs = _Bufs(specs, cuda, seed=50)
    prof = np.random.default_rng(1).normal(0, 2000, 2048).astype(np.float32)  # 1024 complex pairs
    bufs.ctxs[0].set_fpn_profile(prof)
    ref = bufs.single()
    with Batch(bufs.items()) as b:
        b.run(_stream())
        got = bufs.outputs()
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)


def test_batch_rejects_what_it_cannot_run(cuda):
    import torch
    from octproengine_b200.batch import Batch
    d = torch.empty(1 << 20, dtype=torch.uint8, device=cuda)
    o = torch.empty(1 << 18, dtype=torch.float32, device=cuda)
    ctx512 = open_context(_spec(512, 4, UINT16, CUBIC, HANN, 1))
    with pytest.raises(capi.B200Error):
        Batch([(ctx512, d.data_ptr(), o.data_ptr(), 4)])  # length outside {1024, 2048, 4096}
    ctx = open_context(_spec(2048, 4, UINT16, CUBIC, HANN, 1))
    with pytest.raises(capi.B200Error):
        Batch([(ctx, d.data_ptr() + 8, o.data_ptr(), 4)])  # misaligned input
    ctx_req = open_context(_spec(2048, 4, UINT16, CUBIC, HANN, 1).with_(fpn_removal=True))
    ctx_req.request_fpn_determination()
    with pytest.raises(capi.B200Error):
        Batch([(ctx_req, d.data_ptr(), o.data_ptr(), 4)])  # pending FPN determination
    with Batch([(ctx, d.data_ptr(), o.data_ptr(), 4)]) as b:
        with pytest.raises(capi.B200Error):
            b.set_tuning(4096, 4, 1)  # 4096 has one schedule
        with pytest.raises(capi.B200Error):
            b.set_tuning(2048, 4, 3)  # three plans at 2048
        with pytest.raises(capi.B200Error):
            b.set_tuning(2048, 0, 0)


def test_bitshift_in_a_batch(cuda):
    from octproengine_b200.batch import Batch
    specs = [_spec(2048, 40, UINT16, CUBIC, HANN, 11).with_(bitshift=True),
             _spec(1024, 17, UINT8, LANCZOS, GAUSS, 12).with_(bitshift=True),
             _spec(1024, 9, UINT16, LINEAR, HANN, 13)]
    bufs = _Bufs(specs, cuda, seed=60)
    ref = bufs.single()
    with Batch(bufs.items()) as b:
        b.run(_stream())
        got = bufs.outputs()
    for g, r in zip(got, ref):
        assert np.array_equal(g, r)
