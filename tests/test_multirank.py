"""Multi-rank bookkeeping on CPU: world size 2 over gloo (127.0.0.1).

The chain needs no collective (A-scans are independent); what the N-GPU run
shares between ranks -- the B-scan partition and the max-over-ranks timing
that bench.py reports as whole-job throughput -- runs here on two gloo ranks.
"""
import os
import socket

import pytest

from octproengine_b200.multirank import bscan_range, weak_scaling_rate, rank_setup


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from octproengine_b200.multirank import max_over_ranks, bscan_range, weak_scaling_rate, rank_setup
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        w, r, lr = rank_setup()
        first, count = bscan_range(64, w, r)
        ms = 10.0 + 5.0 * r  # rank 1 is slower
        ms_max = max_over_ranks(ms)
        rate = weak_scaling_rate(count * 1024, ms_max / 1e3, w)
        q.put((r, w, lr, first, count, ms_max, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_partition_and_max_time():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    assert [r[0] for r in res] == [0, 1] and all(r[1] == 2 for r in res)
    assert res[0][3:5] == (0, 32) and res[1][3:5] == (32, 32)
    assert res[0][5] == res[1][5] == 15.0  # both ranks report the slowest rank's time
    assert res[0][6] == res[1][6] == pytest.approx(2 * 32 * 1024 / 0.015)


@pytest.mark.parametrize("total,world", [(64, 1), (64, 3), (7, 4), (0, 2), (5, 8)])
def test_bscan_ranges_cover_the_volume_once(total, world):
    seen = []
    for r in range(world):
        first, count = bscan_range(total, world, r)
        seen.extend(range(first, first + count))
    assert seen == list(range(total))


def test_rank_setup_reads_torchrun_environment():
    assert rank_setup({"WORLD_SIZE": "8", "RANK": "5", "LOCAL_RANK": "5"}) == (8, 5, 5)
    assert rank_setup({}) == (1, 0, 0)
    with pytest.raises(ValueError):
        bscan_range(10, 2, 2)
    with pytest.raises(ValueError):
        weak_scaling_rate(1.0, 0.0, 1)


# ---------------------------------------------- data-parallel dispersion fit


def _af_case():
    import numpy as np
    from octproengine_b200 import synth
    from oracle import restate as R
    n = 2048
    ctrue = synth.linearising_coeffs(n)
    raw = synth.as_numpy(synth.generate(synth.SynthParams(n=n, ascans=48, seed=31, d2=14.0, d3=-6.0,
                                                          resampling_truth=ctrue)), "uint16")
    return raw, R.window_curve(n, R.HANN, 0.5, 0.95), np.asarray(ctrue)


def _oracle_fns(raw, win):
    """This rank's forward and adjoint, in float64 (the oracle chain, Lanczos-8)."""
    import numpy as np
    import torch
    from oracle import autofocus64 as O

    def fwd(p8):
        I, _ = O.intensity(raw, p8, win, O.LANCZOS)
        return float(O.entropy_of(I)), float(I.sum())

    def bwd(p8, H, S):
        I, p = O.intensity(raw, p8, win, O.LANCZOS, requires_grad=True)
        G = torch.where(I > 0, -(torch.log(I.detach() / S) + H) / S, torch.zeros_like(I))
        (g,) = torch.autograd.grad((G * I).sum(), p)
        return g.numpy()
    return fwd, bwd


class _WholeVolume:
    """The same objective on all A-scans in one process (no collective)."""

    def __init__(self, raw, win, kmap):
        import numpy as np
        self.raw, self.win, self.kmap, self.count = raw, win, np.asarray(kmap, np.float32), 0

    def __call__(self, theta):
        import numpy as np
        from octproengine_b200.autofocus import CENTRED_TO_POLY, dispersion_poly
        from oracle import autofocus64 as O
        p8 = np.zeros(8)
        p8[:4] = dispersion_poly(theta[0], theta[1]).astype(np.float32)
        p8[4:] = self.kmap
        H, g = O.entropy_and_grad(self.raw, p8, self.win, O.LANCZOS)
        self.count += 1
        return H, CENTRED_TO_POLY.T @ g[:4]


def _fit_worker(rank, world, port, q):
    import numpy as np
    import torch.distributed as dist
    from datetime import timedelta
    from octproengine_b200.autofocus import DistributedFitEvaluator, fit_dispersion
    from octproengine_b200.multirank import bscan_range
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=120))
    try:
        raw, win, kmap = _af_case()
        first, count = bscan_range(raw.shape[0], world, rank)  # A-scans split like B-scans
        fwd, bwd = _oracle_fns(raw[first:first + count], win)
        ev = DistributedFitEvaluator(kmap, local_forward=fwd, local_backward=bwd)
        H, g = ev(np.array([9.0, -2.0]))
        fit = fit_dispersion(None, None, kmap, evaluator=ev, max_iter=4)
        q.put((rank, H, tuple(g), fit.d2, fit.d3, fit.evaluations))
    finally:
        dist.destroy_process_group()


def test_distributed_fit_equals_the_whole_volume_fit():
    import multiprocessing as mp
    import numpy as np
    from octproengine_b200.autofocus import fit_dispersion
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_fit_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    res = sorted(q.get(timeout=5) for _ in range(2))
    raw, win, kmap = _af_case()
    whole = _WholeVolume(raw, win, kmap)
    H, g = whole(np.array([9.0, -2.0]))
    fit = fit_dispersion(None, None, kmap, evaluator=whole, max_iter=4)
    for r in res:
        assert r[1] == pytest.approx(H, rel=1e-12)
        assert np.allclose(r[2], g, rtol=1e-8, atol=1e-12 * np.abs(g).max())
        assert (r[3], r[4], r[5]) == pytest.approx((fit.d2, fit.d3, fit.evaluations), rel=1e-6)
    assert res[0][3:] == res[1][3:]  # both ranks took the same steps


def test_entropy_parts_of_a_split_volume_sum_to_the_whole():
    import numpy as np
    from octproengine_b200.autofocus import entropy_from_parts, entropy_parts
    rng = np.random.default_rng(3)
    I = rng.gamma(0.3, 5.0, size=(40, 512))

    def h_s(x):
        S = x.sum()
        p = x / S
        return float(-(p * np.log(p)).sum()), float(S)
    whole = h_s(I)
    parts = sum(entropy_parts(*h_s(I[a:b])) for a, b in ((0, 13), (13, 40))) + entropy_parts(0.0, 0.0)
    H, S = entropy_from_parts(parts)
    assert H == pytest.approx(whole[0], rel=1e-13) and S == pytest.approx(whole[1], rel=1e-14)
