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
