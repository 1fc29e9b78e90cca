"""Many buffers of uneven geometry in one persistent launch (C ABI ``ope_b200_batch_*``).

Each buffer is described by a configured :class:`capi.Context` (its
ProcessorConfiguration and curves) plus device input/output pointers and an
A-scan count; :class:`Batch` runs all of them in one launch of the batched
kernel (octproengine_b200/csrc/batch.cu), optionally replayed from a CUDA
graph, with a per-length autotuner for the A-scans each CTA takes per grab and
the FFT radix schedule. No counterpart in the reference, which processes one
IOBuffer of one geometry per call.
"""
from __future__ import annotations

import ctypes
from typing import Sequence, Tuple

from . import capi


class BatchItem(ctypes.Structure):
    """Mirror of ``ope_b200_batch_item``."""
    _fields_ = [("ctx", ctypes.c_void_p), ("d_in", ctypes.c_void_p), ("d_out", ctypes.c_void_p),
                ("num_ascans", ctypes.c_int64)]


class Batch:
    def __init__(self, items: Sequence[Tuple[capi.Context, int, int, int]]):
        """items: (context, device input pointer, device output pointer, A-scan count) per buffer."""
        self._ctxs = [it[0] for it in items]  # keep the contexts alive
        arr = (BatchItem * len(items))()
        for k, (ctx, d_in, d_out, m) in enumerate(items):
            arr[k] = BatchItem(ctx.h, int(d_in), int(d_out), int(m))
        h = ctypes.c_void_p()
        rc = capi.lib().ope_b200_batch_create(ctypes.cast(arr, ctypes.c_void_p), len(items), ctypes.byref(h))
        if rc != capi.OK:
            raise capi.B200Error(rc, "batch creation failed (unsupported length, type or FPN mode, or bad pointer)")
        self.h = h

    def close(self) -> None:
        if getattr(self, "h", None):
            capi.lib().ope_b200_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, rc: int) -> None:
        if rc != capi.OK:
            raise capi.B200Error(rc, capi.lib().ope_b200_batch_last_error(self.h).decode())

    def run(self, stream: int = 0) -> None:
        self._check(capi.lib().ope_b200_batch_run(self.h, stream))

    def run_graph(self, stream: int = 0) -> None:
        self._check(capi.lib().ope_b200_batch_run_graph(self.h, stream))

    def set_tuning(self, n: int, pairs_per_team: int, radix_schedule: int = 0) -> None:
        self._check(capi.lib().ope_b200_batch_set_tuning(self.h, n, pairs_per_team, radix_schedule))

    def tuning(self, n: int):
        pp, sc, us = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_float()
        self._check(capi.lib().ope_b200_batch_get_tuning(self.h, n, ctypes.byref(pp), ctypes.byref(sc),
                                                         ctypes.byref(us)))
        return pp.value, sc.value, us.value

    def autotune(self, reps: int = 3) -> None:
        self._check(capi.lib().ope_b200_batch_autotune(self.h, reps))


def radix_plan(n: int, radix_schedule: int) -> str:
    """The FFT radix plan a schedule runs at length n, e.g. "16x8x16"."""
    npass = (int(n).bit_length() - 1 + 3) // 4
    short = n // 16 ** (npass - 1)
    pos = npass - 1 if radix_schedule == 0 else radix_schedule - 1
    return "x".join(str(short if p == pos else 16) for p in range(npass))
