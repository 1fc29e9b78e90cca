"""The FPN determination entry point that allocates no device memory.

Some callers may not allocate device memory while they run: real-time
acquisition threads (cudaMalloc/cudaFree can synchronise the whole device and
stall the frame loop) and integrations that budget all device memory at
start-up. ope_b200_determine_fpn_noalloc keeps its scratch in the library's
static device array instead of a cudaMalloc'd buffer. This file is collected
last so that a run stopping at the first failure has already run every other
test; it also passes when run alone in a fresh process.
"""
import numpy as np
import pytest

import helpers as H
from octproengine_b200 import capi
from octproengine_b200.chain import ChainSpec, open_context, CUBIC, HANN

pytestmark = pytest.mark.gpu


def _spec(n=2048, ascans=256):
    return ChainSpec(signal_length=n, ascans_per_bscan=ascans, bscans_per_buffer=2, resampling=True,
                     interpolation=CUBIC, resampling_coeffs=(0.5, float(n), -100.0, 50.0), windowing=True,
                     window_type=HANN, window_center=0.5, window_fill=0.9, dispersion=True,
                     dispersion_coeffs=(0.0, 0.0, 1.0, -3.0), fpn_removal=True, fpn_bscan_count=1,
                     grayscale_min=20.0, grayscale_max=110.0)


@pytest.mark.parametrize("n,ascans", [(1024, 256), (2048, 256), (4096, 256), (2048, 64)])
def test_noalloc_fpn_matches_allocating_path_twice(cuda, n, ascans):
    """Two calls in a row through the C ABI each give the profile of the
    allocating path (request + process) within the FPN test tolerance; the
    second call proves the shared scratch is cleared between calls. N = 4096
    is the largest length the static scratch serves; 64 A-scans per
    determination (8 per FPN segment) run one CTA per segment, 256 run the
    full 8."""
    import torch
    spec = _spec(n, ascans)
    m, half = spec.num_ascans, spec.signal_length // 2
    raw = H.random_raw(spec, seed=77)
    d_in = torch.from_numpy(raw.view(np.uint8).reshape(-1).copy()).to("cuda:0")
    stream = torch.cuda.current_stream().cuda_stream
    with open_context(spec) as ctx:
        out = torch.empty((m, half), dtype=torch.float32, device="cuda:0")
        ctx.request_fpn_determination()
        ctx.process_device(d_in.data_ptr(), out.data_ptr(), stream)
        torch.cuda.synchronize()
        want = ctx.fpn_profile()
        assert want.size == 2 * half
        prof = torch.empty(2 * half, dtype=torch.float32, device="cuda:0")
        for _ in range(2):
            prof.fill_(float("nan"))
            ctx.determine_fpn_noalloc(d_in.data_ptr(), m, prof.data_ptr(), stream)
            torch.cuda.synchronize()
            assert ctx.synchronize() == 0
            got = prof.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert np.abs(got - want).max() <= 1e-5 * np.abs(want).max()


def test_noalloc_fpn_rejects_sizes_beyond_its_scratch(cuda):
    import torch
    spec = _spec(8192)
    with open_context(spec) as ctx:
        d_in = torch.zeros(spec.num_ascans * spec.signal_length, dtype=torch.int16, device="cuda:0")
        prof = torch.empty(spec.signal_length, dtype=torch.float32, device="cuda:0")
        with pytest.raises(capi.B200Error) as ei:
            ctx.determine_fpn_noalloc(d_in.data_ptr(), spec.num_ascans, prof.data_ptr())
        assert ei.value.code == capi.E_UNSUPPORTED
