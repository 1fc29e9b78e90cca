"""This backend against the reference's own GPU path, per stratum.

RefCUDA = the reference CudaBackend (cuda_backend.cu + cuda_kernels.cu, cuFFT
for the DFT, built with the reference's default --use_fast_math) compiled out
of tree into oracle/_ref and driven through its own ring; float64 = the oracle
restatement in float64. The strata are those of test_parity_strata (dB
max-abs; kappa = FPN cancellation factor). The claim: this backend is no less
accurate than the reference's GPU path on bins >= 40 dB, on displayed bins with
kappa <= 10 and in the cancellation-normalised error, on every benchmark
workload.
"""
import numpy as np
import pytest

import helpers as H
from octproengine_b200 import synth
from test_parity_strata import ORDERED, _cancellation, _cases, _strata

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,spec,sp", _cases(), ids=lambda v: v if isinstance(v, str) else "")
def test_against_reference_cuda_backend(cuda, refcuda, name, spec, sp):
    raw = synth.as_numpy(synth.generate(sp), "uint16")
    gpu = H.gpu_run(spec, raw, fpn_request=spec.fpn_removal)
    res64 = H.oracle_image(spec, raw, mode="f64", determine_fpn=spec.fpn_removal, keep=True)
    p = refcuda.make_params(spec.signal_length, spec.ascans_per_bscan, spec.bscans_per_buffer, 2, resampling=True,
                            interpolation=spec.interpolation, resampling_coeffs=spec.resampling_coeffs,
                            windowing=True, window_type=spec.window_type, window_center=spec.window_center,
                            window_fill=spec.window_fill, dispersion=True, dispersion_coeffs=spec.dispersion_coeffs,
                            fpn_removal=spec.fpn_removal, fpn_bscan_count=spec.fpn_bscan_count,
                            grayscale_min=spec.grayscale_min, grayscale_max=spec.grayscale_max)
    be = refcuda.RefCudaBackend(p)
    try:
        ref = be.process(raw)
    finally:
        be.close()
    g, r, t = (H.to_db(x, spec) for x in (gpu, ref, res64.output))
    kappa = _cancellation(spec, res64.ifft, t)
    gmin = spec.grayscale_min
    rows = {"GPU vs FP64": _strata(np.abs(g - t), t, kappa, gmin),
            "RefCUDA vs FP64": _strata(np.abs(r - t), t, kappa, gmin),
            "GPU vs RefCUDA": _strata(np.abs(g - r), t, kappa, gmin)}
    print(f"\n{name} ({spec.num_ascans} A-scans of {spec.signal_length}), dB max-abs per stratum:")
    for k, v in rows.items():
        print(f"  {k:15s} " + "  ".join(f"{s} {x:.2e}" for s, x in v.items()))
    for s in ORDERED:
        assert rows["GPU vs FP64"][s] <= 1.05 * rows["RefCUDA vs FP64"][s] + 1e-6, (s, rows)
