"""Low-level per-operation API (ope_b200_op_*), each a GPU kernel on host arrays.

Where the reference CPU backend implements the operation, the GPU result is
compared with the reference's own implementation (oracle/_ref, the reference
CpuBackend compiled out of tree): bit for bit for convertInput,
kLinearization (linear, cubic) and windowing, getMinimumVarianceMean; within a
few ulp for Lanczos (device sinf vs the C library's) and ifft (the reference's
FFT is the float32 shim, ours is evaluated in double). The operations the
reference stubs are checked against the oracle restatement.
"""
import ctypes

import numpy as np
import pytest

from octproengine_b200 import capi
from oracle import restate as R

pytestmark = pytest.mark.gpu

N = 2048


def fp(a):
    return capi.fptr(np.ascontiguousarray(a, np.float32))


def _ok(rc):
    assert rc == capi.OK


@pytest.mark.parametrize("dtype,bits", [(np.uint8, 8), (np.uint16, 16), (np.uint32, 32)])
def test_convert_input_matches_reference(cuda, reflib, dtype, bits):
    rng = np.random.default_rng(bits)
    hi = np.iinfo(dtype).max
    raw = rng.integers(0, hi, 4096, dtype=np.uint64).astype(dtype)
    raw[:3] = [0, hi, hi - 1]
    out = np.empty(raw.size, np.float32)
    _ok(capi.lib().ope_b200_op_convert_input(raw.ctypes.data_as(ctypes.c_void_p), bits, raw.size, capi.fptr(out)))
    ref = np.empty(raw.size, np.float32)
    dt = {8: R.UINT8, 16: R.UINT16, 32: R.UINT32}[bits]
    reflib.lib().ope_ref_convert_input(raw.ctypes.data_as(ctypes.c_void_p), dt, raw.size, capi.fptr(ref))
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("method", [R.LINEAR, R.CUBIC, R.LANCZOS])
def test_klinearization_matches_reference(cuda, reflib, method):
    rng = np.random.default_rng(method)
    x = (32768 + rng.normal(0, 3000, N)).astype(np.float32)
    curve = R.resampling_curve(N, (0.5, N - 1.0, -80.0, 40.0))
    out = np.empty(N, np.float32)
    _ok(capi.lib().ope_b200_op_klinearization(fp(x), fp(curve), method, N, N, capi.fptr(out)))
    ref = np.empty(N, np.float32)
    reflib.lib().ope_ref_klinearization(fp(x), fp(curve), method, N, capi.fptr(ref))
    if method == R.LANCZOS:
        assert np.allclose(out, ref, rtol=2e-6, atol=2e-2)  # sinf of the device vs the C library
    else:
        assert np.array_equal(out, ref)


def test_window_and_dispersion_ops(cuda, reflib):
    rng = np.random.default_rng(7)
    x = rng.normal(0, 1000, N).astype(np.float32)
    w = R.window_curve(N, R.HANN, 0.5, 0.9)
    c, s = R.phase_to_cos_sin(R.dispersion_phase(N, (0.0, 1.0, 20.0, -10.0)))
    cs = np.empty(2 * N, np.float32)
    cs[0::2], cs[1::2] = c, s
    out = np.empty(N, np.float32)
    _ok(capi.lib().ope_b200_op_window_dispersion(fp(x), fp(w), None, 1, N, N, capi.fptr(out)))
    ref = np.empty(N, np.float32)
    reflib.lib().ope_ref_windowing(fp(x), fp(w), N, capi.fptr(ref))
    assert np.array_equal(out, ref)
    _ok(capi.lib().ope_b200_op_window_dispersion(fp(x), None, fp(cs), 2, N, N, capi.fptr(out)))
    assert np.array_equal(out, (x * c).astype(np.float32))  # real part of (x + 0i)(cos + i sin)
    _ok(capi.lib().ope_b200_op_window_dispersion(fp(x), fp(w), fp(cs), 3, N, 100, capi.fptr(out)))
    assert np.array_equal(out[:100], ((x * c).astype(np.float32) * w)[:100].astype(np.float32))


@pytest.mark.parametrize("n", [1000, 512, 1024, 2048, 8192])
def test_dft_magnitudes(cuda, reflib, n):
    """Power-of-two lengths run the chain's float32 FFT: within float32 FFT
    rounding (relative to the line's largest magnitude) of the exact DFT and of
    the reference's ifft op; other lengths a direct DFT in double."""
    rng = np.random.default_rng(8)
    x = rng.normal(0, 100, n).astype(np.float32)
    inv = np.empty(n, np.float32)
    fwd = np.empty(n, np.float32)
    _ok(capi.lib().ope_b200_op_dft_magnitude(fp(x), n, 1, capi.fptr(inv)))
    _ok(capi.lib().ope_b200_op_dft_magnitude(fp(x), n, 0, capi.fptr(fwd)))
    truth = np.abs(np.fft.ifft(x.astype(np.float64)) * n)
    tol = 2e-6 * truth.max() if (n & (n - 1)) == 0 else 1e-6 * truth.max()
    assert np.abs(inv - truth).max() <= tol
    assert np.abs(fwd - np.abs(np.fft.fft(x.astype(np.float64)))).max() <= tol
    reflib.set_fft_precision("f64")
    ref = np.empty(n, np.float32)
    reflib.lib().ope_ref_ifft_magnitude(fp(x), n, capi.fptr(ref))
    assert np.abs(inv - ref).max() <= tol


def test_min_variance_mean_matches_reference(cuda, reflib):
    rng = np.random.default_rng(9)
    width, height = 512, 96
    z = rng.normal(0, 50, (height, width, 2)).astype(np.float32)
    z[40:52] *= 0.1  # a quiet segment
    out = np.empty(2 * width, np.float32)
    _ok(capi.lib().ope_b200_op_min_variance_mean(fp(z), width, height, 8, capi.fptr(out)))
    ref = np.empty(2 * width, np.float32)
    reflib.lib().ope_ref_min_var_mean(fp(z), width, height, 8, capi.fptr(ref))
    assert np.array_equal(out, ref)


def test_fpn_removal_op_follows_the_reference_rule(cuda):
    rng = np.random.default_rng(10)
    w, lines = 256, 6
    z = rng.normal(0, 10, (lines, w, 2)).astype(np.float32)
    mean = rng.normal(0, 3, (w, 2)).astype(np.float32)
    out = np.empty(lines * w, np.float32)
    _ok(capi.lib().ope_b200_op_fpn_removal(fp(z), fp(mean), w, lines, capi.fptr(out)))
    flat = z.reshape(-1, 2).copy()
    use = min(lines * w // 2, w)  # meanALineSubtraction on the flattened buffer (cpu_kernels.tpp:460-479)
    flat[:use] -= mean[:use]
    want = np.sqrt((flat[:, 0] * flat[:, 0] + flat[:, 1] * flat[:, 1]).astype(np.float32)).astype(np.float32)
    assert np.array_equal(out, want)


def test_rolling_dc_flip_background_ops(cuda):
    rng = np.random.default_rng(11)
    w, lines = 512, 8
    x = (30000 + rng.normal(0, 2000, (lines, w))).astype(np.float32)
    out = np.empty(lines * w, np.float32)
    _ok(capi.lib().ope_b200_op_rolling_dc_removal(fp(x), 64, w, lines, capi.fptr(out)))
    want = np.stack([R.dc_removal(x[l:l + 1], 64)[0] for l in range(lines)])
    assert np.allclose(out.reshape(lines, w), want, atol=1e-2)
    img = rng.normal(0, 1, (3 * 4, 100)).astype(np.float32)
    flip = np.empty(img.size, np.float32)
    _ok(capi.lib().ope_b200_op_bscan_flip(fp(img), 100, 4, 3, capi.fptr(flip)))
    want = img.reshape(3, 4, 100).copy()
    want[0] = want[0][::-1]  # B-scan 0 has a successor; B-scan 2 is the trailing one
    assert np.array_equal(flip.reshape(3, 4, 100), want)
    bg = rng.normal(0, 1, 100).astype(np.float32)
    sub = np.empty(img.size, np.float32)
    _ok(capi.lib().ope_b200_op_background_subtraction(fp(img), fp(bg), 0.5, 0.25, 100, img.size, capi.fptr(sub)))
    assert np.array_equal(sub.reshape(img.shape), img - (np.float32(0.5) * bg + np.float32(0.25)))


def test_sinusoidal_and_truncate_ops(cuda):
    rng = np.random.default_rng(12)
    img = rng.uniform(0, 1, (2 * 64, 128)).astype(np.float32)
    out = np.empty(img.size, np.float32)
    _ok(capi.lib().ope_b200_op_sinusoidal_correction(fp(img), None, 128, 64, 2, capi.fptr(out)))
    want = R.sinusoidal_correction(img, 64)
    assert np.allclose(out.reshape(img.shape), want, atol=1e-5)
    curve = R.sinusoidal_curve(64)
    _ok(capi.lib().ope_b200_op_sinusoidal_correction(fp(img), fp(curve), 128, 64, 2, capi.fptr(out)))
    assert np.array_equal(out.reshape(img.shape), want)  # same curve: every bit
    z = rng.normal(0, 300, (3, 256)).astype(np.float32)  # 3 lines of 128 complex values
    X = z[:, 0::2] + 1j * z[:, 1::2]
    t = np.empty(3 * 64, np.float32)
    _ok(capi.lib().ope_b200_op_truncate(fp(z), 1, 80.0, 10.0, 0.0, 1.0, 128, 3, capi.fptr(t)))
    want = R.log_scale(X.astype(np.complex64), 1.0, 10.0, 80.0, 0.0, False)  # 128-point lines, bins [0, 64)
    assert np.allclose(t.reshape(3, 64), want, atol=1e-5)


def test_ops_reject_bad_arguments(cuda):
    x = np.zeros(16, np.float32)
    assert capi.lib().ope_b200_op_klinearization(fp(x), fp(x), 3, 16, 16, capi.fptr(x)) == capi.E_INVALID
    assert capi.lib().ope_b200_op_window_dispersion(fp(x), None, None, 1, 16, 16, capi.fptr(x)) == capi.E_INVALID
    assert capi.lib().ope_b200_op_min_variance_mean(fp(x), 4, 2, 8, capi.fptr(x)) == capi.E_INVALID
