"""Differentiable chain (autofocus): forward, hand-written adjoint, fit.

CPU tests check the float64 oracle itself (its autograd against central
finite differences) and the host-side parameter maps. GPU tests call the C ABI
(ope_b200_af_forward / ope_b200_af_backward) through
octproengine_b200.autofocus and compare with the float64 oracle:
forward image and entropy, adjoint gradients for all 8 parameters (entropy
objective and arbitrary image gradients, intensity and dB outputs), central
finite differences of the GPU forward, and the BFGS fit against hidden
dispersion coefficients.
"""
import numpy as np
import pytest
import torch

from octproengine_b200 import synth
from oracle import autofocus64 as O
from oracle import restate as R

N = 2048


def make_case(m=64, seed=5, d2=12.0, d3=-7.0, kpert=1.1, dtype="uint16"):
    kc = list(synth.K_COEFFS)
    kc[3] *= kpert
    ctrue = synth.linearising_coeffs(N, tuple(kc))
    p = synth.SynthParams(n=N, ascans=m, seed=seed, d2=d2, d3=d3, resampling_truth=ctrue, dtype=dtype)
    raw_t = synth.generate(p)
    raw = synth.as_numpy(raw_t, dtype)
    window = R.window_curve(N, R.HANN, 0.5, 0.95)
    return raw_t, raw, window, ctrue


def params_of(d2, d3, kmap):
    from octproengine_b200.autofocus import dispersion_poly
    return np.concatenate([dispersion_poly(d2, d3), np.asarray(kmap, np.float64)]).astype(np.float32)


# ------------------------------------------------------------------ CPU --

def test_centred_map_matches_generator_convention():
    from octproengine_b200.autofocus import dispersion_poly
    for d2, d3 in [(1.0, 0.0), (0.0, 1.0), (-13.5, 7.25)]:
        assert np.allclose(dispersion_poly(d2, d3), synth.compensating_coeffs(d2, d3))


@pytest.mark.parametrize("interp", [O.LINEAR, O.CUBIC, O.LANCZOS])
def test_oracle_gradient_matches_finite_differences(interp):
    _, raw, window, ctrue = make_case(m=8)
    p0 = params_of(9.0, -4.0, ctrue).astype(np.float64)
    H0, g = O.entropy_and_grad(raw, p0, window, interp, f32_curves=False)
    # linear interpolation is only piecewise differentiable in the positions:
    # a small step keeps the difference quotient off the kinks at integer r
    h = 1e-6 if interp == O.LINEAR else 1e-3
    for k in range(8):
        e = np.zeros(8)
        e[k] = h
        fd = (O.entropy_and_grad(raw, p0 + e, window, interp, f32_curves=False)[0] -
              O.entropy_and_grad(raw, p0 - e, window, interp, f32_curves=False)[0]) / (2 * h)
        assert abs(fd - g[k]) <= 2e-3 * np.abs(g).max() + 1e-3 * abs(g[k]), (k, fd, g[k])


def test_polynomial_wavenumber_map_inverts_resampling():
    c = synth.linearising_coeffs(N)
    k = synth.k_map_from_resampling(N, c)
    j = np.arange(N) / (N - 1.0)
    r = sum(c[m] * j ** m for m in range(4))
    inside = (r >= 0) & (r <= N - 1)  # wavenumbers sampled inside the raw record
    assert inside.sum() > N - 8
    err = np.interp(r, np.arange(N), k) - np.arange(N)
    assert np.max(np.abs(err[inside])) < 1e-3


# ------------------------------------------------------------------ GPU --

def _af(cuda, interp, window, dtype="uint16"):
    from octproengine_b200.autofocus import Autofocus
    return Autofocus(N, dtype, interp, window=window)


@pytest.mark.gpu
@pytest.mark.parametrize("interp", [O.LINEAR, O.CUBIC, O.LANCZOS])
def test_forward_matches_fp64(cuda, interp):
    from octproengine_b200.autofocus import OUT_INTENSITY, OUT_DB
    raw_t, raw, window, ctrue = make_case(m=64)
    p = params_of(10.0, -5.0, ctrue)
    af = _af(cuda, interp, window)
    d_raw = raw_t.to(cuda)
    d_p = torch.from_numpy(p).to(cuda)
    I = torch.empty((64, N // 2), dtype=torch.float32, device=cuda)
    dB = torch.empty_like(I)
    hs = torch.empty(2, dtype=torch.float64, device=cuda)
    af.forward(d_raw, d_p, OUT_INTENSITY, out=I, hs=hs)
    af.forward(d_raw, d_p, OUT_DB, out=dB)
    torch.cuda.synchronize()
    I64, _ = O.intensity(raw, p.astype(np.float64), window, interp)
    I64 = I64.numpy()
    shown = I64 > I64.max() * 1e-5  # within 50 dB of the strongest bin
    err_db = np.abs(10 * np.log10(I.cpu().numpy()[shown].astype(np.float64) / I64[shown]))
    assert err_db.max() < 0.02, err_db.max()
    ref_db = 10 * np.log10(I64 / (N // 2))
    assert np.abs(dB.cpu().numpy()[shown] - ref_db[shown]).max() < 0.02
    H64 = float(O.entropy_of(torch.as_tensor(I64)))
    assert abs(hs[0].item() - H64) < 1e-6 * H64
    assert abs(hs[1].item() - I64.sum()) < 1e-5 * I64.sum()


@pytest.mark.gpu
@pytest.mark.parametrize("interp", [O.LINEAR, O.CUBIC, O.LANCZOS])
def test_entropy_gradient_matches_fp64(cuda, interp):
    from octproengine_b200.autofocus import ChainEntropy
    raw_t, raw, window, ctrue = make_case(m=64, seed=7)
    p = params_of(4.0, 3.0, np.asarray(ctrue) + np.array([0.0, 0.0, 1.5, -1.0]))
    af = _af(cuda, interp, window)
    d_p = torch.from_numpy(p).to(cuda).requires_grad_(True)
    H = ChainEntropy.apply(raw_t.to(cuda), d_p, af)
    H.backward()
    g = d_p.grad.cpu().numpy().astype(np.float64)
    H64, g64 = O.entropy_and_grad(raw, p.astype(np.float64), window, interp)
    assert abs(H.item() - H64) < 1e-6 * H64
    scale = np.abs(g64).max()
    assert np.all(np.abs(g - g64) <= 1e-2 * scale + 1e-2 * np.abs(g64)), (g, g64)


@pytest.mark.gpu
@pytest.mark.parametrize("db", [False, True])
def test_image_gradient_matches_fp64(cuda, db):
    from octproengine_b200.autofocus import ChainImage, OUT_DB, OUT_INTENSITY
    raw_t, raw, window, ctrue = make_case(m=32, seed=9)
    p = params_of(-6.0, 2.0, ctrue)
    af = _af(cuda, O.LANCZOS, window)
    rng = np.random.default_rng(3)
    G = rng.standard_normal((32, N // 2)).astype(np.float32)
    if not db:
        G *= 1e-12  # intensities are ~1e12: keep the objective O(1)
    d_p = torch.from_numpy(p).to(cuda).requires_grad_(True)
    img = ChainImage.apply(raw_t.to(cuda), d_p, af, OUT_DB if db else OUT_INTENSITY)
    (img * torch.from_numpy(G).to(cuda)).sum().backward()
    g = d_p.grad.cpu().numpy().astype(np.float64)
    g64 = O.image_grad(raw, p.astype(np.float64), window, O.LANCZOS, G.astype(np.float64), db=db)
    scale = np.abs(g64).max()
    assert np.all(np.abs(g - g64) <= 2e-2 * scale + 2e-2 * np.abs(g64)), (g, g64)


@pytest.mark.gpu
def test_entropy_gradient_matches_gpu_finite_differences(cuda):
    raw_t, raw, window, ctrue = make_case(m=256, seed=11)
    p = params_of(8.0, -6.0, np.asarray(ctrue) + np.array([0.0, 0.0, 2.0, -2.0]))
    af = _af(cuda, O.LANCZOS, window)
    d_raw = raw_t.to(cuda)
    hs = torch.empty(2, dtype=torch.float64, device=cuda)
    grad = torch.empty(8, dtype=torch.float32, device=cuda)
    d_p = torch.from_numpy(p).to(cuda)
    af.forward(d_raw, d_p, hs=hs)
    af.backward(d_raw, d_p, grad, hs=hs)
    g = grad.cpu().numpy().astype(np.float64)
    h = 1e-3
    fd = np.zeros(8)
    for k in range(8):
        for sgn in (1, -1):
            q = p.astype(np.float64).copy()
            q[k] += sgn * h
            af.forward(d_raw, torch.from_numpy(q.astype(np.float32)).to(cuda), hs=hs)
            fd[k] += sgn * hs[0].item() / (2 * h)
    # the float32 parameter vector rounds p +- h; use the steps actually taken
    steps = np.array([(np.float32(v + h) - np.float32(v - h)) for v in p.astype(np.float64)], np.float64)
    fd = fd * (2 * h) / steps
    # c0 and c1 shift and stretch the k axis, to which the image entropy is
    # nearly invariant: their gradients are small residuals of large per-sample
    # terms, while the float32 resampling positions (ulp 1.2e-4 near r = 2000,
    # as the reference evaluates them) turn a 1e-3 step into a jittered one.
    # Their adjoint is checked against the float64 gradient instead.
    checked = np.array([1, 1, 1, 1, 0, 0, 1, 1], bool)
    big = checked & (np.abs(g) > 0.05 * np.abs(g).max())
    assert big.sum() >= 4
    assert np.all(np.abs(fd[big] - g[big]) <= 0.05 * np.abs(g[big])), (fd, g)


@pytest.mark.gpu
def test_fit_recovers_hidden_dispersion(cuda):
    from octproengine_b200.autofocus import fit_dispersion
    rng = np.random.default_rng(2024)
    d2, d3 = rng.uniform(-40, 40), rng.uniform(-20, 20)
    raw_t, raw, window, ctrue = make_case(m=256, seed=13, d2=d2, d3=d3)
    af = _af(cuda, O.LANCZOS, window)
    res = fit_dispersion(af, raw_t.to(cuda), ctrue)
    err = max(abs(res.d2 - d2) / max(abs(d2), 1.0), abs(res.d3 - d3) / max(abs(d3), 1.0))
    assert err < 0.01, (res, d2, d3)


def test_kmap_family_interpolates_the_linearising_coefficients():
    fam = synth.KmapFamily(N)
    for sc in (0.81, 1.0, 1.137):
        want = np.array(synth.linearising_coeffs(N, fam.k_coeffs(sc)))
        assert np.allclose(fam(sc), want, rtol=0, atol=1e-6 * np.abs(want).max())


def test_kmap_is_identifiable_by_entropy_in_float64():
    """The objective, not the arithmetic: in float64, BFGS on (d2, d3, s) from
    d = 0 and the nominal k-map (s = 1) ends at the hidden (d2, d3, s) of a
    five-reflector scene -- a k-map error moves each reflector's phase in
    proportion to its depth, dispersion does not."""
    from scipy.optimize import minimize
    from octproengine_b200.autofocus import dispersion_poly, CENTRED_TO_POLY
    fam = synth.KmapFamily(N)
    d2, d3, st = -19.07, -8.06, 1.1257
    ctrue = synth.linearising_coeffs(N, fam.k_coeffs(st))
    raw = synth.as_numpy(synth.generate(synth.SynthParams(n=N, ascans=64, seed=72, d2=d2, d3=d3,
                                                          resampling_truth=ctrue)), "uint16")
    window = R.window_curve(N, R.HANN, 0.5, 0.95)

    def fg(y):  # y = (d2, d3, 100 (s - 1))
        s = 1.0 + 0.01 * y[2]
        J = (fam(s + 1e-4) - fam(s - 1e-4)) / 2e-4
        H, g = O.entropy_and_grad(raw, np.concatenate([dispersion_poly(y[0], y[1]), fam(s)]), window, O.LANCZOS,
                                  f32_curves=False)
        return H, np.concatenate([CENTRED_TO_POLY.T @ g[:4], [0.01 * float(g[4:] @ J)]])

    r = minimize(fg, np.zeros(3), jac=True, method="BFGS", options={"gtol": 1e-9, "maxiter": 200})
    s = 1.0 + 0.01 * r.x[2]
    assert abs(s - st) / st < 0.005 and abs(r.x[0] - d2) / abs(d2) < 0.02 and abs(r.x[1] - d3) / abs(d3) < 0.02, r.x


def test_some_scenes_have_entropy_minima_away_from_the_truth():
    """Float64 evidence for the joint fit's failures: on the scene of benchmark
    seed 5 (hidden d2 24.40, d3 12.32 rad, k-map cubic scale 1.0061) a point
    far from the truth -- where BFGS from the nominal k-map ends, in float64
    as on the GPU -- has a LOWER entropy than the truth itself, so no
    optimiser of this objective can recover that scene."""
    from octproengine_b200.autofocus import dispersion_poly
    fam = synth.KmapFamily(N)
    rng = np.random.default_rng(5)
    d2, d3 = float(rng.uniform(-40, 40)), float(rng.uniform(-20, 20))
    st = 1.0 + float(rng.uniform(-0.2, 0.2))
    ctrue = synth.linearising_coeffs(N, fam.k_coeffs(st))
    raw = synth.as_numpy(synth.generate(synth.SynthParams(n=N, ascans=128, seed=75, d2=d2, d3=d3,
                                                          resampling_truth=ctrue)), "uint16")
    window = R.window_curve(N, R.HANN, 0.5, 0.95)

    def H(a, b, s):
        I, _ = O.intensity(raw, np.concatenate([dispersion_poly(a, b), fam(s)]), window, O.LANCZOS,
                           f32_curves=False)
        return float(O.entropy_of(I))

    assert H(-0.51, -5.21, 0.9327) < H(d2, d3, st)


@pytest.mark.gpu
def test_kmap_fit_gradient_matches_fp64(cuda):
    """dH/d(d2, d3, s) of KmapFitEvaluator (full adjoint on the GPU, chain rule
    through the k-map family on the host) against float64 autograd."""
    from octproengine_b200.autofocus import KmapFitEvaluator, dispersion_poly, CENTRED_TO_POLY
    fam = synth.KmapFamily(N)
    raw_t, raw, window, _ = make_case(m=128, seed=31, d2=14.0, d3=-6.0, kpert=0.9)
    af = _af(cuda, O.LANCZOS, window)
    ev = KmapFitEvaluator(af, raw_t.to(cuda), fam, [1.0])
    theta = np.array([10.0, -4.0, 0.95])
    H, g = ev(theta)
    p64 = np.concatenate([dispersion_poly(theta[0], theta[1]), fam(theta[2])])
    H64, g64 = O.entropy_and_grad(raw, p64, window, O.LANCZOS)
    J = (fam(theta[2] + 1e-4) - fam(theta[2] - 1e-4)) / 2e-4
    want = np.concatenate([CENTRED_TO_POLY.T @ g64[:4], [float(g64[4:] @ J)]])
    assert abs(H - H64) <= 1e-5 * abs(H64)
    assert np.all(np.abs(g - want) <= 0.01 * np.abs(want) + 1e-4 * np.abs(want).max()), (g, want)


@pytest.mark.gpu
def test_joint_fit_recovers_dispersion_and_kmap_from_the_nominal_kmap(cuda):
    """fit_dispersion_kmap from d = 0 and the nominal k-map recovers the hidden
    dispersion and the k-map's cubic coefficient (perturbed by 12.6 %) to 1 %."""
    from octproengine_b200.autofocus import fit_dispersion_kmap
    fam = synth.KmapFamily(N)
    d2, d3, st = -19.07, -8.06, 1.1257
    ctrue = synth.linearising_coeffs(N, fam.k_coeffs(st))
    p = synth.SynthParams(n=N, ascans=512, seed=72, d2=d2, d3=d3, resampling_truth=ctrue)
    raw_t = synth.generate(p)
    window = R.window_curve(N, R.HANN, 0.5, 0.95)
    af = _af(cuda, O.LANCZOS, window)
    res = fit_dispersion_kmap(af, raw_t.to(cuda), fam, [1.0])
    s = float(res.kappa[0])
    errs = (abs(res.d2 - d2) / abs(d2), abs(res.d3 - d3) / abs(d3), abs(s - st) / st)
    assert max(errs) < 0.01, (res, errs)
    assert np.allclose(res.kmap, fam(s))


@pytest.mark.gpu
def test_bitshift_applies_to_forward_and_adjoint(cuda):
    """With the bitshift flag the fit works on the samples >> 4, as the chain
    does (DataParameters::bitshift): entropy and all 8 gradient entries equal
    those of an unshifted handle given the data shifted on the host."""
    from octproengine_b200.autofocus import Autofocus
    raw_t, raw, window, ctrue = make_case(m=64, seed=41)
    shifted = torch.from_numpy((raw >> 4).astype(np.uint16).view(np.int16).copy())
    p = torch.from_numpy(params_of(8.0, -3.0, ctrue)).to(cuda)
    res = []
    for data, flag in ((raw_t, True), (shifted, False)):
        af = Autofocus(N, "uint16", O.LANCZOS, window=window, bitshift=flag)
        d = data.to(cuda).contiguous()
        hs = torch.empty(2, dtype=torch.float64, device=cuda)
        g = torch.empty(8, dtype=torch.float32, device=cuda)
        af.forward(d, p, hs=hs)
        af.backward(d, p, g, hs=hs)
        torch.cuda.synchronize()
        res.append((hs.cpu().numpy(), g.cpu().numpy()))
        af.close()
    assert np.array_equal(res[0][0], res[1][0]) and np.array_equal(res[0][1], res[1][1])


@pytest.mark.gpu
def test_reused_evaluator_serves_new_data_like_a_fresh_one(cuda):
    from octproengine_b200.autofocus import FitEvaluator, fit_dispersion
    cases = [make_case(m=128, seed=s, d2=d2, d3=d3) for s, d2, d3 in ((21, 15.0, -8.0), (22, -25.0, 6.0))]
    window, ctrue = cases[0][2], cases[0][3]
    af = _af(cuda, O.LANCZOS, window)
    buf = cases[0][0].to(cuda)
    ev = FitEvaluator(af, buf, ctrue)
    for raw_t, _, _, _ in cases:
        buf.copy_(raw_t.to(cuda))  # new data in the evaluator's tensor
        reused = fit_dispersion(af, buf, ctrue, evaluator=ev)
        fresh = fit_dispersion(af, raw_t.to(cuda), ctrue)
        assert (reused.d2, reused.d3, reused.evaluations) == (fresh.d2, fresh.d3, fresh.evaluations)
    with pytest.raises(ValueError):
        fit_dispersion(af, cases[0][0].to(cuda), ctrue, evaluator=ev)  # another tensor


@pytest.mark.gpu
def test_grid_sweep_finds_the_nearest_grid_point(cuda):
    from octproengine_b200.autofocus import grid_sweep
    d2, d3 = 13.0, -6.5
    raw_t, raw, window, ctrue = make_case(m=64, seed=17, d2=d2, d3=d3)
    af = _af(cuda, O.LANCZOS, window)
    res = grid_sweep(af, raw_t.to(cuda), ctrue, n2=17, n3=17)
    assert abs(res.d2 - d2) <= 80.0 / 16 and abs(res.d3 - d3) <= 40.0 / 16, res


@pytest.mark.gpu
def test_rejects_bad_arguments(cuda):
    from octproengine_b200 import capi
    from octproengine_b200.autofocus import Autofocus
    with pytest.raises(capi.B200Error):
        Autofocus(3000, "uint16", O.LANCZOS)
    af = Autofocus(N, "uint16", O.LANCZOS)
    d_p = torch.zeros(8, dtype=torch.float32, device=cuda)
    raw = torch.zeros((4, N), dtype=torch.int16, device=cuda)
    with pytest.raises(capi.B200Error):
        af.forward(raw, d_p)  # neither an image nor (H, S) requested
    with pytest.raises(TypeError):
        af.forward(raw.float(), d_p, hs=torch.empty(2, dtype=torch.float64, device=cuda))


@pytest.mark.gpu
def test_small_copies_move_fit_parameters_without_copy_engines(cuda):
    import ctypes
    import torch
    from octproengine_b200 import capi
    L = capi.lib()
    h = torch.arange(20, dtype=torch.float32).pin_memory()
    d = torch.zeros(20, dtype=torch.float32, device=cuda)
    back = torch.zeros(20, dtype=torch.float32).pin_memory()
    pageable = np.zeros(20, np.float32)
    assert L.ope_b200_af_kernel_accessible(ctypes.c_void_p(h.data_ptr())) == 1
    assert L.ope_b200_af_kernel_accessible(ctypes.c_void_p(d.data_ptr())) == 1
    assert L.ope_b200_af_kernel_accessible(ctypes.c_void_p(pageable.ctypes.data)) == 0
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert L.ope_b200_af_small_copy(ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(h.data_ptr()), 80, s) == capi.OK
    assert L.ope_b200_af_small_copy(ctypes.c_void_p(back.data_ptr() + 4), ctypes.c_void_p(d.data_ptr()), 75,
                                    s) == capi.OK  # unaligned destination, odd size
    torch.cuda.synchronize()
    assert torch.equal(d.cpu(), h)
    want = np.zeros(20, np.float32).view(np.uint8)
    want[4:79] = h.numpy().view(np.uint8)[:75]
    assert np.array_equal(back.numpy().view(np.uint8), want)
    assert L.ope_b200_af_small_copy(ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(h.data_ptr()), 5000,
                                    s) == capi.E_INVALID


@pytest.mark.gpu
def test_distributed_fit_on_one_nccl_rank_equals_the_local_fit(cuda):
    """The data-parallel fit's two all-reduces (entropy partial sums, gradient)
    over NCCL: on one rank it must land where the single-process fit does."""
    import socket
    from datetime import timedelta
    import torch.distributed as dist
    from octproengine_b200.autofocus import fit_dispersion, fit_dispersion_distributed
    raw_t, raw, window, ctrue = make_case(m=128, seed=41, d2=-18.0, d3=9.0)
    af = _af(cuda, O.LANCZOS, window)
    d_raw = raw_t.to(cuda)
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=timedelta(seconds=60), device_id=cuda)
    try:
        got = fit_dispersion_distributed(af, d_raw, ctrue)
    finally:
        dist.destroy_process_group()
    want = fit_dispersion(af, d_raw, ctrue)
    assert abs(got.d2 - want.d2) < 1e-4 and abs(got.d3 - want.d3) < 1e-4, (got, want)
    assert got.entropy == pytest.approx(want.entropy, rel=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("interp", [O.LINEAR, O.CUBIC, O.LANCZOS])
def test_dispersion_only_adjoint_matches_the_full_one(cuda, interp):
    raw_t, raw, window, ctrue = make_case(m=96, seed=23)
    p = params_of(11.0, -4.0, ctrue)
    af = _af(cuda, interp, window)
    d_raw = raw_t.to(cuda)
    d_p = torch.from_numpy(p).to(cuda)
    hs = torch.empty(2, dtype=torch.float64, device=cuda)
    af.forward(d_raw, d_p, hs=hs)
    full = torch.empty(8, dtype=torch.float32, device=cuda)
    disp = torch.full((8,), float("nan"), dtype=torch.float32, device=cuda)
    af.backward(d_raw, d_p, full, hs=hs)
    af.backward(d_raw, d_p, disp, hs=hs, dispersion_only=True)
    f, d = full.cpu().numpy().astype(np.float64), disp.cpu().numpy().astype(np.float64)
    assert np.all(d[4:] == 0.0)
    # the same adjoint up to the rounding of the recomputed resampled samples
    assert np.allclose(d[:4], f[:4], rtol=1e-4, atol=1e-5 * np.abs(f[:4]).max()), (d, f)


@pytest.mark.gpu
def test_dispersion_only_adjoint_reuses_only_matching_tables(cuda):
    """After a forward with the same parameter pointer the adjoint reuses its
    tables; after a forward with another pointer it builds its own: the same
    gradient either way."""
    raw_t, raw, window, ctrue = make_case(m=64, seed=29)
    af = _af(cuda, O.LANCZOS, window)
    d_raw = raw_t.to(cuda)
    A = torch.from_numpy(params_of(11.0, -4.0, ctrue)).to(cuda)
    B = torch.from_numpy(params_of(-20.0, 7.0, ctrue)).to(cuda)
    hs = torch.empty(2, dtype=torch.float64, device=cuda)
    hsB = torch.empty(2, dtype=torch.float64, device=cuda)
    g = [torch.empty(8, dtype=torch.float32, device=cuda) for _ in range(3)]
    af.forward(d_raw, A, hs=hs)
    af.backward(d_raw, A, g[0], hs=hs, dispersion_only=True)  # reuses the tables of A
    af.forward(d_raw, B, hs=hsB)
    af.backward(d_raw, A, g[1], hs=hs, dispersion_only=True)  # tables of B present: rebuilds for A
    af.forward(d_raw, A, hs=hs)
    af.backward(d_raw, A, g[2], hs=hs, dispersion_only=True)
    assert torch.equal(g[0], g[1]) and torch.equal(g[0], g[2])
