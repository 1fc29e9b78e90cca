#!/usr/bin/env python3
"""Benchmark of the B200 OCT chain backend.

Workload (one step = one pass of the chain over one volume buffer):
2048 samples x 1024 A-scans x 64 B-scans uint16 per GPU (512 MiB of algorithmic
traffic), cubic k-linearisation, Gaussian window, dispersion compensation,
fixed-pattern-noise removal with a profile determined beforehand, float32 log
output. Inputs are seeded synthetic spectra (octproengine_b200.synth) made on
the device; they and the outputs (256 MiB each) exceed the 126 MB L2, so no
flush is needed between steps.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0). Under torchrun each rank processes its own
buffer (weak scaling, no collective on the data path); time is the max over
ranks of the device time between barriers.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N, ASCANS, BSCANS = 2048, 1024, 64
METRIC = "A-scans/s (2048-pt chain)"
UNIT = "A-scans/s"
WORKLOAD = ("2048 samples x 1024 A-scans x 64 B-scans uint16 per GPU, cubic resampling, Gaussian window, "
            "dispersion compensation, FPN removal, float32 log output")
# The workload settings in plain numbers (ope::InterpolationMethod, ope::WindowType),
# shared by both arms so that the reference arm needs nothing from the package.
INTERP = {"linear": 0, "cubic": 1, "lanczos": 2}
WINDOW_GAUSS, WINDOW_CENTER, WINDOW_FILL = 1, 0.5, 0.9
DISPERSION_D2_D3 = (12.0, -6.0)
GRAYSCALE_MIN, GRAYSCALE_MAX = 30.0, 110.0
COUNTERS = os.path.join(ROOT, "profiles", "chain_kernel_n2048_cubic_u16.json")


def synth_module():
    """The seeded synthetic-spectrum generator (octproengine_b200/synth.py: numpy
    and torch only, no native library), loaded as a standalone module so that
    the reference arm imports nothing of the package."""
    import importlib.util
    name = "_ope_bench_synth"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "octproengine_b200", "synth.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def bench_config(world=1, bscans=None):
    """The `config` object of the JSON line: identical in both arms."""
    b = BSCANS if bscans is None else bscans
    return {"workload": WORKLOAD, "signal_length": N, "ascans_per_bscan": ASCANS, "bscans_per_buffer": b,
            "input": "uint16", "interpolation": "cubic", "window": "gauss", "dispersion": list(DISPERSION_D2_D3),
            "fpn_removal": True, "output": "float32 log", "global_batch_ascans": world * ASCANS * b,
            "l2": "inputs and outputs larger than L2", "parallelism": f"{world} independent buffers (no collective)"}


def bench_spec(interp=None):
    from octproengine_b200.chain import ChainSpec
    synth = synth_module()
    return ChainSpec(signal_length=N, ascans_per_bscan=ASCANS, bscans_per_buffer=BSCANS, resampling=True,
                     interpolation=INTERP["cubic"] if interp is None else interp,
                     resampling_coeffs=synth.linearising_coeffs(N), windowing=True, window_type=WINDOW_GAUSS,
                     window_center=WINDOW_CENTER, window_fill=WINDOW_FILL, dispersion=True,
                     dispersion_coeffs=synth.compensating_coeffs(*DISPERSION_D2_D3), fpn_removal=True,
                     fpn_bscan_count=1, grayscale_min=GRAYSCALE_MIN, grayscale_max=GRAYSCALE_MAX)


def algorithmic_bytes_per_ascan(n=N, in_bytes=2):
    return n * in_bytes + (n // 2) * 4


def algorithmic_flops_per_ascan(n=N):
    """Nominal floating-point operations of one A-scan of the cubic chain: the
    inverse DFT counted as 5 N log2 N (the conventional FFT count), the
    reference's cubic Hermite formula 19 per sample, window 1 and phase 2 per
    sample, and per output bin FPN 2, |X|^2 3, log 1 and the grayscale affine
    4. 167 936 at N = 2048. Context for the measured pipe counters only."""
    return 5 * n * int(np.log2(n)) + n * (19 + 3) + (n // 2) * (2 + 3 + 1 + 4)


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def kernel_counters():
    """ncu counters of one chain-kernel launch (profiles/*.json, written from a
    capture whose command the file names), or None."""
    if not os.path.exists(COUNTERS):
        return None
    with open(COUNTERS) as f:
        return json.load(f)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup():
    from octproengine_b200.multirank import rank_setup
    return rank_setup()


def ref_params(lib, bscans: int, interp: str = "cubic"):
    """Reference configuration of the benchmark workload (plain numbers)."""
    synth = synth_module()
    return lib.make_params(N, ASCANS, bscans, 2, resampling=True, interpolation=INTERP[interp],
                           resampling_coeffs=synth.linearising_coeffs(N), windowing=True, window_type=WINDOW_GAUSS,
                           window_center=WINDOW_CENTER, window_fill=WINDOW_FILL, dispersion=True,
                           dispersion_coeffs=synth.compensating_coeffs(*DISPERSION_D2_D3), fpn_removal=True,
                           grayscale_min=GRAYSCALE_MIN, grayscale_max=GRAYSCALE_MAX)


def cpu_reference_run(steps: int, warmup: int, threads: int, bscans_per_thread: int = 1):
    """Times the reference CPU backend (oracle/_ref, FFT = project shim in
    float32 mode, not FFTW) on `threads` independent backends, one B-scan of
    the benchmark workload each per step."""
    from concurrent.futures import ThreadPoolExecutor
    from oracle import reflib
    synth = synth_module()
    if not reflib.available():
        reflib.build()
    reflib.set_fft_precision("f32")
    p = ref_params(reflib, bscans_per_thread)
    raw = synth.as_numpy(synth.generate(synth.SynthParams(n=N, ascans=ASCANS, bscans=bscans_per_thread,
                                                          seed=1)), "uint16")
    prof = np.zeros(N, np.float32)
    backends = []
    for _ in range(threads):
        be = reflib.RefBackend(p)
        be.set_fpn(prof)
        backends.append(be)

    def one(i):
        backends[i].process(raw)

    with ThreadPoolExecutor(max_workers=threads) as ex:
        for _ in range(warmup):
            list(ex.map(one, range(threads)))
        t0 = time.perf_counter()
        for _ in range(steps):
            list(ex.map(one, range(threads)))
        dt = time.perf_counter() - t0
    for be in backends:
        be.close()
    ascans = steps * threads * ASCANS * bscans_per_thread
    return ascans / dt, dt, ascans


def cuda_reference_run(steps: int, warmup: int, interp: str = "cubic"):
    """Times the reference CUDA backend (oracle/_ref/libope_cuda_ref.so: the
    reference's cuda_backend.cu + cuda_kernels.cu, cuFFT for the DFT, built with
    the reference's default flags) on the benchmark workload through its own
    API: each step is one process() of a 64-B-scan buffer from the backend's
    registered input ring (2 buffers, the reference default), H2D + kernels +
    D2H, counted at its output callback. Its first frame determines the FPN
    profile (warm-up); timed frames subtract it."""
    from oracle import refcuda
    synth = synth_module()
    if not refcuda.available():
        refcuda.build()
    p = ref_params(refcuda, BSCANS, interp)
    raw = synth.as_numpy(synth.generate(synth.SynthParams(n=N, ascans=ASCANS, bscans=BSCANS, seed=100,
                                                          background_ripple=True)), "uint16")
    be = refcuda.RefCudaBackend(p)
    try:
        be.fill_inputs(raw)
        be.stream(warmup)
        dt = be.stream(steps)
    finally:
        be.close()
    m = ASCANS * BSCANS
    return {"value": steps * m / dt, "unit": UNIT, "ms_per_step": 1e3 * dt / steps,
            "h2d_bytes_per_step": m * N * 2, "d2h_bytes_per_step": m * (N // 2) * 4}


def run_reference(args):
    """The reference arm: the reference's own implementation of the path, with
    nothing of this package loaded (plain numbers for the workload, the data
    generator loaded as a standalone module, rank from the environment)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    line = {
        "impl": "reference", "metric": METRIC, "value": None, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(world),
    }
    if not args.no_cpu_baseline:
        try:
            rate, dt, ascans = cpu_reference_run(args.steps, args.warmup, threads)
        except Exception as e:  # the reference library was not built for this machine
            print(json.dumps({"impl": "reference", "unavailable": str(e).splitlines()[0][:200]}), flush=True)
            return 0
        rate1, _, _ = cpu_reference_run(3, 1, 1)  # one Processor on one core, as the reference runs
        line.update({
            "value": rate, "ms_per_step": 1e3 * dt / args.steps,
            "cpu_baseline": {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                             "sample": f"{ascans} A-scans: {threads} reference CpuBackend instances in parallel, "
                                       f"1 B-scan (1024 A-scans) each per step; FFT = project shim (float32 "
                                       f"radix-2), not FFTW",
                             "sample_ascans_per_step": threads * ASCANS,
                             "single_instance": {"value": rate1, "cores": 1,
                                                 "sample": "3 B-scans through one CpuBackend (its one worker "
                                                           "thread)"}},
            "e2e": {"value": rate, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        })
    if not args.no_cuda_reference:
        # the reference's own GPU path on the same workload, end to end through its API
        try:
            cb = cuda_reference_run(args.steps, args.warmup)
            cb["variants"] = {"lanczos8": cuda_reference_run(max(3, args.steps // 2), args.warmup, "lanczos")}
            cb["kind"] = ("reference CudaBackend (cuda_backend.cu + cuda_kernels.cu, cuFFT), --use_fast_math, "
                          "sm_100; end to end: registered host ring, H2D + chain + D2H per buffer")
            line["cuda_backend"] = cb
        except Exception as e:  # no GPU, or the library could not be built here
            line["cuda_backend"] = {"unavailable": str(e).splitlines()[0][:200]}
    print(json.dumps(line), flush=True)
    return 0


def autofocus_trial(dev, seed, ascans=1024, family=None):
    """Autofocus on one 2048 x 1024 uint16 B-scan: a joint gradient fit of
    the dispersion and the k-map versus 64 x 64 grid sweeps of the same
    forward chain, on this GPU.

    Hidden truth: d2 ~ U[-40, 40], d3 ~ U[-20, 20] rad (centred normalised-k
    phase) and the cubic coefficient of the wavenumber map scaled by
    s ~ 1 + U[-20 %, 20 %]; the data's wavenumber map is the inverse of the
    true resampling polynomial. The joint fit starts from d = 0 and the
    NOMINAL k-map (s = 1) and fits (d2, d3, s) with the full adjoint; the
    dispersion-only fit and the sweeps are given a k-map (the true one, or for
    the sweep also the nominal one, which is what a sweep over (d2, d3) can
    use without knowing the truth). Lanczos-8, Hann window. Error of d2, d3 =
    |fit - true| / max(|true|, 1 rad); of the k-map = |s_fit - s| / s.
    """
    import torch
    from octproengine_b200 import capi, synth
    from octproengine_b200.autofocus import (Autofocus, fit_dispersion, fit_dispersion_kmap, grid_sweep,
                                             KmapFitEvaluator, LANCZOS)
    family = family or synth.KmapFamily(N)
    rng = np.random.default_rng(seed)
    d2, d3 = float(rng.uniform(-40, 40)), float(rng.uniform(-20, 20))
    s_true = 1.0 + float(rng.uniform(-0.2, 0.2))
    ctrue = synth.linearising_coeffs(N, family.k_coeffs(s_true))
    cnom = family(1.0)
    raw = synth.generate(synth.SynthParams(n=N, ascans=ascans, seed=seed + 70, d2=d2, d3=d3,
                                           resampling_truth=ctrue), device=dev)
    window = capi.generate_window_curve(N, 0, 0.5, 0.95)  # Hann
    af = Autofocus(N, "uint16", LANCZOS, window=window, device=dev.index or 0)

    def err(a, b):
        return max(abs(a - d2) / max(abs(d2), 1.0), abs(b - d3) / max(abs(d3), 1.0))

    # first launches (kernel attributes, graph capture) outside the clock
    fit_dispersion(af, raw, ctrue, max_iter=2)
    grid_sweep(af, raw, ctrue, n2=2, n3=2)
    ev = KmapFitEvaluator(af, raw, family, [1.0])
    torch.cuda.synchronize(dev)
    joint = fit_dispersion_kmap(af, raw, family, [1.0], evaluator=ev)
    fit = fit_dispersion(af, raw, ctrue)  # each evaluation replays one CUDA graph
    sweep = grid_sweep(af, raw, ctrue, n2=64, n3=64)  # the 4096 forward passes in one CUDA graph
    sweep_nom = grid_sweep(af, raw, cnom, n2=64, n3=64)
    sweep_err = err(sweep.d2, sweep.d3)
    t_equal = next((h[3] for h in fit.history if err(h[0], h[1]) <= sweep_err), None)
    s_fit = float(joint.kappa[0])
    af.close()
    return {"seed": seed, "d2": d2, "d3": d3, "kmap_cubic_scale": s_true,
            "joint_fit_s": joint.seconds, "joint_fit_evals": joint.evaluations,
            "joint_fit_err_dispersion": err(joint.d2, joint.d3), "joint_fit_err_kmap": abs(s_fit - s_true) / s_true,
            "joint_fit_d2": joint.d2, "joint_fit_d3": joint.d3, "joint_fit_kmap_cubic_scale": s_fit,
            "fit_s": fit.seconds, "fit_err": err(fit.d2, fit.d3), "fit_evals": fit.evaluations,
            "fit_d2": fit.d2, "fit_d3": fit.d3, "sweep_s": sweep.seconds, "sweep_err": sweep_err,
            "sweep_d2": sweep.d2, "sweep_d3": sweep.d3, "fit_s_to_sweep_err": t_equal,
            "sweep_nominal_kmap_s": sweep_nom.seconds, "sweep_nominal_kmap_err": err(sweep_nom.d2, sweep_nom.d3)}


def autofocus_bench(dev, seeds=range(8), ascans=1024):
    from octproengine_b200 import synth
    family = synth.KmapFamily(N)
    trials = [autofocus_trial(dev, s, ascans, family) for s in seeds]
    med = lambda k: float(np.median([t[k] for t in trials]))
    eq = [t["sweep_s"] / t["fit_s_to_sweep_err"] for t in trials if t["fit_s_to_sweep_err"]]
    jw = [max(t["joint_fit_err_dispersion"], t["joint_fit_err_kmap"]) for t in trials]
    return {
        "workload": (f"2048 x {ascans} uint16 B-scan per trial, {len(trials)} seeded trials (hidden d2 ~ U[-40,40], "
                     "d3 ~ U[-20,20] rad, k-map cubic coefficient scaled by 1 + U[-20 %, 20 %]), Lanczos-8, Hann "
                     "window, entropy objective; error = max |fit - true| / max(|true|, 1 rad) over (d2, d3), and "
                     "|s_fit - s| / s for the k-map"),
        "unit": "s per B-scan",
        "joint_fit": {
            "what": "BFGS on (d2, d3, k-map cubic scale) from d = 0 and the nominal k-map, full adjoint",
            "seconds_median": med("joint_fit_s"), "evaluations_median": med("joint_fit_evals"),
            "error_dispersion_median": med("joint_fit_err_dispersion"), "error_kmap_median": med("joint_fit_err_kmap"),
            "error_max": float(max(jw)), "trials_within_1pct": int(sum(e < 0.01 for e in jw)),
            "trials_kmap_within_1pct": int(sum(t["joint_fit_err_kmap"] < 0.01 for t in trials)),
            "trials_within_3pct": int(sum(e < 0.03 for e in jw)),
            "speedup_vs_sweep_median": float(np.median([t["sweep_s"] / t["joint_fit_s"] for t in trials])),
            "sweep_at_nominal_kmap_error_median": med("sweep_nominal_kmap_err"),
        },
        "fit_seconds_median": med("fit_s"),
        "fit_error_median": med("fit_err"),
        "fit_error_max": float(max(t["fit_err"] for t in trials)),
        "fit_trials_within_1pct": int(sum(t["fit_err"] < 0.01 for t in trials)),
        "fit_note": "dispersion-only fit given the true k-map",
        "sweep_64x64_seconds_median": med("sweep_s"),
        "sweep_error_median": med("sweep_err"),
        "speedup_vs_sweep_median": float(np.median([t["sweep_s"] / t["fit_s"] for t in trials])),
        "speedup_at_equal_error_median": float(np.median(eq)) if eq else None,
        "trials": trials,
    }


def batch_bench(dev, seed=3, count=32, steps=20):
    """32 uneven buffers in one persistent launch replayed from a CUDA graph.

    Buffers drawn from `seed`: N in {1024, 2048, 4096}, A-scan counts uniform
    in [256, 2048], input uint8 / uint16 / float32, resampling linear / cubic /
    Lanczos-8 and window Hann / Gauss / sine / flat-top per buffer, dispersion
    on, log output. The autotuner picks pairs-per-team and the radix schedule
    per length first. Reported: total A-scans/s of the one-launch batch, the
    same buffers as sequential single-buffer launches, and per length the HBM
    fraction of that length's buffers launched alone, beside the rate those
    buffers would reach at the single-buffer kernel's steady rate for each
    buffer's configuration (input type, resampling; one long launch each).
    """
    import torch
    from octproengine_b200 import synth
    from octproengine_b200.batch import Batch
    from octproengine_b200.chain import ChainSpec, open_context, UINT8, UINT16, FLOAT32, LINEAR, CUBIC, \
        LANCZOS, HANN, GAUSS, SINE, FLAT_TOP
    rng = np.random.default_rng(seed)
    names = {UINT8: "uint8", UINT16: "uint16", FLOAT32: "float32"}
    bytes_in = {UINT8: 1, UINT16: 2, FLOAT32: 4}
    bufs = []
    for k in range(count):
        n = int(rng.choice([1024, 2048, 4096]))
        m = int(rng.integers(256, 2049))
        dt = int(rng.choice([UINT8, UINT16, FLOAT32]))
        interp = int(rng.choice([LINEAR, CUBIC, LANCZOS]))
        win = int(rng.choice([HANN, GAUSS, SINE, FLAT_TOP]))
        spec = ChainSpec(signal_length=n, ascans_per_bscan=m, input_dtype=dt, resampling=True, interpolation=interp,
                         resampling_coeffs=synth.linearising_coeffs(n), windowing=True, window_type=win,
                         window_center=0.5, window_fill=0.9, dispersion=True,
                         dispersion_coeffs=synth.compensating_coeffs(12.0, -6.0), grayscale_min=0.0,
                         grayscale_max=100.0, device=dev.index or 0)
        x = synth.generate(synth.SynthParams(n=n, ascans=m, seed=1000 + k, dtype=names[dt]), device=dev)
        o = torch.empty((m, n // 2), dtype=torch.float32, device=dev)
        bufs.append((spec, open_context(spec), x, o))
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream

    def items(sel):
        return [(c, x.data_ptr(), o.data_ptr(), s.num_ascans) for s, c, x, o in sel]

    def timed(fn, reps):
        for _ in range(3):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    batch = Batch(items(bufs))
    batch.autotune(3)
    tuning = {n: batch.tuning(n) for n in (1024, 2048, 4096)}
    ms_graph = timed(lambda: batch.run_graph(sp), steps)
    ms_seq = timed(lambda: [c.process_device(x.data_ptr(), o.data_ptr(), sp, num_ascans=s.num_ascans)
                            for s, c, x, o in bufs], steps)
    total = sum(s.num_ascans for s, _, _, _ in bufs)
    peak = measured_peak()[0]
    per_len = {}
    from octproengine_b200.batch import radix_plan
    for n in (1024, 2048, 4096):
        sel = [b for b in bufs if b[0].signal_length == n]
        if not sel:
            continue
        sub = Batch(items(sel))
        sub.set_tuning(n, tuning[n][0], tuning[n][1])
        ms = timed(lambda: sub.run_graph(sp), steps)
        # the same buffers as single-buffer launches (each its own chain kernel),
        # the rate the batch is compared with at this length
        ms_single = timed(lambda: [c.process_device(x.data_ptr(), o.data_ptr(), sp, num_ascans=s.num_ascans)
                                   for s, c, x, o in sel], steps)
        # each buffer's own configuration at the single-buffer kernel's steady
        # rate: one launch over >= 32768 A-scans of it (its rows repeated), so
        # the time these buffers would take at that rate is sum(m_i / rate_i)
        ms_steady = 0.0
        for s, c, x, _ in sel:
            reps_rows = -(-32768 // s.num_ascans)
            xb = x.repeat(reps_rows, 1)
            ob = torch.empty((xb.shape[0], n // 2), dtype=torch.float32, device=dev)
            ms_big = timed(lambda: c.process_device(xb.data_ptr(), ob.data_ptr(), sp, num_ascans=xb.shape[0]), 5)
            ms_steady += ms_big * s.num_ascans / xb.shape[0]
            del xb, ob
        nbytes = sum(s.num_ascans * (n * bytes_in[s.input_dtype] + (n // 2) * 4) for s, _, _, _ in sel)
        asc = sum(s.num_ascans for s, _, _, _ in sel)
        per_len[str(n)] = {"buffers": len(sel), "ascans": asc, "ascans_per_s": asc / (ms / 1e3),
                           "gbs": nbytes / (ms / 1e3) / 1e9, "hbm_frac": nbytes / (ms / 1e3) / 1e9 / peak,
                           "single_buffer_launches_ascans_per_s": asc / (ms_single / 1e3),
                           "batch_over_single": ms_single / ms,
                           "single_kernel_steady_ascans_per_s": asc / (ms_steady / 1e3),
                           "batch_over_steady": ms_steady / ms,
                           "pairs_per_team": tuning[n][0], "radix_schedule": tuning[n][1],
                           "radix_plan": radix_plan(n, tuning[n][1])}
        sub.close()
    batch.close()
    for _, c, _, _ in bufs:
        if c.synchronize() != 0:
            raise RuntimeError("batched chain reported a device status")
        c.close()
    return {"workload": f"{count} buffers (seed {seed}): N in {{1024, 2048, 4096}}, A-scans U[256, 2048], "
                        "uint8/uint16/float32, linear/cubic/Lanczos-8, Hann/Gauss/sine/flat-top, one persistent "
                        "launch replayed from a CUDA graph",
            "ascans": total, "value": total / (ms_graph / 1e3), "unit": "A-scans/s", "ms_per_batch": ms_graph,
            "sequential_single_launches": {"value": total / (ms_seq / 1e3), "ms_per_batch": ms_seq},
            "per_length": per_len, "gpu_launches_per_batch": 1}


def ring_stream(ctx, inputs, frames: int, fit=None) -> float:
    """Pushes `frames` buffers (cycling over the pinned host tensors `inputs`)
    back to back through the context's frame ring (submit / wait / release,
    as many in flight as the ring has slots); each frame's output lands in the
    slot's pinned host buffer. `fit(k, ticket)`, when given, runs on the host
    while frames are in flight, before frame k is waited for. Returns wall
    seconds from the first submit to the last completed frame."""
    from collections import deque
    depth = ctx_ring_depth(ctx)
    tickets = deque()
    k = done = 0
    t0 = time.perf_counter()
    while done < frames:
        while k < frames and len(tickets) < depth:
            tickets.append(ctx.submit(inputs[k % len(inputs)].data_ptr()))
            k += 1
        if fit is not None:
            fit(done, tickets[0])
        t = tickets.popleft()
        ctx.wait(t, 60000)
        ctx.release(t)
        done += 1
    return time.perf_counter() - t0


def ctx_ring_depth(ctx) -> int:
    from octproengine_b200 import capi
    return int(capi.lib().ope_b200_ring_depth(ctx.h))


def streaming_bench(dev, chunks=16, bscans_per_chunk=32, pool=4, n=4096, ascans=1024, seed=5):
    """The streaming-volume workload: 4096 samples x 1024 A-scans x 512 B-scans
    uint16 (4 GiB raw) pushed from pinned host memory through the frame ring in
    32-B-scan chunks (cubic resampling, Hann window, dispersion compensation,
    float32 log output, the chunk's output back in pinned host memory), with a
    gradient dispersion fit (Lanczos-8, entropy) of one B-scan per chunk on a
    separate stream, overlapped with the ring. The host holds `pool` distinct
    chunks (seeded synthetic scenes sharing one hidden dispersion) and cycles
    over them, as a frame grabber cycles over its buffers. Fit error = max over
    (d2, d3) of |fit - true| / max(|true|, 1 rad) against the generating
    dispersion."""
    import torch
    from octproengine_b200 import capi, synth
    from octproengine_b200.chain import ChainSpec, open_context, CUBIC, HANN
    from octproengine_b200.autofocus import Autofocus, FitEvaluator, fit_dispersion, dispersion_poly, \
        frame_input_view, LANCZOS
    rng = np.random.default_rng(seed)
    d2, d3 = float(rng.uniform(-40, 40)), float(rng.uniform(-20, 20))
    s = 2048.0 / n  # the k-map's non-linearity scaled to the record length
    kc = (synth.K_COEFFS[0], synth.K_COEFFS[1], synth.K_COEFFS[2] * s, synth.K_COEFFS[3] * s * s)
    ctrue = synth.linearising_coeffs(n, kc)
    m = ascans * bscans_per_chunk
    spec = ChainSpec(signal_length=n, ascans_per_bscan=ascans, bscans_per_buffer=bscans_per_chunk,
                     resampling=True, interpolation=CUBIC, resampling_coeffs=ctrue, windowing=True,
                     window_type=HANN, window_center=0.5, window_fill=0.95, dispersion=True,
                     dispersion_coeffs=tuple(dispersion_poly(d2, d3)), grayscale_min=20.0, grayscale_max=100.0,
                     device=dev.index or 0)
    pinned = []
    x = None
    for p in range(pool):
        x = synth.generate(synth.SynthParams(n=n, ascans=ascans, bscans=bscans_per_chunk, seed=300 + p, d2=d2,
                                             d3=d3, resampling_truth=ctrue), device=dev)
        h = torch.empty(x.numel() * 2, dtype=torch.uint8).pin_memory()
        h.copy_(x.view(torch.uint8).reshape(-1).cpu())
        pinned.append(h)
    # device-resident chain on one chunk (kernel only)
    out = torch.empty((m, n // 2), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    ctx = open_context(spec)
    for _ in range(3):
        ctx.process_device(x.data_ptr(), out.data_ptr(), stream.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(10):
        ctx.process_device(x.data_ptr(), out.data_ptr(), stream.cuda_stream)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    kms = e0.elapsed_time(e1) / 10
    del x, out
    ctx.close()
    peak, _ = measured_peak()
    res = {"workload": (f"{n} samples x {ascans} A-scans x {chunks * bscans_per_chunk} B-scans uint16 "
                        f"({chunks * m * n * 2 / 2**30:.0f} GiB raw) in {bscans_per_chunk}-B-scan chunks through the "
                        f"frame ring from pinned host memory ({pool} distinct chunks cycled), cubic, Hann, "
                        f"dispersion, float32 log output to pinned host; fit: one {ascans}-A-scan B-scan per "
                        f"chunk read in place from the ring slot, Lanczos-8 entropy, started from the previous "
                        f"chunk's result, on its own stream"),
           "unit": "A-scans/s", "hidden_d2": d2, "hidden_d3": d3,
           "device_resident_chunk": {"value": m / (kms / 1e3), "ms_per_chunk": kms,
                                     "hbm_frac": m * algorithmic_bytes_per_ascan(n) / (kms / 1e3) / 1e9 / peak}}
    window = capi.generate_window_curve(n, HANN, 0.5, 0.95)
    af = Autofocus(n, "uint16", LANCZOS, window=window, device=dev.index or 0)
    fit_stream = torch.cuda.Stream(dev)
    fits = []
    evaluators = {}  # per ring slot: a view of its device input and one captured fit graph

    def fit(k, ticket):
        # the chunk's first B-scan, read in place from the ring slot's device copy
        with torch.cuda.stream(fit_stream):
            view = frame_input_view(ctx, ticket, ascans, fit_stream)
            key = view.data_ptr()
            if key not in evaluators:
                evaluators[key] = (view, FitEvaluator(af, view, ctrue))
            view, ev = evaluators[key]
            # the dispersion of one volume changes little from chunk to chunk: each
            # fit starts where the previous chunk's ended (the first from zero)
            init = (fits[-1].d2, fits[-1].d3) if fits else (0.0, 0.0)
            fits.append(fit_dispersion(af, view, ctrue, init=init, evaluator=ev))

    def err(f):
        return max(abs(f.d2 - d2) / max(abs(d2), 1.0), abs(f.d3 - d3) / max(abs(d3), 1.0))

    for depth in (2, 3):
        ctx = open_context(spec.with_(num_input_buffers=depth))
        ring_stream(ctx, pinned, 2)  # slots, pinned outputs, first launches
        dt = ring_stream(ctx, pinned, chunks)
        res[f"ring_depth{depth}"] = {"value": chunks * m / dt, "seconds": dt,
                                     "host_gbs": chunks * m * (n * 2 + n // 2 * 4) / dt / 1e9}
        if depth == 2:
            ring_stream(ctx, pinned, depth, fit=fit)  # one fit graph per ring slot, captured here
            fits.clear()
            torch.cuda.synchronize(dev)
            dt = ring_stream(ctx, pinned, chunks, fit=fit)
            torch.cuda.synchronize(dev)
            errs = [err(f) for f in fits]
            res["with_fits"] = {"value": chunks * m / dt, "seconds": dt, "fits": len(fits),
                                "fit_seconds_median": float(np.median([f.seconds for f in fits])),
                                "fit_seconds_total": float(sum(f.seconds for f in fits)),
                                "fit_evaluations_median": float(np.median([f.evaluations for f in fits])),
                                "fit_error_median": float(np.median(errs)), "fit_error_max": float(max(errs)),
                                "fits_within_1pct": int(sum(e < 0.01 for e in errs))}
        ctx.close()
    af.close()
    res["value"] = res["with_fits"]["value"]
    return res


def run_ours(args):
    import torch
    from octproengine_b200 import synth
    from octproengine_b200.chain import open_context, LANCZOS

    world, rank, local = dist_setup()
    dist = None
    if world > 1:
        import torch.distributed as dist_mod
        from datetime import timedelta
        dist = dist_mod
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    interp = INTERP[args.interp]
    spec = bench_spec(interp).with_(device=local, bscans_per_buffer=BSCANS)
    M = spec.num_ascans
    x = synth.generate(synth.SynthParams(n=N, ascans=ASCANS, bscans=BSCANS, seed=100 + rank,
                                         background_ripple=True), device=dev)
    out = torch.empty((M, N // 2), dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    ctx = open_context(spec)
    # FPN profile determined once from the first B-scan of the buffer
    ctx.request_fpn_determination()
    ctx.process_device(x.data_ptr(), out.data_ptr(), sp)
    torch.cuda.synchronize(dev)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    for _ in range(args.warmup):
        ctx.process_device(x.data_ptr(), out.data_ptr(), sp)
    barrier()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        # nvidia-smi needs a moment to start: wait for its first sample, then
        # keep the same work running for ~0.5 s so the sampled clocks are the
        # clocks under this load, then time the K steps inside the sampling window
        t_wait = time.time()
        while not clk.lines and time.time() - t_wait < 5.0:
            time.sleep(0.05)
        t_soak = time.time()
        while time.time() - t_soak < 0.5:
            for _ in range(50):
                ctx.process_device(x.data_ptr(), out.data_ptr(), sp)
            torch.cuda.synchronize(dev)
        barrier()
        ev0.record(stream)
        for _ in range(args.steps):
            ctx.process_device(x.data_ptr(), out.data_ptr(), sp)
        ev1.record(stream)
        barrier()
        time.sleep(0.25)
    from octproengine_b200.multirank import max_over_ranks, weak_scaling_rate
    ms = ev0.elapsed_time(ev1)
    ms_max = max_over_ranks(ms, device=dev)  # the slowest rank's device time
    if ctx.synchronize() != 0:
        raise RuntimeError("chain kernel reported a device status")
    ms_step = ms_max / args.steps
    value = weak_scaling_rate(M, ms_step / 1e3, world)

    # kernel-only launch duration (the one chain kernel per step)
    kernel_ms = ms / args.steps
    bytes_launch = M * algorithmic_bytes_per_ascan()
    achieved = bytes_launch / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    counters = kernel_counters()

    variants = {}
    if args.kernel_only:
        ctx.close()
        if dist is not None:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "ms_per_step": ms_step,
                              "kernel_only": True, "bscans": BSCANS, "interp": args.interp,
                              "hbm_frac": (M * algorithmic_bytes_per_ascan() / (ms / args.steps / 1e3) / 1e9)
                              / measured_peak()[0]}), flush=True)
        return 0
    # Lanczos variant and FPN determination frame (same buffer)
    spec_l = spec.with_(interpolation=LANCZOS)
    ctx_l = open_context(spec_l)
    ctx_l.set_fpn_profile(ctx.fpn_profile())
    for _ in range(2):
        ctx_l.process_device(x.data_ptr(), out.data_ptr(), sp)
    torch.cuda.synchronize(dev)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    reps = max(3, args.steps // 2)
    e0.record(stream)
    for _ in range(reps):
        ctx_l.process_device(x.data_ptr(), out.data_ptr(), sp)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    lms = e0.elapsed_time(e1) / reps
    variants["lanczos8"] = {"value": M / (lms / 1e3), "unit": UNIT, "ms_per_step": lms,
                            "hbm_frac": bytes_launch / (lms / 1e3) / 1e9 / peak}
    ctx_l.close()
    # rolling-average DC removal (window 64) on the same buffer: exact window
    # sums; the reference's float prefix order on these full-range 16-bit
    # samples (row totals above 2^24: the serial prefix); and the reference
    # order on 12-bit samples (the same buffer through DataParameters::bitshift:
    # row totals below 2^24, so the exact prefix equals the float one)
    for name, kw in (("rolling_dc_exact_sums", {}), ("rolling_dc_reference_order", {"dc_reference_order": True}),
                     ("rolling_dc_reference_order_12bit", {"dc_reference_order": True, "bitshift": True})):
        ctx_d = open_context(spec.with_(dc_removal=True, dc_window=64, **kw))
        ctx_d.set_fpn_profile(ctx.fpn_profile())
        for _ in range(2):
            ctx_d.process_device(x.data_ptr(), out.data_ptr(), sp)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        for _ in range(reps):
            ctx_d.process_device(x.data_ptr(), out.data_ptr(), sp)
        e1.record(stream)
        torch.cuda.synchronize(dev)
        dms = e0.elapsed_time(e1) / reps
        variants[name] = {"value": M / (dms / 1e3), "unit": UNIT, "ms_per_step": dms}
        ctx_d.close()
    e0.record(stream)
    for _ in range(reps):
        ctx.request_fpn_determination()
        ctx.process_device(x.data_ptr(), out.data_ptr(), sp)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    fms = e0.elapsed_time(e1) / reps
    variants["fpn_determination_frame"] = {"value": M / (fms / 1e3), "unit": UNIT, "ms_per_step": fms}

    # end to end through the public API with host buffers (pinned), H2D + D2H timed
    xh = torch.empty((M, N), dtype=torch.int16).pin_memory()
    xh.copy_(x.cpu())
    oh = torch.empty((M, N // 2), dtype=torch.float32).pin_memory()
    raw_np = xh.numpy().view(np.uint16)
    out_np = oh.numpy()
    for _ in range(2):
        ctx.process_host(raw_np, out_np)
    e2e_steps = max(3, min(args.steps, 10))
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        ctx.process_host(raw_np, out_np)
    e2e_dt = max_over_ranks(time.perf_counter() - t0, device=dev)
    e2e_value = weak_scaling_rate(M * e2e_steps, e2e_dt, world)

    # sustained end to end through the frame ring (frames back to back, as the
    # reference's ring is driven): depth 2, the reference's default
    ctx_r = open_context(spec.with_(num_input_buffers=2))
    ctx_r.set_fpn_profile(ctx.fpn_profile())
    ring_in = [xh.view(torch.uint8).reshape(-1)]
    ring_stream(ctx_r, ring_in, 2)
    barrier()
    ring_dt = max_over_ranks(ring_stream(ctx_r, ring_in, e2e_steps), device=dev)
    ctx_r.close()
    e2e_stream = {"value": weak_scaling_rate(M * e2e_steps, ring_dt, world), "unit": UNIT,
                  "api": "ope_b200_submit / wait / release, frames back to back", "ring_depth": 2,
                  "h2d_bytes_per_step": M * N * 2, "d2h_bytes_per_step": M * (N // 2) * 4}

    autofocus = None
    if world == 1 and not args.no_autofocus:
        autofocus = autofocus_bench(dev)
    batched = None
    if world == 1 and not args.no_batch:
        batched = batch_bench(dev)
    streaming = None
    if world == 1 and not args.no_streaming:
        streaming = streaming_bench(dev)

    cpu_base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        try:
            # a bounded sample: 20 B-scans per core (about 20 core-seconds of work)
            rate, dt, ascans = cpu_reference_run(20, 2, threads)
            rate1, _, _ = cpu_reference_run(3, 1, 1)
            cpu_base = {"value": rate, "unit": UNIT, "cores": threads, "kind": "reference",
                        "sample": f"{ascans} A-scans in {dt:.1f} s ({threads} reference CpuBackend instances x "
                                  f"20 B-scans of the workload); FFT = project shim (float32 radix-2), not FFTW",
                        "single_instance": {"value": rate1, "cores": 1,
                                            "sample": "3 B-scans through one CpuBackend (its one worker thread)"}}
        except Exception as e:  # the reference library was not built for this machine
            cpu_base = {"unavailable": str(e).splitlines()[0][:200]}
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    clocks = clk.summary()
    traffic = None
    pipes = None
    if counters:
        # DRAM bytes of one captured launch, scaled to this launch by A-scan count
        per_ascan = (counters["dram_bytes_read"] + counters["dram_bytes_write"]) / counters["ascans"]
        traffic = per_ascan * M
        pipes = {k: counters[k] for k in ("fma_pipe_active_pct", "issue_active_pct", "warps_active_pct",
                                          "thread_inst_per_ascan", "l1_data_pipe_pct") if k in counters}
        pipes.update({"flops_per_ascan_nominal": algorithmic_flops_per_ascan(),
                      "source": f"ncu, one launch over {counters['ascans']} A-scans: {counters['command']}"})
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(world),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": traffic,
                     "traffic_note": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch over "
                                      f"{counters['ascans']} A-scans, scaled to {M} by A-scan count; writes "
                                      f"still held in L2 when the kernel ends are not counted") if counters else None,
                     "algorithmic_bytes": bytes_launch},
        # the chain's other roof: the FP32 pipe, as ncu counted it for one launch
        "fp32_pipe": pipes,
        # end to end through the reference-facing streaming path (the frame ring that
        # process(IOBuffer&) feeds); the one-call synchronous path beside it
        "e2e": e2e_stream,
        "e2e_sync": {"value": e2e_value, "unit": UNIT, "api": "ope_b200_process_host, one call per buffer",
                     "h2d_bytes_per_step": M * N * 2, "d2h_bytes_per_step": M * (N // 2) * 4},
        "gpu_launches": args.steps,
        "clocks": clocks,
        "variants": variants,
    }
    if autofocus:
        line["autofocus"] = autofocus
    if batched:
        line["batched"] = batched
    if streaming:
        line["streaming_volume"] = streaming
    if cpu_base:
        line["cpu_baseline"] = cpu_base
    print(json.dumps(line), flush=True)
    return 0


def main():
    global BSCANS
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cuda-reference", action="store_true",
                    help="reference arm: skip timing the reference CUDA backend")
    ap.add_argument("--no-autofocus", action="store_true", help="skip the autofocus fit-versus-sweep line")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched uneven-buffer line")
    ap.add_argument("--no-streaming", action="store_true", help="skip the streaming-volume line")
    ap.add_argument("--bscans", type=int, default=BSCANS, help="B-scans per buffer (profiling uses fewer)")
    ap.add_argument("--interp", default="cubic", choices=["linear", "cubic", "lanczos"])
    ap.add_argument("--kernel-only", action="store_true",
                    help="only the timed device loop (for ncu captures): no variants, e2e or CPU baseline")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    BSCANS = args.bscans
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
