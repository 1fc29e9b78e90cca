"""Host-side tests of the reference-facing API layers (no GPU needed).

* the ``octproengine`` Python module: the reference binding's names, enums,
  configuration defaults (include/processorconfiguration.h:16-115 of the
  reference), custom curves, INI persistence, callback registry and the
  errors raised without a device;
* ``libope_host.so``: the C++ classes export the symbols a reference caller
  links against, and a reference example program compiles and links against
  ``include/ope`` + ``libope_host.so`` unchanged (when the reference sources
  are present).
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import octproengine_b200 as pkg
from octproengine_b200 import build as B

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ope():
    B.build()
    return pkg.reference_api()


def test_module_surface(ope):
    for name in ["Processor", "ProcessorConfiguration", "DataParameters", "ProcessingParameters",
                 "ResamplingParameters", "WindowingParameters", "DispersionCompensationParameters",
                 "BackgroundRemovalParameters", "PostProcessingParameters", "IOBuffer", "Backend", "DataType",
                 "InterpolationMethod", "WindowType", "InitializationError", "ConfigurationError",
                 "BufferError", "ProcessingError", "BackendError"]:
        assert hasattr(ope, name), name
    methods = ["initialize", "stop", "load_config", "save_config", "set_config", "set_input_parameters",
               "set_backend", "get_backend", "set_callback", "add_output_callback", "remove_output_callback",
               "clear_output_callbacks", "get_callback_count", "process", "get_next_available_buffer",
               "set_resampling_coefficients", "set_custom_resampling_curve", "use_custom_resampling_curve",
               "enable_resampling", "set_interpolation_method", "set_dispersion_coefficients",
               "set_custom_dispersion_curve", "use_custom_dispersion_curve", "enable_dispersion_compensation",
               "set_window_parameters", "set_custom_window_curve", "use_custom_window_curve", "enable_windowing",
               "set_grayscale_range", "set_signal_multiplicator_and_addend", "enable_log_scaling",
               "enable_background_removal", "set_background_removal_window_size", "enable_bscan_flip",
               "enable_sinusoidal_scan_correction", "enable_fixed_pattern_noise_removal",
               "enable_post_process_background_subtraction", "request_post_process_background_recording",
               "set_post_process_background_weight", "set_post_process_background_offset",
               "has_post_process_background_profile", "get_post_process_background_profile_size",
               "get_post_process_background_profile", "set_post_process_background_profile",
               "save_post_process_background_profile_to_file", "load_post_process_background_profile_from_file",
               "request_fixed_pattern_noise_determination", "enable_continuous_fixed_pattern_noise_determination",
               "set_fixed_pattern_noise_bscan_count", "has_fixed_pattern_noise_profile",
               "get_fixed_pattern_noise_profile_size", "get_fixed_pattern_noise_profile",
               "set_fixed_pattern_noise_profile", "save_fixed_pattern_noise_profile_to_file",
               "load_fixed_pattern_noise_profile_from_file", "__enter__", "__exit__"]
    for m in methods:
        assert hasattr(ope.Processor, m), m


def test_enum_values(ope):
    # values of include/types.h:6-19 and include/processorconfiguration.h:11-33 of the reference
    assert int(ope.DataType.UINT8) == 1 and int(ope.DataType.UINT16) == 2 and int(ope.DataType.FLOAT32) == 9
    assert int(ope.DataType.COMPLEX_FLOAT64) == 12
    assert [int(ope.InterpolationMethod.LINEAR), int(ope.InterpolationMethod.CUBIC),
            int(ope.InterpolationMethod.LANCZOS)] == [0, 1, 2]
    assert [int(getattr(ope.WindowType, n)) for n in
            ["HANN", "GAUSS", "SINE", "LANCZOS", "RECTANGULAR", "FLAT_TOP"]] == list(range(6))
    assert int(ope.Backend.CUDA) == 0 and int(ope.Backend.CPU) == 1 and int(ope.Backend.B200) == 2


def test_configuration_defaults(ope):
    c = ope.ProcessorConfiguration()
    d = c.data
    assert (d.signal_length, d.samples_per_buffer, d.ascans_per_bscan, d.bscans_per_buffer) == (1024, 1024 * 512,
                                                                                               512, 1)
    assert d.input_data_type == ope.DataType.UINT16 and not d.bitshift
    assert d.get_bit_depth() == 16 and d.get_bytes_per_sample() == 2
    p = c.processing
    assert (p.n_streams, p.n_buffers, p.grid_size, p.block_size) == (8, 4, 4096, 128)
    r = c.resampling
    assert not r.enabled and r.interpolation_method == ope.InterpolationMethod.LINEAR and r.use_coefficients
    assert r.coefficients == [0.0, 1.0, 0.0, 0.0] and not r.use_custom_curve
    w = c.windowing
    assert not w.enabled and w.window_type == ope.WindowType.HANN
    assert w.window_center_position == pytest.approx(0.5) and w.window_fill_factor == pytest.approx(0.95)
    q = c.dispersion
    assert not q.enabled and q.use_coefficients and q.coefficients == [0.0] * 4 and q.factor == 1.0
    assert not c.background_removal.enabled and c.background_removal.rolling_average_window_size == 64
    pp = c.post_processing
    assert not pp.background_removal and pp.background_weight == 1.0 and pp.background_offset == 0.0
    assert pp.log_scaling and pp.grayscale_max == 100.0 and pp.grayscale_min == 30.0
    assert pp.addend == 0.0 and pp.multiplicator == 1.0
    assert not pp.bscan_flip and not pp.sinusoidal_scan_correction and not pp.fixed_pattern_noise_removal
    assert pp.fixed_pattern_noise_bscan_count == 1 and not pp.continuous_fixed_pattern_noise_determination
    assert c.validate()
    with pytest.raises(RuntimeError):
        c.resampling.coefficients = [1.0, 2.0]


def test_custom_curves_adjusted_to_signal_length(ope):
    c = ope.ProcessorConfiguration()
    assert not c.has_custom_resampling_curve() and c.get_custom_resampling_curve().size == 0
    c.data.signal_length = 8
    c.set_custom_resampling_curve(np.arange(5, dtype=np.float32))
    c.set_custom_window_curve(np.ones(12, dtype=np.float32))
    c.set_custom_dispersion_curve(np.arange(8, dtype=np.float64))  # cast to float32
    assert c.has_custom_resampling_curve() and c.has_custom_window_curve() and c.has_custom_dispersion_curve()
    np.testing.assert_array_equal(c.get_custom_resampling_curve(), [0, 1, 2, 3, 4, 0, 0, 0])
    np.testing.assert_array_equal(c.get_custom_window_curve(), np.ones(8))
    np.testing.assert_array_equal(c.get_custom_dispersion_curve(), np.arange(8))
    with pytest.raises(ope.BufferError):
        c.set_custom_window_curve(np.ones((2, 4), dtype=np.float32))


def test_ini_roundtrip(ope, tmp_path):
    c = ope.ProcessorConfiguration()
    c.data.signal_length = 2048
    c.data.ascans_per_bscan = 1024
    c.data.bscans_per_buffer = 64
    c.data.samples_per_buffer = 2048 * 1024 * 64
    c.data.input_data_type = ope.DataType.UINT8
    c.resampling.enabled = True
    c.resampling.interpolation_method = ope.InterpolationMethod.LANCZOS
    c.resampling.coefficients = [0.5, 1.25, -3e-5, 1e-9]
    c.windowing.window_type = ope.WindowType.FLAT_TOP
    c.windowing.window_fill_factor = 0.8
    c.dispersion.coefficients = [0.0, 0.0, 12.5, -3.25]
    c.background_removal.rolling_average_window_size = 32
    c.post_processing.grayscale_min = 12.0
    c.post_processing.bscan_flip = True
    c.post_processing.fixed_pattern_noise_bscan_count = 7
    c.set_custom_window_curve(np.linspace(0, 1, 2048, dtype=np.float32))
    path = str(tmp_path / "cfg.ini")
    assert c.save_to_file(path)
    d = ope.ProcessorConfiguration()
    assert d.load_from_file(path)
    assert d.data.signal_length == 2048 and d.data.bscans_per_buffer == 64
    assert d.data.input_data_type == ope.DataType.UINT8
    assert d.resampling.interpolation_method == ope.InterpolationMethod.LANCZOS
    assert d.resampling.coefficients == pytest.approx([0.5, 1.25, -3e-5, 1e-9], rel=1e-7)
    assert d.windowing.window_type == ope.WindowType.FLAT_TOP
    assert d.dispersion.coefficients == pytest.approx([0.0, 0.0, 12.5, -3.25])
    assert d.background_removal.rolling_average_window_size == 32
    assert d.post_processing.bscan_flip and d.post_processing.fixed_pattern_noise_bscan_count == 7
    np.testing.assert_array_equal(d.get_custom_window_curve(), np.linspace(0, 1, 2048, dtype=np.float32))
    assert not d.load_from_file(str(tmp_path / "missing.ini"))


def test_processor_without_device(ope, tmp_path):
    p = ope.Processor(ope.Backend.B200)
    assert p.get_backend() == ope.Backend.B200 and "B200" in repr(p)
    p.set_input_parameters(1024, 256, 1, ope.DataType.UINT16)
    cfg = p.config
    assert cfg.data.signal_length == 1024 and cfg.data.samples_per_buffer == 1024 * 256
    # simple setters land in the configuration before initialization
    p.set_grayscale_range(5.0, 80.0)
    p.enable_bscan_flip(True)
    p.set_resampling_coefficients([1.0, 2.0, 3.0, 4.0])
    p.set_dispersion_coefficients([0.0, 0.0, 1.0, 2.0], 0.5)
    p.set_window_parameters(ope.WindowType.GAUSS, 0.4, 0.9)
    c = p.config
    assert (c.post_processing.grayscale_min, c.post_processing.grayscale_max) == (5.0, 80.0)
    assert c.post_processing.bscan_flip and c.resampling.coefficients == [1.0, 2.0, 3.0, 4.0]
    assert c.dispersion.factor == 0.5 and c.windowing.window_type == ope.WindowType.GAUSS
    with pytest.raises(RuntimeError):
        p.use_custom_resampling_curve(True)  # nothing set yet
    with pytest.raises(ValueError):
        p.set_fixed_pattern_noise_bscan_count(0)
    # callbacks
    ids = [p.add_output_callback(lambda a: None) for _ in range(3)]
    assert p.get_callback_count() == 3
    assert p.remove_output_callback(ids[1]) and not p.remove_output_callback(ids[1])
    assert p.get_callback_count() == 2
    p.set_callback(lambda a: None)
    assert p.get_callback_count() == 1
    p.clear_output_callbacks()
    assert p.get_callback_count() == 0
    # profiles before initialization live in the configuration
    assert not p.has_fixed_pattern_noise_profile()
    assert not p.has_post_process_background_profile()
    bg = np.linspace(0, 1, 512, dtype=np.float32)
    p.set_post_process_background_profile(bg)
    assert p.has_post_process_background_profile()
    np.testing.assert_array_equal(p.get_post_process_background_profile(), bg)
    path = str(tmp_path / "bg.csv")
    p.save_post_process_background_profile_to_file(path)
    with open(path) as f:
        lines = f.read().splitlines()
    assert lines[0] == "Sample Number;Sample Value" and lines[1] == "0;0" and len(lines) == 513
    q = ope.Processor(ope.Backend.B200)
    q.set_input_parameters(1024, 256, 1, ope.DataType.UINT16)
    q.load_post_process_background_profile_from_file(path)
    np.testing.assert_allclose(q.get_post_process_background_profile(), bg, rtol=1e-5)
    with pytest.raises(ope.ConfigurationError):
        q.load_fixed_pattern_noise_profile_from_file(path)  # one value per line, and not initialized
    with pytest.raises(ope.BufferError):
        p.set_fixed_pattern_noise_profile(np.ones(5, dtype=np.float32))
    with pytest.raises(ope.BufferError):
        p.process(np.zeros(16, dtype=np.uint16))  # not a view of an IOBuffer
    # the configuration file round trip goes through the Processor too
    cfg_path = str(tmp_path / "p.ini")
    p.save_config(cfg_path)
    q.load_config(cfg_path)
    assert q.config.post_processing.grayscale_max == 80.0
    with pytest.raises(ope.ConfigurationError):
        q.load_config(str(tmp_path / "nope.ini"))


def test_single_backend_build_selects_b200_only(ope):
    """libope_host.so holds the B200 backend alone: Backend::CPU and
    Backend::CUDA (the reference library's own backends) are refused with an
    argument error naming the backend, never silently replaced; the reference
    library built with the Backend::B200 patch holds all three
    (tests/test_dropin.py)."""
    for b, name in ((ope.Backend.CPU, "CPU"), (ope.Backend.CUDA, "CUDA")):
        with pytest.raises(ValueError, match=name):
            ope.Processor(b)
    p = ope.Processor(ope.Backend.B200)
    with pytest.raises(ValueError):
        p.set_backend(ope.Backend.CPU)
    assert p.get_backend() == ope.Backend.B200


def test_initialize_without_device_raises(ope):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    p = ope.Processor(ope.Backend.B200)
    p.set_input_parameters(1024, 64, 1, ope.DataType.UINT16)
    with pytest.raises(ope.InitializationError):
        p.initialize()
    assert p.get_next_available_buffer is not None


def test_host_library_exports():
    B.build()
    nm = shutil.which("nm")
    if not nm:
        pytest.skip("nm not available")
    out = subprocess.run([nm, "-DC", "--defined-only", B.HOST_LIB], capture_output=True, text=True).stdout
    for sym in ["ope::Processor::Processor(ope::Backend)", "ope::Processor::process(ope::IOBuffer&)",
                "ope::Processor::getNextAvailableInputBuffer()", "ope::Processor::addOutputCallback",
                "ope::ProcessorConfiguration::saveToFile", "ope::IOBuffer::allocateMemory(unsigned long)",
                "ope::getDataTypeBitDepth(ope::DataType)", "ope::Processor::setFixedPatternNoiseProfile"]:
        assert sym in out, sym
    ctypes.CDLL(B.HOST_LIB)


from oracle.reflib import REFERENCE_TREE  # noqa: E402  (named by the environment or the oracle build)

REF_EXAMPLE = os.path.join(REFERENCE_TREE or "/nonexistent", "examples", "example_basic.cpp")


@pytest.mark.skipif(not os.path.exists(REF_EXAMPLE), reason="reference sources not present")
def test_reference_example_builds_against_headers(tmp_path):
    """The reference's example program compiles and links, unmodified, against
    include/ope and libope_host.so (it selects Backend::CUDA, which this
    single-backend build refuses at run time; the build and link are checked)."""
    B.build()
    exe = str(tmp_path / "example_basic")
    cmd = ["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include", "ope"), REF_EXAMPLE, "-o", exe,
           "-L", B.LIBDIR, "-lope_host", "-lope_b200", "-Wl,-rpath," + B.LIBDIR, "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
