"""The C ABI boundary without a GPU: every symbol include/*.h declares is
exported by the library and bound in capi.py; configuration errors are
reported as status codes before any device work; the curve generators of the
library are bit-identical to the oracle restatement."""
import ctypes
import os
import re

import numpy as np
import pytest

from octproengine_b200 import capi
from oracle import restate as R

HEADER_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_symbols():
    names = []
    for f in sorted(os.listdir(HEADER_DIR)):
        if f.endswith(".h"):
            txt = open(os.path.join(HEADER_DIR, f)).read()
            names += re.findall(r"OPE_B200_API\s+[^;(]*?\b(ope_b200_\w+)\s*\(", txt)
    return names


def test_header_declares_entry_points():
    names = declared_symbols()
    assert len(names) >= 25
    assert "ope_b200_process_device" in names and "ope_b200_create" in names


@pytest.mark.parametrize("name", declared_symbols())
def test_symbol_exported_and_bound(name):
    lib = ctypes.CDLL(capi.LIB_PATH)
    assert hasattr(lib, name)
    assert name in capi.SIGNATURES


def test_abi_version():
    assert capi.lib().ope_b200_abi_version() == 1


@pytest.mark.parametrize("field,value,code", [
    ("signal_length", 0, capi.E_INVALID),
    ("ascans_per_bscan", -3, capi.E_INVALID),
    ("signal_length", 1000, capi.E_UNSUPPORTED),   # not a power of two
    ("signal_length", 16384, capi.E_UNSUPPORTED),
    ("input_dtype", 10, capi.E_UNSUPPORTED),       # FLOAT64
    ("fpn_bscan_count", 0, capi.E_INVALID),
])
def test_invalid_configuration_rejected(field, value, code):
    cfg = capi.default_config()
    setattr(cfg, field, value)
    h = ctypes.c_void_p()
    rc = capi.lib().ope_b200_create(ctypes.byref(cfg), ctypes.byref(h))
    assert rc == code and not h.value


def test_dc_removal_window_must_be_positive():
    cfg = capi.default_config()
    cfg.dc_removal_enabled = 1
    cfg.dc_window = 0
    h = ctypes.c_void_p()
    assert capi.lib().ope_b200_create(ctypes.byref(cfg), ctypes.byref(h)) == capi.E_INVALID


def test_default_config_matches_reference_defaults():
    """ProcessorConfiguration defaults (include/processorconfiguration.h:49-171)."""
    c = capi.default_config()
    assert (c.signal_length, c.ascans_per_bscan, c.bscans_per_buffer, c.input_dtype) == (1024, 512, 1, 2)
    assert (c.dc_window, c.log_scaling, c.grayscale_min, c.grayscale_max) == (64, 1, 30.0, 100.0)
    assert (c.addend, c.multiplicator, c.fpn_bscan_count, c.bg_weight, c.bg_offset) == (0.0, 1.0, 1, 1.0, 0.0)


@pytest.mark.parametrize("n", [256, 1000, 2048, 4096])
@pytest.mark.parametrize("coeffs", [(0.5, 2048.0, -100.0, 50.0), (0.0, 1.0, 0.0, 0.0), (3.0, 900.0, 40.0, -7.0)])
def test_resampling_curve_bit_exact(n, coeffs):
    assert np.array_equal(capi.generate_resampling_curve(n, coeffs), R.resampling_curve(n, coeffs))


@pytest.mark.parametrize("n", [512, 2048, 3000])
def test_dispersion_phase_and_cos_sin_bit_exact(n):
    coeffs = (0.1, -2.0, 7.0, -3.0)
    ph = capi.generate_dispersion_phase(n, coeffs)
    assert np.array_equal(ph, R.dispersion_phase(n, coeffs))
    cs = capi.phase_to_cos_sin(ph)
    c, s = R.phase_to_cos_sin(ph)
    assert np.array_equal(cs[0::2], c) and np.array_equal(cs[1::2], s)


@pytest.mark.parametrize("wtype", range(6))
@pytest.mark.parametrize("n,center,fill", [(512, 0.5, 0.95), (2048, 0.9, 0.85), (1000, 0.1, 0.5), (4096, 1.3, 1.2)])
def test_window_curve_bit_exact(wtype, n, center, fill):
    assert np.array_equal(capi.generate_window_curve(n, wtype, center, fill), R.window_curve(n, wtype, center, fill))
