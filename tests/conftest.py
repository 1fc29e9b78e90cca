"""Shared fixtures. Tests marked ``gpu`` need an sm_100 GPU; all others run on CPU."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an NVIDIA B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def emu():
    """The CPU emulation of the chain kernel (tests/emu)."""
    import helpers
    return helpers.emu_lib()


@pytest.fixture(scope="session")
def reflib():
    """The reference CPU backend built out of tree (oracle/_ref)."""
    from oracle import reflib as R
    if not R.available():
        try:
            R.build()
        except Exception as e:  # pragma: no cover - depends on the machine
            pytest.skip(f"reference oracle not buildable here: {e}")
    if not R.available():
        pytest.skip("reference oracle library not present")
    return R


@pytest.fixture(scope="session")
def refcuda():
    """The reference CUDA backend built out of tree (oracle/_ref), a comparison baseline."""
    from oracle import refcuda as R
    if not R.available():
        try:
            R.build()
        except Exception as e:  # pragma: no cover - depends on the machine
            pytest.skip(f"reference CUDA backend not buildable here: {e}")
    if not R.available():
        pytest.skip("reference CUDA backend library not present")
    return R


@pytest.fixture(scope="session")
def dropin():
    """The reference library built with the Backend::B200 patch (oracle/_ref)."""
    from oracle import dropin as D
    try:
        D.build()
    except Exception as e:  # pragma: no cover - depends on the machine
        pytest.skip(f"drop-in reference library not buildable here: {e}")
    if not D.available():
        pytest.skip("drop-in reference library not present")
    return D


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from octproengine_b200 import capi
    capi.lib()  # fails loudly if the native library is missing
    if not capi.lib().ope_b200_device_supported(0):
        pytest.skip("device 0 is not an sm_100 GPU")
    return torch.device("cuda:0")
