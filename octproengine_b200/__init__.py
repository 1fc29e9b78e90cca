"""B200 (sm_100a) backend for the OCTproEngine per-A-scan processing chain.

Layers:
  * ``capi``   -- ctypes binding of the C ABI (include/ope_b200.h), the drop-in boundary;
  * ``chain``  -- ChainSpec (ProcessorConfiguration fields) and context set-up with generated curves;
  * ``synth``  -- seeded synthetic spectra for tests and benchmarks;
  * ``build``  -- in-tree build of the native libraries;
  * ``reference_api()`` -- the ``octproengine`` Python module (the reference's
    Processor API over this backend).
"""
import importlib
import os
import sys

__version__ = "0.1.0"

LIBDIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")


def reference_api():
    """Imports and returns the built ``octproengine`` module (``import octproengine``)."""
    if LIBDIR not in sys.path:
        sys.path.insert(0, LIBDIR)
    try:
        return importlib.import_module("octproengine")
    except ImportError as e:
        raise ImportError("octproengine module not built: run `python -m octproengine_b200.build`") from e
