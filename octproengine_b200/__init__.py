"""B200 (sm_100a) backend for the OCTproEngine per-A-scan processing chain.

Layers:
  * ``capi``   -- ctypes binding of the C ABI (include/ope_b200.h), the drop-in boundary;
  * ``chain``  -- ChainSpec (ProcessorConfiguration fields) and context set-up with generated curves;
  * ``synth``  -- seeded synthetic spectra for tests and benchmarks;
  * ``build``  -- in-tree build of the native libraries.
"""
__version__ = "0.1.0"
