"""Test oracle for the OCT A-scan chain. TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may import anything from this package, and only as the checker:
nothing in ``octproengine_b200`` imports it and no product path routes through
it.

Contents:
  * ``restate``  -- a numpy restatement of the reference CPU chain
    (``src/backends/cpu/cpu_kernels.tpp``, ``cpu_backend.cpp:169-357``,
    ``src/core/processorconfiguration.cpp:438-589``, ``processor.cpp:77-99``):
    float32 arithmetic in the reference's evaluation order for every stage
    before the FFT, the inverse DFT in float64, and an all-float64 "truth" mode.
  * ``reflib``   -- ctypes access to ``_ref/libope_cpu_ref.so``, the reference's
    own ``CpuBackend`` compiled out of tree (``Makefile``) against a
    project-written FFTW-API shim (``fftw_shim/``). FFT = project shim, not FFTW.

Parity pin: the restatement is checked against the reference library and
against the committed golden fixtures in ``tests/golden/`` that were produced by
the reference library (``tests/golden/make_golden.py``).
"""
