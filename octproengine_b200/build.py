"""Builds the native libraries of the B200 backend in-tree.

* ``lib/libope_b200.so`` -- the CUDA chain kernels (sm_100a) and the C ABI
  declared in ``include/ope_b200.h``; compiled with nvcc for
  ``-gencode arch=compute_100a,code=sm_100a``.
* ``lib/libope_host.so`` -- the C++ host layer (ope::Processor,
  ope::ProcessorConfiguration, ope::IOBuffer, ope::B200Backend) on top of the C
  ABI, for C++ callers of the reference API.
* ``lib/octproengine<EXT_SUFFIX>`` -- the Python module ``octproengine`` (the
  reference's Python API) over the host layer; import it with ``lib`` on
  ``sys.path`` or through ``octproengine_b200.reference_api()``.

Objects are rebuilt only when a source or any header of the package is newer.
Run ``python -m octproengine_b200.build`` (or ``__graft_entry__.build()``).
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys
import sysconfig

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
PYBIND = os.path.join(PKG, "pybind")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")

CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "-Xcompiler", "-ffp-contract=off", "-diag-suppress", "128",
    "-I", INCLUDE,
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-pthread", "-I", INCLUDE,
             "-I", os.path.join(CUDA_HOME, "include")]

CHAIN_LIB = os.path.join(LIBDIR, "libope_b200.so")
HOST_LIB = os.path.join(LIBDIR, "libope_host.so")
PY_MODULE = os.path.join(LIBDIR, "octproengine" + (sysconfig.get_config_var("EXT_SUFFIX") or ".so"))


def _headers(d: str):
    return glob.glob(os.path.join(d, "*.h")) + glob.glob(os.path.join(d, "*.cuh")) + \
        glob.glob(os.path.join(INCLUDE, "*.h")) + glob.glob(os.path.join(INCLUDE, "ope", "*.h"))


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, verbose=False):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed ({r.returncode}): {' '.join(cmd)}\n{r.stdout}")
    return r.stdout


def build_chain(jobs: int = 0, verbose: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")) + glob.glob(os.path.join(CSRC, "*.cpp")))
    hdrs = _headers(CSRC)
    todo = []
    objs = []
    for s in srcs:
        o = os.path.join(OBJDIR, os.path.basename(s) + ".o")
        objs.append(o)
        if _stale(o, [s] + hdrs):
            todo.append((s, o))
    jobs = jobs or max(1, min(len(todo), os.cpu_count() or 4))
    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = [ex.submit(_run, [NVCC] + NVCC_FLAGS + ["-c", s, "-o", o], verbose) for s, o in todo]
            for f in futs:
                f.result()
    if todo or _stale(CHAIN_LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", CHAIN_LIB] + objs +
             ["-lpthread"], verbose)
    return CHAIN_LIB


def build_host(verbose: bool = False) -> str:
    srcs = sorted(glob.glob(os.path.join(HOST, "*.cpp")))
    if not srcs:
        return ""
    deps = srcs + _headers(HOST) + [CHAIN_LIB]
    if _stale(HOST_LIB, deps):
        cxx = shutil.which("g++") or "g++"
        _run([cxx] + CXX_FLAGS + ["-shared", "-o", HOST_LIB] + srcs +
             ["-L", LIBDIR, "-lope_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return HOST_LIB


def build_python_module(verbose: bool = False) -> str:
    srcs = sorted(glob.glob(os.path.join(PYBIND, "*.cpp")))
    if not srcs:
        return ""
    try:
        import pybind11
    except ImportError as e:  # pragma: no cover - pybind11 ships with the image
        raise RuntimeError("pybind11 is required to build the octproengine Python module") from e
    deps = srcs + _headers(HOST) + [HOST_LIB]
    if _stale(PY_MODULE, deps):
        cxx = shutil.which("g++") or "g++"
        _run([cxx] + CXX_FLAGS + ["-fvisibility=hidden", "-shared", "-I", pybind11.get_include(),
                                  "-I", sysconfig.get_paths()["include"], "-o", PY_MODULE] + srcs +
             ["-L", LIBDIR, "-lope_host", "-lope_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    return PY_MODULE


def build(verbose: bool = False) -> None:
    if not os.path.exists(NVCC):
        raise RuntimeError(f"nvcc not found at {NVCC}")
    build_chain(verbose=verbose)
    build_host(verbose=verbose)
    build_python_module(verbose=verbose)


if __name__ == "__main__":
    build(verbose="-v" in sys.argv)
    print(CHAIN_LIB)
