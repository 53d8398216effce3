"""In-tree build of the native parts of gprat_b200.

    python -m gprat_b200.build          # or: from gprat_b200.build import build_all

Produces (next to the sources, so they travel with the tree):
  gprat_b200/lib/libgprat_cuda.so  CUDA kernels + C ABI (include/gprat_cu.h), sm_100a
  gprat_b200/lib/libgprat.so       C++ mirror of the reference host API (gprat::GP, ...)
  gprat_b200/gprat*.so             pybind11 module `gprat` (the reference's Python API)

Rebuilds a target only when one of its inputs is newer.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig
from typing import List

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
INCLUDE = os.path.join(ROOT, "include")
CSRC = os.path.join(PKG, "csrc")
CPP = os.path.join(PKG, "cpp")
LIB = os.path.join(PKG, "lib")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.path.dirname(os.path.dirname(NVCC))
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CUDA_LIB = os.path.join(LIB, "libgprat_cuda.so")
HOST_LIB = os.path.join(LIB, "libgprat.so")


def _ext_suffix() -> str:
    return sysconfig.get_config_var("EXT_SUFFIX") or ".so"


PY_MODULE = os.path.join(PKG, "gprat" + _ext_suffix())


def _stale(target: str, inputs: List[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(i) > t for i in inputs)


def _run(cmd: List[str], verbose: bool) -> None:
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_cuda(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(LIB, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(INCLUDE, "*.h")))
    if not force and not _stale(CUDA_LIB, sources + headers + [__file__]):
        return CUDA_LIB
    objdir = os.path.join(PKG, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    procs = []
    for src in sources:
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        objs.append(obj)
        if not force and not _stale(obj, [src] + headers + [__file__]):
            continue
        cmd = [NVCC, *ARCH, "-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC,
               "--expt-relaxed-constexpr", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((src, subprocess.Popen(cmd)))
    for src, p in procs:
        if p.wait() != 0:
            raise RuntimeError(f"nvcc failed on {src}")
    _run([NVCC, *ARCH, "-shared", "-o", CUDA_LIB, *objs, "-lcudart"], verbose)
    return CUDA_LIB


def build_host(verbose: bool = False, force: bool = False) -> str:
    """C++ mirror of the reference host API, linked against libgprat_cuda.so."""
    os.makedirs(LIB, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CPP, "*.cpp")))
    sources = [s for s in sources if not os.path.basename(s).startswith("py_")]
    headers = sorted(glob.glob(os.path.join(INCLUDE, "gprat", "*.hpp")) + glob.glob(os.path.join(INCLUDE, "*.h")))
    if not sources:
        return HOST_LIB
    if not force and not _stale(HOST_LIB, sources + headers + [CUDA_LIB, __file__]):
        return HOST_LIB
    cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-I", INCLUDE, "-I", os.path.join(INCLUDE, "gprat"), "-I", CPP, "-I",
           os.path.join(CUDA_HOME, "include"), *sources, "-o", HOST_LIB, "-L", LIB, "-lgprat_cuda",
           "-Wl,-rpath,$ORIGIN", "-L", os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-pthread"]
    _run(cmd, verbose)
    return HOST_LIB


def build_python(verbose: bool = False, force: bool = False) -> str:
    """pybind11 module `gprat` (the reference's Python API) over libgprat.so."""
    import pybind11

    sources = sorted(glob.glob(os.path.join(CPP, "py_*.cpp")))
    headers = sorted(glob.glob(os.path.join(INCLUDE, "gprat", "*.hpp")))
    if not sources:
        return PY_MODULE
    if not force and not _stale(PY_MODULE, sources + headers + [HOST_LIB, __file__]):
        return PY_MODULE
    py_inc = sysconfig.get_paths()["include"]
    cmd = ["g++", "-std=c++20", "-O2", "-fPIC", "-shared", "-I", INCLUDE, "-I", os.path.join(INCLUDE, "gprat"), "-I", CPP, "-I", pybind11.get_include(),
           "-I", py_inc, *sources, "-o", PY_MODULE, "-L", LIB, "-lgprat", "-lgprat_cuda", "-Wl,-rpath,$ORIGIN/lib",
           "-pthread"]
    _run(cmd, verbose)
    return PY_MODULE


def build_all(verbose: bool = False, force: bool = False) -> None:
    build_cuda(verbose, force)
    build_host(verbose, force)
    build_python(verbose, force)


if __name__ == "__main__":
    build_all(verbose=True, force="--force" in sys.argv)
