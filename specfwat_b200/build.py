"""Compile the CUDA solver into ``specfwat_b200/libsem_b200.so`` (sm_100a).

The library is built in-tree with nvcc; the Python package loads it from
there.  ``python -m specfwat_b200.build`` rebuilds it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libsem_b200.so")
SOURCES = ["sem_api.cu", "sem_kernels.cu", "sem_noalloc.cu", "sem_probe.cu", "sem_smooth.cu",
           "sem_measure.cu", "sem_precond.cu", "sem_grid.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


HOST_LIB = os.path.join(HERE, "host", "libspecfwat_host.so")


def build_host(verbose: bool = False) -> str:
    """The C++ host side (``host/prepare_fwd.cpp``, the PrepareFWD driver
    over the C ABI) as ``host/libspecfwat_host.so``, linked against the
    CUDA library beside it."""
    cxx = shutil.which("g++") or "g++"
    cmd = [cxx, "-std=c++17", "-O2", "-fPIC", "-shared", "-Wall",
           "-I", os.path.join(ROOT, "include"),
           os.path.join(HERE, "host", "prepare_fwd.cpp"),
           "-L", HERE, "-l:libsem_b200.so", "-Wl,-rpath,$ORIGIN/..", "-o", HOST_LIB]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return HOST_LIB


def build(verbose: bool = False, extra=()) -> str:
    srcs = [os.path.join(HERE, "csrc", s) for s in SOURCES]
    cmd = [nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17",
           "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr",
           "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(HERE, "csrc"),
           *extra, "-o", LIB, *srcs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    build_host(verbose)
    return LIB


if __name__ == "__main__":
    build(verbose=True, extra=sys.argv[1:])
