"""Build libvh.so (the CUDA step and its C ABI) in-tree for sm_100a.

    python -m viral_b200.build [--verbose]

The library is written next to this file (viral_b200/libvh.so) so that it
travels with the repository snapshot; nothing is installed.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libvh.so")
CHECK_LIB = os.path.join(HERE, "libvh_check.so")

SOURCES = ["vh_api.cu", "vh_static.cu", "vh_batch.cu", "vh_adjoint.cu", "vh_adjoint3.cu", "vh_cgc.cu", "vh_inputs.cpp", "vh_io.cpp",
           "vh_freezeout.cpp", "vh_freezeout_dev.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def build_check(verbose: bool = False) -> str:
    """libvh_check.so: host entry points onto the device arithmetic (tests)."""
    src = os.path.join(CSRC, "vh_check.cu")
    deps = [src] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh")]
    if os.path.exists(CHECK_LIB) and all(os.path.getmtime(d) <= os.path.getmtime(CHECK_LIB) for d in deps):
        return CHECK_LIB
    cmd = [nvcc(), *ARCH, "-O2", "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"),
           "-I", CSRC, "-o", CHECK_LIB, src]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed building libvh_check.so")
    return CHECK_LIB


DRIVER = os.path.join(HERE, "vh_run")


def build_driver(verbose: bool = False) -> str:
    """vh_run: the C++ host driver (the reference's main loop over the C ABI)."""
    src = os.path.join(HERE, "host", "vh_run.cpp")
    deps = [src, LIB, os.path.join(ROOT, "include", "vh.h")]
    if os.path.exists(DRIVER) and all(os.path.getmtime(d) <= os.path.getmtime(DRIVER) for d in deps):
        return DRIVER
    cmd = ["g++", "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"), src, "-L", HERE, "-lvh",
           "-Wl,-rpath,$ORIGIN", "-o", DRIVER]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("g++ failed building vh_run")
    return DRIVER


def build(verbose: bool = False, extra: list[str] | None = None) -> str:
    srcs = [os.path.join(CSRC, s) for s in SOURCES]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "vh.h")]
    if os.path.exists(LIB) and not extra:
        t = os.path.getmtime(LIB)
        if all(os.path.getmtime(d) <= t for d in deps):
            return LIB
    cmd = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-I", os.path.join(ROOT, "include"), "-I", CSRC, "-o", LIB, *srcs]
    if verbose:
        cmd += ["-Xptxas", "-v"]
    if extra:
        cmd += extra
    r = subprocess.run(cmd, capture_output=True, text=True)
    if verbose or r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed building libvh.so")
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv)
    build_check(verbose="--verbose" in sys.argv)
    build_driver(verbose="--verbose" in sys.argv)
    print(LIB)
