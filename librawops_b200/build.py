"""Builds the sm_100a shared library of the render path, in tree.

    python -m librawops_b200.build            # -> librawops_b200/_lib/librawengine_b200.so

nvcc compiles every csrc/*.cu for sm_100a (no fast-math: the IEEE division,
rounding and powf semantics are part of the parity contract), g++ compiles the
host-only csrc/*.cpp (the C++ drop-in surface of include/rawengine/, C++20),
and one shared library is linked that exports the C ABI of
include/rawengine_b200.h and the rawengine:: classes.  Objects are rebuilt
only when a source or header is newer than the library.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
OUT_DIR = os.path.join(PKG, "_lib")
LIB = os.path.join(OUT_DIR, "librawengine_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
HOST_CXX = "g++"
CUDA_INCLUDE = os.path.join(os.path.dirname(os.path.dirname(NVCC)), "include")
CXX_FLAGS = ["-std=c++20", "-O2", "-g", "-fPIC", "-fvisibility=hidden", "-Wall", "-Wextra",
             "-Wno-unused-parameter", "-I", os.path.join(ROOT, "include"), "-I", CSRC,
             "-I", CUDA_INCLUDE]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def _sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _host_sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cpp")))


def _deps():
    return _sources() + _host_sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h")) + \
        glob.glob(os.path.join(ROOT, "include", "rawengine", "*.hpp"))


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in _deps())


def build(verbose: bool = False, force: bool = False) -> str:
    if not force and not stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs = []
    procs = []
    for src in _sources():
        obj = os.path.join(OUT_DIR, os.path.basename(src)[:-3] + ".o")
        cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    for src in _host_sources():
        obj = os.path.join(OUT_DIR, os.path.basename(src)[:-4] + ".host.o")
        cmd = [HOST_CXX, *CXX_FLAGS, "-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
    failed = False
    for src, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode or (src.endswith(".cpp") and out):
            sys.stderr.write(out.decode())
        failed |= p.returncode != 0
    if failed:
        raise RuntimeError("nvcc failed")
    cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
