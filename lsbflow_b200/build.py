"""Builds the CUDA library ``liblsbgpu.so`` in-tree for sm_100a with nvcc, and the native
driver ``lsb_run`` (host C++ over the library's C ABI) with g++.

    python -m lsbflow_b200.build          # incremental (object files under _build/)
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "liblsbgpu.so")
DRIVER_SRC = os.path.join(HERE, "driver", "lsb_run.cpp")
DRIVER = os.path.join(HERE, "lsb_run")
CXX = os.environ.get("CXX", "g++")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-I", INCLUDE, "-I", CSRC]


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    objs = []
    for src in _sources():
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if (not force and os.path.exists(obj) and os.path.getmtime(obj) >= os.path.getmtime(src)
                and os.path.getmtime(obj) >= hdr_mtime):
            continue
        cmd = [NVCC, *ARCH, *FLAGS, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    if force or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    build_driver(verbose=verbose, force=force)
    return LIB


def build_driver(verbose: bool = False, force: bool = False) -> str:
    """lsb_run, linked against the in-tree library (found next to the binary at run time)."""
    deps = [DRIVER_SRC, LIB] + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    if not force and os.path.exists(DRIVER) and os.path.getmtime(DRIVER) >= max(os.path.getmtime(d) for d in deps):
        return DRIVER
    cmd = [CXX, "-std=c++17", "-O2", "-Wall", "-Wextra", "-I", INCLUDE, DRIVER_SRC, "-L", HERE, "-llsbgpu",
           "-Wl,-rpath,$ORIGIN", "-o", DRIVER]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return DRIVER


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
