"""Build and run oracle/cpu_step.cpp, the C++/OpenMP restatement of the reference's time
step that times the CPU baseline (test infrastructure: only tests/, __graft_entry__ and the
bench's CPU-baseline leg and reference arm use it).

    python -m oracle.cpu_baseline          # builds oracle/cpu_step with g++ -O3 -fopenmp
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "cpu_step.cpp")
BIN = os.path.join(HERE, "cpu_step")
HEADER = os.path.join(ROOT, "include", "lsbgpu.h")


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles cpu_step (native code for the host it runs on: -march=native is left out so
    that the binary built here also runs on the GPU box's host)."""
    if (not force and os.path.exists(BIN) and os.path.getmtime(BIN) >= os.path.getmtime(SRC)
            and os.path.getmtime(BIN) >= os.path.getmtime(HEADER)):
        return BIN
    # the first compiler that builds it with OpenMP (a $CXX toolchain may lack libgomp)
    err = None
    for cxx in ("/usr/bin/g++", "g++", os.environ.get("CXX")):
        if not cxx:
            continue
        cmd = [cxx, "-O3", "-std=c++17", "-fopenmp", "-Wall", "-Wextra", "-I", os.path.join(ROOT, "include"), SRC,
               "-o", BIN]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode == 0:
            return BIN
        err = r.stderr
    raise RuntimeError(f"cpu_step does not build: {err}")


def run(st, u, v, w, nsteps: int, threads: int, want_state: bool = True):
    """Steps the seeded velocity ``nsteps`` times with ``threads`` OpenMP threads; returns the
    stepping time in seconds and (``want_state``) u, v, w, p after the last step."""
    from lsbflow_b200 import lib

    exe = build()
    c = st.cfg
    shape = (c.nzp, c.ny, c.nx)
    with tempfile.TemporaryDirectory() as d:
        setup = os.path.join(d, "setup.bin")
        state = os.path.join(d, "state.bin")
        out = os.path.join(d, "out.bin")
        lib.write_setup_file(setup, st)
        with open(state, "wb") as f:
            for a in (u, v, w):
                f.write(np.ascontiguousarray(a, dtype="<f8").tobytes())
            f.write(np.array([st.dt], dtype="<f8").tobytes())
        args = [exe, setup, str(st.nx_lg), str(st.ny_lg), state, str(nsteps), str(threads)]
        if want_state:
            args.append(out)
        res = subprocess.run(args, check=True, capture_output=True, text=True)
        sec = float(res.stdout.split("seconds")[1].split()[0])
        if not want_state:
            return sec, None
        raw = np.fromfile(out, dtype="<f8")
        n = int(np.prod(shape))
        fields = {k: raw[i * n:(i + 1) * n].reshape(shape) for i, k in enumerate(("uf", "vf", "wf", "pf"))}
        return sec, fields


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
