"""Extract the golden vectors of the reference's shipped run (run/ directory) into
``reference_run.npz``.  Run in a checkout where the reference tree is available:

    python tests/golden/make_golden.py /path/to/lsbflow

What is extracted (all from the reference's run/ folder):
* grid.dat   : nx, ny, nzp, (x0, xl, xlen, ylen, zlen), xpts, ypts, zpts, gf
* paral.dat  : ubar, ubarp, ubarpp, wbar, wbarp, wbarpp
* output.txt : the 31 interior-D2 eigenvalues (7 digits), the blasfl iteration
               count, the initial dt, the Blasius table columns
* prev_q00001.dat / prev_q00002.dat (float32 snapshots after 10 and 20 steps of
  the input.dat run): headers, the u profile at (x1, y1), and the maximum
  deviations of u from that profile and of |v|, |w|, |p| over the whole grid
* input.dat  : copied as text (the namelist of that run)
* energy.dat : the Orr-Sommerfeld sweep table (Re, alpha*, omega_i, <dE/dt>, err%)
* output_lintest.txt : per case of that sweep the header (Re_d, x0, alpha*, Re(cguess)),
               the last omega of the inverse iteration (10 digits), the final dt
               and the number of time steps
"""
import os
import re
import struct
import sys

import numpy as np


def records(fn):
    b = open(fn, "rb").read()
    i, out = 0, []
    while i < len(b):
        n = struct.unpack("<i", b[i:i + 4])[0]
        out.append(b[i + 4:i + 4 + n])
        i += 8 + n
    return out


def read_q(fn):
    b = np.fromfile(fn, "<f4")
    pre = b[:7].copy()
    nx, ny, nzp, nypl = (int(x) for x in pre[3:7])
    res = nx * ny * nzp
    out = []
    for v in range(5):
        a = b[7 + v * res:7 + (v + 1) * res]
        g = np.empty((nzp, ny, nx), np.float32)
        for r in range(ny // nypl):
            blk = a[r * nx * nypl * nzp:(r + 1) * nx * nypl * nzp].reshape(nypl, nzp, nx)
            g[:, r * nypl:(r + 1) * nypl, :] = blk.transpose(1, 0, 2)
        out.append(g)
    return pre, out


def main(ref):
    run = os.path.join(ref, "run")
    d = {}
    g = records(os.path.join(run, "grid.dat"))
    d["grid_dims"] = np.frombuffer(g[0], "<i4").copy()
    d["grid_params"] = np.frombuffer(g[1], "<f8").copy()
    for name, rec in zip(["xpts", "ypts", "zpts", "gf"], g[2:6]):
        d[name] = np.frombuffer(rec, "<f8").copy()
    p = records(os.path.join(run, "paral.dat"))
    for name, rec in zip(["ubar", "ubarp", "ubarpp", "wbar", "wbarp", "wbarpp"], p[1:7]):
        d[name] = np.frombuffer(rec, "<f8").copy()
    txt = open(os.path.join(run, "output.txt")).read()
    ev = txt.split("eigenvalues =")[1].split("max iter")[0]
    d["eig_d2"] = np.array([float(l.split(",")[0]) for l in ev.strip().splitlines()])
    d["blasfl_iters"] = np.array(int(re.search(r"converged at iter=\s*(\d+)", txt).group(1)))
    d["dt0"] = np.array(float(re.search(r"dt=\s*([0-9.Ee+-]+)", txt).group(1)))
    tab = txt.split("zpts, ubar, ubarp, ubarpp, wbar, tbar =")[1].split("based input")[0]
    rows = [[float(x) for x in l.replace(" ", "").rstrip(",").split(",")] for l in tab.strip().splitlines()]
    d["blasius_table"] = np.array(rows)
    for step, fn in ((10, "prev_q00001.dat"), (20, "prev_q00002.dat")):
        pre, q = read_q(os.path.join(run, fn))
        u, v, w, temp, pp = q
        prof = u[:, 0, 0].astype(np.float64)
        d[f"q{step}_header"] = pre
        d[f"q{step}_uprof"] = prof
        d[f"q{step}_udev"] = np.array(np.abs(u - u[:, :1, :1]).max())
        d[f"q{step}_vmax"] = np.array(np.abs(v).max())
        d[f"q{step}_wmax"] = np.array(np.abs(w).max())
        d[f"q{step}_pmax"] = np.array(np.abs(pp).max())
    d["input_dat"] = np.array(open(os.path.join(run, "input.dat")).read())
    en = open(os.path.join(run, "energy.dat")).read().strip().splitlines()[1:]
    d["os_energy_table"] = np.array([[float(x) for x in l.strip().rstrip(",").split(",")] for l in en])
    lt = open(os.path.join(run, "output_lintest.txt")).read()
    cases = []
    for blk in lt.split(" Re_d =")[1:]:
        h = re.match(r"\s*([-\d.Ee+]+)\s*, x0 =\s*([-\d.Ee+]+)\s*, astar =\s*([-\d.Ee+]+)\s*, "
                     r"cguess = \(\s*([-\d.Ee+]+)", blk)
        sec = blk.split("solving for most unstable eigenvalue")[1].split("time reqd")[0]
        it = re.findall(r"\n\s+\d+,\s*([-\d.Ee+]+)\s*,\s*([-\d.Ee+]+)\s*,", sec)[-1]
        dt = float(re.search(r"final time step dt =\s*([-\d.Ee+]+)", blk).group(1))
        nst = float(re.search(r"# of its performed =\s*(\d+)", blk).group(1))
        cases.append([float(x) for x in h.groups()] + [float(it[0]), float(it[1]), dt, nst])
    d["os_cases"] = np.array(cases)  # Re_d, x0, alpha*, cguess_r, omega_r, omega_i, dt, nsteps
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_run.npz")
    np.savez_compressed(out, **d)
    print("wrote", out, os.path.getsize(out), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/lsbflow")
    main(sys.argv[1])
