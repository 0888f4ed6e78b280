"""Acceptance runs on the stated configurations, through the C ABI.

* the 64 x 16 x 65 plain DNS (ceiling dipole A = 0.3, fringe, 3/2-rule products,
  Re_delta* = 500, dt = 0.01): 100 steps against the FP64 oracle with the dense z
  operator (the device's linear map), u, v, w, p each within 1e-10 relative L2;
* the 256 x 64 x 129 dynamic-Smagorinsky LES: whole FP64 steps against the oracle;
* the 128 x 4 x 97 Orr-Sommerfeld test (Re_delta* = 1000, alpha delta* = 0.25): 500 steps
  in FP64 and in the mixed form, the perturbation energy per step against the oracle and
  <dE/dt> against the Orr-Sommerfeld omega_i (lintest, src/orrsomm.f90:566-622);
* a long dynamic-Smagorinsky LES (128 x 32 x 65, 2000 steps) in both forms: finite fields
  and spanwise mean / rms profiles (u + ubar, v, w averaged over y and over the second
  half of the run, as run/spanwiseavg.m averages q snapshots) of the mixed form within
  1e-4 of the FP64 ones.
"""
import os

import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import ic
from lsbflow_b200 import linstab as L
from lsbflow_b200.config import workload
from oracle import lsb_oracle as O

pytestmark = pytest.mark.gpu

TOL_STEP = 1e-10
TOL_OS_MIXED = 5e-6


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def device(cfg, u, v, w, nsteps):
    from lsbflow_b200 import lib
    st = hs.make_setup(cfg)
    s = lib.Solver(st)
    try:
        s.upload(u, v, w, dt=st.dt)
        s.step(nsteps)
        return s.download()
    finally:
        s.close()


def oracle(st, u, v, w, nsteps, zder="dense"):
    old, oldw = O.ZDER, O.WORKERS
    O.ZDER, O.WORKERS = zder, os.cpu_count() or 1
    try:
        ost = O.State.zeros_like(st, u, v, w, st.dt)
        for _ in range(nsteps):
            O.timestep(st, ost)
        return ost
    finally:
        O.ZDER, O.WORKERS = old, oldw


def test_dns64_100_steps_against_oracle():
    cfg = workload("dns64")
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 7, 1e-3)
    got = device(cfg, u, v, w, 100)
    ost = oracle(st, u, v, w, 100)
    for key, ref in (("uf", ost.uf), ("vf", ost.vf), ("wf", ost.wf), ("pf", ost.pf)):
        assert rel(got[key], ref) < TOL_STEP, (key, rel(got[key], ref))
    assert got["istep"] == 100


def test_les256_steps_against_oracle():
    cfg = workload("les256")
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 1000, 5e-3)
    nsteps = 3
    got = device(cfg, u, v, w, nsteps)
    ost = oracle(st, u, v, w, nsteps)
    for key, ref in (("uf", ost.uf), ("vf", ost.vf), ("wf", ost.wf), ("pf", ost.pf)):
        assert rel(got[key], ref) < TOL_STEP, (key, rel(got[key], ref))


def os_run(cfg, nsteps):
    from lsbflow_b200 import lib
    st = hs.make_setup(cfg)
    z = np.zeros((st.grid.nzp, cfg.ny, cfg.nx))
    uf, vf, wf = z.copy(), z.copy(), z.copy()
    mode = L.setup_linstab(st, uf, vf, wf)
    s = lib.Solver(st)
    e = []
    try:
        s.upload(uf, vf, wf, dt=st.dt)
        for _ in range(nsteps):
            s.step(1)
            e.append(s.diag()["energy_pert"])
    finally:
        s.close()
    return st, mode, (uf, vf, wf), np.array(e)


def test_os128_500_steps_fp64_and_mixed():
    nsteps = 500
    cfg = workload("os128")
    st, mode, (uf, vf, wf), dev = os_run(cfg, nsteps)
    ost = O.State.zeros_like(st, uf, vf, wf, st.dt)
    ref = []
    for _ in range(nsteps):
        O.timestep(st, ost)
        ref.append(O.lintest(st, ost)[1])
    ref = np.array(ref)
    assert np.max(np.abs(dev - ref) / ref) < 1e-9
    gd = L.mean_growth(L.growth_rates(dev, st.dt))
    go = L.mean_growth(L.growth_rates(ref, st.dt))
    assert abs(gd - go) < 1e-6 * abs(go), (gd, go)
    assert mode.omega.imag > 0 and abs(gd - mode.omega.imag) < 5e-3 * mode.omega.imag, (gd, mode.omega.imag)
    # the mixed form from the same mode: its growth rate against the FP64 device run's
    # (measured 2.0e-6 relative: the FP32 transforms of a 1e-5 perturbation on a unit mean
    # flow; held to 5e-6)
    _, _, _, mix = os_run(cfg.replace(precision=1), nsteps)
    gm = L.mean_growth(L.growth_rates(mix, st.dt))
    assert abs(gm - gd) < TOL_OS_MIXED * abs(gd), (gm, gd)


def long_run(cfg, u, v, w, nsteps, every=20):
    from lsbflow_b200 import lib
    st = hs.make_setup(cfg)
    s = lib.Solver(st)
    acc_m = acc_r = None
    n = 0
    try:
        s.upload(u, v, w, dt=st.dt)
        done = 0
        while done < nsteps:
            s.step(every)
            done += every
            if done > nsteps // 2:
                m, r = s.spanwise_stats()
                acc_m = m if acc_m is None else acc_m + m
                acc_r = r if acc_r is None else acc_r + r
                n += 1
        d = s.diag()
        final = s.download()
    finally:
        s.close()
    return acc_m / n, acc_r / n, d, final


def test_long_dynamic_les_profiles_2000_steps():
    cfg = workload("ens128", sgsmodel=1)
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 1000, 5e-3)
    m0, r0, d0, f0 = long_run(cfg, u, v, w, 2000)
    m1, r1, d1, f1 = long_run(cfg.replace(precision=1), u, v, w, 2000)
    for d, f in ((d0, f0), (d1, f1)):
        assert d["nonfinite"] == 0
        assert all(np.isfinite(f[k]).all() for k in ("uf", "vf", "wf", "pf"))
        assert d["umax"] < 2.0
    for q in range(3):  # u + ubar, v, w
        assert rel(m1[q], m0[q]) < 1e-4, ("mean", q, rel(m1[q], m0[q]))
        assert rel(r1[q], r0[q]) < 1e-4, ("rms", q, rel(r1[q], r0[q]))
