"""The Orr-Sommerfeld linear test on the device: the injected mode stepped by lsb_step,
its perturbation energy taken by lsb_diag every step (lintest, src/orrsomm.f90:566-622),
against the FP64 oracle stepping the same mode.

Tolerances: per-step perturbation energies 1e-9 relative; the mean growth rate <dE/dt>
1e-6 relative to the oracle's.  The growth rate against the Orr-Sommerfeld omega_i is
the physics check (the reference's own sweep lands at 0.04%-10%)."""
import os

import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import linstab as L
from lsbflow_b200.config import workload
from oracle import lsb_oracle as O

pytestmark = pytest.mark.gpu

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_run.npz"))


def device_and_oracle(cfg, nsteps):
    from lsbflow_b200 import lib
    st = hs.make_setup(cfg)
    z = np.zeros((st.grid.nzp, cfg.ny, cfg.nx))
    uf, vf, wf = z.copy(), z.copy(), z.copy()
    mode = L.setup_linstab(st, uf, vf, wf)
    s = lib.Solver(st)
    s.upload(uf, vf, wf, dt=st.dt)
    dev = []
    for _ in range(nsteps):
        s.step(1)
        dev.append(s.diag()["energy_pert"])
    s.close()
    ost = O.State.zeros_like(st, uf, vf, wf, st.dt)
    ref = []
    for _ in range(nsteps):
        O.timestep(st, ost)
        ref.append(O.lintest(st, ost)[1])
    return st, mode, np.array(dev), np.array(ref)


def test_sweep_case_growth_on_device():
    c = GOLD["os_cases"][0]
    st, mode, dev, ref = device_and_oracle(L.sweep_case(c[0], c[2], c[3]), int(c[7]))
    assert np.max(np.abs(dev - ref) / ref) < 1e-9
    gd = L.mean_growth(L.growth_rates(dev, st.dt))
    go = L.mean_growth(L.growth_rates(ref, st.dt))
    assert abs(gd - go) < 1e-6 * abs(go), (gd, go)
    assert abs(gd - GOLD["os_energy_table"][0, 3]) < 1e-5


def test_os128_growth_on_device():
    # Re_d* = 1000, alpha d* = 0.25: an unstable Tollmien-Schlichting wave
    cfg = workload("os128")
    st, mode, dev, ref = device_and_oracle(cfg, 200)
    assert mode.omega.imag > 0
    assert np.max(np.abs(dev - ref) / ref) < 1e-9
    gd = L.mean_growth(L.growth_rates(dev, st.dt))
    go = L.mean_growth(L.growth_rates(ref, st.dt))
    assert abs(gd - go) < 1e-6 * abs(go), (gd, go)
    assert abs(gd - mode.omega.imag) < 5e-3 * abs(mode.omega.imag), (gd, mode.omega.imag)
