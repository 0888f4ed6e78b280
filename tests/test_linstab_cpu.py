"""Orr-Sommerfeld set-up and the linear growth test on the CPU, pinned to the reference's
shipped linear-stability sweep (run/output_lintest.txt, run/energy.dat via the golden
fixture).  The oracle steps the injected mode with the restated timestep()."""
import os

import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import linstab as L
from oracle import lsb_oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_run.npz"))
CASES = GOLD["os_cases"]          # Re_d, x0, alpha*, cguess_r, omega_r, omega_i, dt, nsteps
TABLE = GOLD["os_energy_table"]   # Re, alpha*, omega_i, <dE/dt>, err%


def half_ulp6(v):
    """Half a unit in the 6th significant digit: the rounding of the log's G14.6 output."""
    return 0.5 * 10.0 ** (np.floor(np.log10(abs(v))) - 5)


def test_case_grid_matches_log():
    for c in CASES:
        cfg = L.sweep_case(c[0], c[2], c[3])
        assert abs(cfg.x0 - c[1]) < 1e-9 * c[1]
        st = hs.make_setup(cfg)
        # the log prints dt with 6 significant digits
        assert abs(st.dt - c[6]) <= half_ulp6(c[6]), (c[:3], st.dt, c[6])


def test_os_matrix_boundary_rows():
    st = hs.make_setup(L.sweep_case(1805.0, 0.5))
    a, b = L.os_matrices(st, st.grid.alpha)
    nzp = st.grid.nzp
    n = nzp + 2
    assert a.shape == (n, n)
    assert np.all(b[[0, 1, 2, n - 2], :][:, :nzp] == 0)
    assert a[0, 0] == 1 and np.count_nonzero(a[0]) == 1       # psi = 0 at the ceiling
    assert np.allclose(a[1, :nzp], st.d[nzp - 1])             # d psi / dz at the wall
    assert a[2, nzp - 1] == 1 and b[2, n - 2] == 1 / st.grid.alpha


# The iteration's restarts draw random numbers (from /dev/urandom in the reference), and
# the OS operator at nzp = 65 is ill-conditioned (|A| ~ 1e11): the final omega carries the
# iteration's noise.  Below Re_d = 3000 that noise is < 3e-6; above, near-neutral modes
# (Re 4055 / 4805 at alpha* = 0.5) wander by up to 1.2e-3.
def _omega_tol(re_d):
    return 5e-6 if re_d < 3000 else 2e-3


@pytest.mark.parametrize("i", range(len(CASES)))
def test_iterated_omega_matches_log(i):
    c = CASES[i]
    st = hs.make_setup(L.sweep_case(c[0], c[2], c[3]))
    m = L.os_mode(st, all_eigenvalues=False)
    ref = complex(c[4], c[5])
    assert abs(m.omega - ref) / abs(ref) < _omega_tol(c[0]), (c[:3], m.omega, ref)
    # energy.dat's omega_i (6 digits) is the same number
    assert abs(m.omega.imag - TABLE[i, 2]) <= half_ulp6(TABLE[i, 2]) + _omega_tol(c[0]) * abs(ref)


def test_mode_normalisation_and_divergence():
    st = hs.make_setup(L.sweep_case(2555.0, 0.85))
    m = L.os_mode(st, all_eigenvalues=False)
    z = st.grid.zpts
    e = L.mode_energy(m.uvec, z) + L.mode_energy(m.vvec, z) + L.mode_energy(m.wvec, z)
    assert abs(e - 1e-10) < 1e-22
    # i alpha u + dw/dz = 0 for u = D psi, w = -i alpha psi
    div = 1j * m.alphax * m.uvec + st.d @ m.wvec
    assert np.abs(div).max() < 1e-12 * np.abs(m.uvec).max()


def run_lintest(cfg, nsteps=None):
    st = hs.make_setup(cfg)
    z = np.zeros((st.grid.nzp, cfg.ny, cfg.nx))
    uf, vf, wf = z.copy(), z.copy(), z.copy()
    mode = L.setup_linstab(st, uf, vf, wf)
    s = O.State.zeros_like(st, uf, vf, wf, st.dt)
    en = []
    for _ in range(nsteps or cfg.nsteps):
        O.timestep(st, s)
        en.append(O.lintest(st, s)[1])
    return st, mode, np.array(en), uf, vf, wf


# <dE/dt> of the sweep: the DNS of the reference reproduces omega_i to 0.04%-10%
# (err% column); the restated step lands within 1e-5 (absolute) of the reference's own
# <dE/dt> on every case.  The sweep's input.dat is not shipped, so this pin is approximate.
@pytest.mark.parametrize("i", [0, 7, 12, 18, 22])
def test_growth_rate_matches_energy_dat(i):
    c = CASES[i]
    st, mode, en, *_ = run_lintest(L.sweep_case(c[0], c[2], c[3]))
    g = L.mean_growth(L.growth_rates(en, st.dt))
    assert abs(g - TABLE[i, 3]) < 1.0e-5, (c[:3], g, TABLE[i, 3])
    assert abs(g - mode.omega.imag) < 1.0e-5
