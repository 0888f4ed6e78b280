"""Orr-Sommerfeld linear-stability set-up and the energy-growth test (host, FP64).

Restates the reference's linear-stability path:

* ``os_matrices``        -- the generalized eigenproblem A psi = omega B psi of
                            solve_orrsomm (src/orrsomm.f90:150-258): the OS operator on the
                            Gauss-Lobatto points built from d, d2, d4 = d2 d2 and the Blasius
                            profile, with the reference's "membrane wall" boundary rows
                            (n = nzp + 2 unknowns: psi, the wall displacement and its rate).
* ``os_eigenvalues``     -- all eigenvalues (zggevx, :260-296) as (phi, gam) pairs.
* ``os_inverse_iteration``-- the two-sided inverse iteration from the guess
                            omega = alpha*cguess*u0 (:318-500), with its inner/outer
                            convergence tests and its "regression avoided" rule.  The
                            reference's restarts on a bad guess draw from /dev/urandom
                            (:418-428, :480-485); here they draw from a seeded generator.
* ``os_mode``            -- psi -> (u = D psi, v = 0, w = -i alpha psi) normalised to the
                            energy eps with the reference's trapezoid (energy(), :669-682).
* ``setup_linstab``      -- setup_linstab (src/init.f90:589-644): the mode added to the
                            kx = alpha column of the spectral velocities.
* ``growth_rates``       -- lintest (src/orrsomm.f90:566-622): E_n from ener, growth
                            (E_n - E_{n-1}) / (2 E_n dt), and <dE/dt> over steps 2..n
                            (write_linstab_results, :75-76).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.linalg as sla

from .config import LsbConfig
from .hostsetup import Setup

_C0 = 1.0e-40  # c01..c04 of the membrane-wall rows (rigid limit), src/orrsomm.f90:148-151


def reynolds_linstab(cfg: LsbConfig) -> float:
    """Re based on the 99.9% thickness 6.02 sqrt(nu x0 / U) (src/init.f90:609)."""
    return 6.02 * math.sqrt(cfg.xnu * cfg.x0 / cfg.u0) * cfg.u0 / cfg.xnu


def x0_for_re(re_d: float, xnu: float = 0.001, u0: float = 1.0) -> float:
    """x0 of set_linstab_param (src/orrsomm.f90:22)."""
    return re_d ** 2 * xnu / (6.02 ** 2 * u0)


def sweep_case(re_d: float, astar: float, cguess: float = 0.4, **over) -> LsbConfig:
    """One case of the shipped linear-stability sweep (linstab = 2, src/orrsomm.f90:15-31;
    run/energy.dat, run/output_lintest.txt).  The sweep's input.dat is not shipped; its grid
    is inferred from the log: nzp = 65 (67 OS eigenvalues = nzp + 2), nx = 64 (the initial
    dt = cfl*dx printed per case), zlen = 33.3333 / mapping 2 / blfac 8 as in run/input.dat
    (the iterated omega then agrees with the log to ~1e-8), cfl = 0.1, 25 steps, plain
    DNS without fringe or boundary forcing.  ny is immaterial for the 2-D mode."""
    cfg = LsbConfig(nx=64, ny=4, nz=64, linstab=1, astar=astar, x0=x0_for_re(re_d), cguess=complex(cguess, 0.0),
                    zlen=33.3333, mapping=2, blfac=8.0, xnu=0.001, u0=1.0, cfl=0.1, dtadapt=0, nsteps=25,
                    dealiasflag=0, forcing=0, bctype=0, sgsflag=0)
    return cfg.replace(**over)


def os_matrices(st: Setup, alphax: float, betax: float = 0.0):
    """A and B of solve_orrsomm (src/orrsomm.f90:172-257), complex (nzp+2)^2."""
    cfg = st.cfg
    nzp = st.grid.nzp
    n = nzp + 2
    rey = 1.0 / cfg.xnu
    wav2 = alphax ** 2 + betax ** 2
    d, d2 = st.d, st.d2
    d4 = d2 @ d2
    eye = np.eye(nzp)
    a = np.zeros((n, n), dtype=np.complex128)
    b = np.zeros((n, n), dtype=np.complex128)
    a[:nzp, :nzp] = (d4 - 2.0 * wav2 * d2 + wav2 * wav2 * eye
                     - 1j * alphax * rey * (st.ubar[:, None] * (d2 - wav2 * eye) - np.diag(st.ubarpp)))
    b[:nzp, :nzp] = -1j * rey * (d2 - wav2 * eye)
    # wall row of the membrane condition, then the boundary rows (:217-246)
    a[n - 1, :nzp] = -1j * _C0 / (alphax * rey) * (d2[nzp - 1, :] @ d)
    b[[0, 1, 2, n - 2, n - 1], :] = 0.0
    a[[0, 2, n - 2], :] = 0.0
    a[1, :nzp] = d[nzp - 1, :]
    a[0, 0] = 1.0
    a[2, nzp - 1] = 1.0
    b[2, n - 2] = 1.0 / alphax
    a[1, n - 2] = st.ubarp[nzp - 1]
    a[1, n - 1] = 0.0
    a[n - 2, n - 1] = 1.0
    b[n - 2, n - 2] = -1j
    a[n - 1, n - 2] = _C0 + _C0 * wav2 - 1j * wav2 * (_C0 / rey) * (st.ubarp[nzp - 1] / alphax)
    a[n - 1, n - 1] = _C0
    b[n - 1, n - 1] = 1j
    return a, b


def os_eigenvalues(a: np.ndarray, b: np.ndarray):
    """All generalized eigenvalues as the (phi, gam) pairs zggevx returns (omega = phi/gam),
    and the reference's scaled (Re, Im) / |gam| pair (:283-291)."""
    w = sla.eig(a, b, right=False, homogeneous_eigvals=True)
    phi, gam = w[0], w[1]
    ag = np.abs(gam)
    reig = np.where(ag > 0, phi.real / np.where(ag > 0, ag, 1.0), phi.real)
    aeig = np.where(ag > 0, phi.imag / np.where(ag > 0, ag, 1.0), phi.imag)
    return phi, gam, reig, aeig


@dataclass
class InverseIteration:
    omega: complex
    psi: np.ndarray          # (n,) right eigenvector (normalised to sum |psi| = 1)
    history: list            # omega after each outer iteration (as the reference prints)
    restarts: int


def os_inverse_iteration(a: np.ndarray, b: np.ndarray, omega0: complex, alphax: float, iiter: int = 10,
                         it: int = 10, seed: int = 0) -> InverseIteration:
    """The iteration of solve_orrsomm (src/orrsomm.f90:318-500)."""
    n = a.shape[0]
    rng = np.random.default_rng(seed)
    omk = complex(omega0)
    phi = np.ones(n, dtype=np.complex128)
    gam = np.ones(n, dtype=np.complex128)
    btrans = b.conj().T
    history = []
    restarts = 0
    omkp1 = omk
    phikp1, gamkp1 = phi, gam
    for i in range(1, iiter + 1):
        ck = a - omk * b
        residualk_norm = np.sum(np.abs(ck @ phi))
        lu = sla.lu_factor(ck)
        for ii in range(1, it + 1):
            inner_rk_norm = np.sum(np.abs(ck @ phi))
            rhs_phi = sla.lu_solve(lu, b @ phi)
            rhs_gam = sla.lu_solve(lu, btrans @ gam, trans=2)
            phikp1 = rhs_phi / np.sum(np.abs(rhs_phi))
            gamkp1 = rhs_gam / np.sum(np.abs(rhs_gam))
            inner_rkp1_norm = np.sum(np.abs(ck @ phikp1))
            if np.sum(np.abs(phikp1 - phi)) < 5.0e-5 or inner_rkp1_norm < 5.0e-6:
                if inner_rkp1_norm > inner_rk_norm:
                    phikp1, gamkp1 = phi, gam
                phi, gam = phikp1, gamkp1
                break
            if inner_rkp1_norm >= inner_rk_norm and ii < iiter - 1:
                restarts += 1
                r = rng.random(n) + 1j * rng.random(n)
                phikp1 = phi + 0.001 * r
                phikp1 = phikp1 / np.sum(np.abs(phikp1))
                gamkp1 = gam + 0.001 * r
                gamkp1 = gamkp1 / np.sum(np.abs(gamkp1))
            phi, gam = phikp1, gamkp1
        omkp1 = np.vdot(gamkp1, a @ phikp1) / np.vdot(gamkp1, b @ phikp1)
        history.append(complex(omkp1))
        residualkp1_norm = np.sum(np.abs((a - omkp1 * b) @ phikp1))
        if abs(omkp1 - omk) < 1.0e-14 and residualkp1_norm < 1.5e-6:
            if residualkp1_norm >= residualk_norm:
                omkp1, phikp1, gamkp1 = omk, phi, gam
            break
        if abs(omkp1 - omk) < 1.0e-14 and residualkp1_norm > 1.5e-6:
            restarts += 1
            omkp1 = (0.3 + 0.1 * rng.random()) * alphax
        if residualkp1_norm >= residualk_norm:
            omkp1, phikp1, gamkp1 = omk, phi, gam
        omk = omkp1
    return InverseIteration(complex(omkp1), phikp1, history, restarts)


def mode_energy(q: np.ndarray, zpts: np.ndarray) -> float:
    """energy() of src/orrsomm.f90:669-682: a trapezoid over k = 2..nzp-1 of |q|^2, x 2/7."""
    nzp = len(zpts)
    e = 0.0
    for k in range(1, nzp - 1):  # Fortran k = 2..nzp-1
        e = e - 0.5 * (abs(q[k + 1]) ** 2 + abs(q[k]) ** 2) * (zpts[k + 1] - zpts[k])
    return e * 2.0 / 7.0


@dataclass
class OsMode:
    omega: complex
    alphax: float
    uvec: np.ndarray
    vvec: np.ndarray
    wvec: np.ndarray
    eigenvalues: tuple
    iteration: InverseIteration


def os_mode(st: Setup, eps: float = 1.0e-10, alphax: float | None = None, betax: float = 0.0,
            omega0: complex | None = None, all_eigenvalues: bool = True, seed: int = 0) -> OsMode:
    """solve_orrsomm with iglb = -1 as setup_linstab calls it (src/init.f90:600-619)."""
    cfg = st.cfg
    if alphax is None:
        alphax = st.grid.alpha
    if omega0 is None:
        omega0 = alphax * complex(cfg.cguess) * cfg.u0
    a, b = os_matrices(st, alphax, betax)
    eig = os_eigenvalues(a, b) if all_eigenvalues else None
    itr = os_inverse_iteration(a, b, omega0, alphax, seed=seed)
    nzp = st.grid.nzp
    psi = itr.psi[:nzp].copy()
    uvec = st.d @ psi
    wvec = -1j * alphax * psi
    vvec = np.zeros(nzp, dtype=np.complex128)
    zp = st.grid.zpts
    etot = mode_energy(uvec, zp) + mode_energy(vvec, zp) + mode_energy(wvec, zp)
    xnorm = math.sqrt(eps / etot)
    return OsMode(itr.omega, alphax, uvec * xnorm, vvec * xnorm, wvec * xnorm, eig, itr)


def setup_linstab(st: Setup, uf: np.ndarray, vf: np.ndarray, wf: np.ndarray, mode: OsMode | None = None):
    """Adds the mode to the kx = alpha column (spectral index 2, 3 of row ky = 0),
    src/init.f90:624-635.  Fields are spectral [nzp][ny][nx]; returns the mode."""
    if mode is None:
        mode = os_mode(st)
    for f, q in ((uf, mode.uvec), (vf, mode.vvec), (wf, mode.wvec)):
        f[:, 0, 2] += q.real
        f[:, 0, 3] += q.imag
    return mode


def growth_rates(energies: np.ndarray, dts) -> np.ndarray:
    """grow(istep) = (E_n - E_{n-1}) / (2 E_n dt), 0 at the first step (src/orrsomm.f90:605-616)."""
    e = np.asarray(energies, dtype=np.float64)
    dts = np.broadcast_to(np.asarray(dts, dtype=np.float64), e.shape)
    g = np.zeros_like(e)
    g[1:] = 1.0 / (2.0 * e[1:]) * (e[1:] - e[:-1]) / dts[1:]
    return g


def mean_growth(grow: np.ndarray) -> float:
    """avgdedt = sum(grow2) / (nsteps - 1) (src/orrsomm.f90:75)."""
    return float(np.sum(grow) / (len(grow) - 1))
