"""Host-side FP64 set-up of one LSBFLOW run.

Everything here runs once per run on the host and produces *inputs* of the
device time step, exactly as the reference passes grid arrays, the Chebyshev
matrices and the Helmholtz eigenbasis (diag, smat, simat) to its hot path:

* ``setup_grid``       -- src/init.f90:130-273 (mappings 0-3; dx = xlen/(nx-1) while
                          alpha = 2 pi/xlen, kept as in the reference)
* ``cheb_d``           -- src/chebyshev.f90:9-159 closed-form Gauss-Lobatto D, D2 = D.D
* ``dct_diff_matrix``  -- src/chebyshev.f90:204-270 (the DCT-I derivative used for
                          nz > 31) written as the dense matrix it applies per column
* ``diagonalize``      -- src/helmholtz.f90:13-126 (eig of D2(2:nz,2:nz), E^-1 by LU)
* ``blasfl``           -- src/init.f90:497-586 Newton iteration for the Blasius profile
* ``setup_ic``         -- src/init.f90:296-494, ic = 0 branch
* ``fringe_lambda``    -- src/navierstokes.f90:92-186 lambda(x) of ``force`` (ftype 1)
* ``lift_functions``   -- src/helmholtz.f90:239-307 (hbot, htop and their 2nd derivatives)
* ``dealias_sizes``    -- src/dealiasing.f90:133-154 with nproch = 1

LAPACK's dggev/dgetri/dgesv are replaced by numpy's LAPACK-backed eig/inv/solve:
the eigenbasis only enters through E diag E^-1, whose product is independent of
eigenvector scaling and ordering.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import scipy.fft

from .config import LsbConfig

PI = 4.0 * math.atan(1.0)
TWOPI = 8.0 * math.atan(1.0)


@dataclass
class Grid:
    nx: int
    ny: int
    nz: int
    nzp: int
    xpts: np.ndarray
    ypts: np.ndarray
    zpts: np.ndarray
    gf: np.ndarray
    xi: np.ndarray
    wavx: np.ndarray      # (nx,) interleaved: wavx[2i] = wavx[2i+1] = i*alpha
    wavy: np.ndarray      # (ny,) FFT order
    alpha: float
    beta: float
    dx: float
    dy: float
    xl: float
    aa: float
    bb: float
    xlen: float
    ylen: float
    zlen: float
    x0: float


def setup_grid(cfg: LsbConfig) -> Grid:
    """Restates setup_grid (src/init.f90:130-273) for one process (myid = 0)."""
    nx, ny, nz = cfg.nx, cfg.ny, cfg.nz
    nzp = nz + 1
    xlen, ylen, zlen, x0 = cfg.xlen, cfg.ylen, cfg.zlen, cfg.x0
    if cfg.linstab >= 1:  # src/init.f90:147-150
        xlen = TWOPI * 6.02 * math.sqrt(cfg.xnu * cfg.x0 / cfg.u0) / cfg.astar
        ylen = xlen
    dx = xlen / (nx - 1.0)
    xpts = x0 + np.arange(nx) * dx
    dy = ylen / (ny - 1.0)
    ypts = np.arange(ny) * dy
    alpha = TWOPI / xlen
    wavx = np.repeat(np.arange(nx // 2) * alpha, 2)
    beta = TWOPI / ylen
    wavy = np.zeros(ny)
    nyh = ny // 2
    for j in range(1, nyh + 1):
        wavy[ny - j] = -j * beta
        wavy[j - 1] = (j - 1.0) * beta
    zpts = np.zeros(nzp)
    gf = np.zeros(nzp)
    xi = np.zeros(nzp)
    aa = bb = 0.0
    k = np.arange(1, nzp + 1, dtype=np.float64)
    if cfg.mapping == 0:
        xl = zlen
        xi = xl / 2.0 * np.cos(PI * (k - 1.0) / nz)
        zpts = xi.copy()
        gf = np.ones(nzp)
    elif cfg.mapping == 1:
        xl = 1.0
        aa = 1.0
        bb = 1.875 * math.sqrt(cfg.xnu * x0 / cfg.u0)
        xi[1:] = xl / 2.0 * (1.0 + np.cos(PI * (k[1:] - 1.0) / nz))
        zpts[1:] = bb * xi[1:] / (aa - xi[1:])
        gf[1:] = (aa - xi[1:]) ** 2.0 / (bb * aa)
        xi[0] = 1.0
        zpts[0] = 1.0e20
        zlen = zpts[0]
        gf[0] = 0.0
    elif cfg.mapping == 2:
        xl = 1.0
        bb = 1.875 * math.sqrt(cfg.xnu * (x0 + cfg.blfac * xlen) / cfg.u0)
        aa = 1.0 + bb / zlen
        xi = xl / 2.0 * (1.0 + np.cos(PI * (k - 1.0) / float(nz)))
        zpts = bb * xi / (aa - xi)
        gf = (aa - xi) ** 2.0 / (aa * bb)
    elif cfg.mapping == 3:
        xl = zlen
        xi = xl / 2.0 * np.cos(PI * (k - 1.0) / float(nz))
        zpts = xl / 2.0 + xi
        gf = np.ones(nzp)
    else:
        raise ValueError("mapping must be 0..3")
    return Grid(nx, ny, nz, nzp, xpts, ypts, zpts, gf, xi, wavx, wavy, alpha, beta,
                dx, dy, xl, aa, bb, xlen, ylen, zlen, x0)


def _ff(i: int, nr: int) -> float:
    v = nr * 0.5 / math.tan(PI * i / (2.0 * nr)) if i != 0 else 0.0
    if i % 2 == 0:
        v = -v
    if i == 0:
        v = 0.0
    return v


def _den(kr: int, jr: int, nr: int) -> float:
    d = nr * math.sin(PI * kr / nr)
    if jr == 0 or jr == nr:
        d *= 2.0
    if kr == 0:
        d = 0.5 * nr
        if jr % 2 == 1:
            d = -d
        if jr == 0 or jr == nr:
            d = 1.0
    return d


def _xnum(kr: int, jr: int, nr: int) -> float:
    if kr == 0:
        if jr == 0:
            return (1.0 / 3.0) * nr * nr + 1.0 / 6.0
        if jr == nr:
            return -0.5 if nr % 2 == 1 else 0.5
        return (0.5 * (nr + 0.5) * ((nr + 0.5) + (1.0 / math.tan(PI * jr / (2.0 * nr))) ** 2)
                + 1.0 / 8.0 - 0.25 / (math.sin(PI * jr / (2.0 * nr)) ** 2.0) - 0.5 * nr * nr)
    return _ff(kr + jr, nr) + _ff(kr - jr, nr)


def _del(k: int, j: int, n: int, xl: float) -> float:
    kr, jr, nr, fac = k - 1, j - 1, n - 1, 1.0
    if kr == nr:
        kr, jr, fac = 0, nr - jr, -1.0
    return fac * _xnum(kr, jr, nr) / _den(kr, jr, nr) * (2.0 / xl)


def cheb_d(grid: Grid):
    """build_cheb_zder_matrix (src/chebyshev.f90:9-48): returns dor, d, d2."""
    n = grid.nzp
    dor = np.empty((n, n))
    for i in range(n):
        for j in range(n):
            dor[i, j] = _del(i + 1, j + 1, n, grid.xl)
    d = dor * grid.gf[:, None]
    d2 = d @ d
    return dor, d, d2


def dct_diff_apply(y: np.ndarray, gf: np.ndarray, xl: float, p: int) -> np.ndarray:
    """dct_diff (src/chebyshev.f90:204-270) along the last axis of ``y``.

    FFTW's REDFT00 is scipy's unnormalised DCT-I.
    """
    n = y.shape[-1]
    half = 0.5 * xl
    nlog = 2 * (n - 1)
    beta = np.array(y, dtype=np.float64, copy=True)
    for _ in range(p):
        alpha = scipy.fft.dct(beta, type=1, axis=-1)
        alpha[..., 1:n - 1] = alpha[..., 1:n - 1] / half
        beta = np.zeros_like(alpha)
        beta[..., n - 2] = 2.0 * (n - 1.0) * alpha[..., n - 1]
        for k in range(n - 1, 1, -1):  # Fortran k = n-1 .. 2 ; beta(k-1)=beta(k+1)+2(k-1)alpha(k)
            beta[..., k - 2] = beta[..., k] + 2.0 * (k - 1.0) * alpha[..., k - 1]
        out = scipy.fft.dct(beta, type=1, axis=-1)
        beta = out * gf / nlog
    return beta


def dct_diff_matrix(grid: Grid, p: int) -> np.ndarray:
    """The linear map of dct_diff(p) as an (nzp, nzp) matrix: column j = map(e_j)."""
    eye = np.eye(grid.nzp)
    return dct_diff_apply(eye, grid.gf, grid.xl, p).T.copy()


def diagonalize(d2int: np.ndarray):
    """diagonalize_matrix (src/helmholtz.f90:13-126): lam, E, E^-1 of D2 interior."""
    lam, e = np.linalg.eig(d2int)
    if np.max(np.abs(lam.imag)) > 0:
        raise RuntimeError("complex eigenvalues in the Chebyshev D2 interior block")
    lam = lam.real.copy()
    e = e.real.copy()
    ei = np.linalg.inv(e)
    return lam, e, ei


def blasfl(eps, itmax, alph, zpts, dor, d, d2):
    """Newton solve of the Blasius equation (src/init.f90:497-586)."""
    nzp = zpts.shape[0]
    nzpp = nzp + 1
    f = (-1.0 + np.exp(-zpts * alph)) / alph
    d3 = d2 @ d
    rat = 1.0 / (1.0 + zpts)
    it_conv = None
    for ii in range(1, itmax + 1):
        rhs = d2 @ f
        A = np.zeros((nzpp, nzpp))
        A[:nzp, :nzp] = (0.5 * rat * f)[:, None] * d2 + rat[:, None] * d3 + (0.5 * zpts * rat)[:, None] * d2
        A[np.arange(nzp), np.arange(nzp)] += 0.5 * rat * rhs
        A[:nzp, nzpp - 1] = d[:nzp, nzp - 1]
        A[0, :nzp] = dor[0, :nzp]
        A[nzp - 1, :nzp] = 0.0
        A[nzpp - 1, :nzp] = d[nzp - 1, :nzp]
        A[0, nzpp - 1] = 0.0
        A[nzp - 1, nzpp - 1] = 0.0
        A[nzpp - 1, nzpp - 1] = 0.0
        A[nzp - 1, nzp - 1] = 1.0
        temp1 = d3 @ f
        temp2 = d2 @ f
        df = np.zeros(nzpp)
        df[:nzp] = -0.5 * rat * f * temp2 - 0.5 * zpts * rat * temp2 - rat * temp1
        df[0] = 0.0
        df[nzp - 1] = 0.0
        df[nzpp - 1] = 0.0
        df = np.linalg.solve(A, df)
        f = f + df[:nzp]
        err = np.sum(np.abs(df[:nzp]))
        if err <= eps:
            it_conv = ii
            break
    ubar = 1.0 + d @ f
    wbar = 0.5 * (zpts * ubar - (f + zpts))
    return ubar, wbar, it_conv


@dataclass
class Setup:
    cfg: LsbConfig
    grid: Grid
    dor: np.ndarray
    d: np.ndarray
    d2: np.ndarray
    dz1: np.ndarray         # matrix applied by dfdz   (dct_diff p=1 if nz>31 else d)
    dz2: np.ndarray         # matrix applied by d2fdz2 (dct_diff p=2 if nz>31 else d2)
    lam: np.ndarray
    E: np.ndarray
    Ei: np.ndarray
    ubar: np.ndarray
    ubarp: np.ndarray
    ubarpp: np.ndarray
    wbar: np.ndarray
    wbarp: np.ndarray
    wbarpp: np.ndarray
    blasfl_iters: int | None
    dt: float
    nx_lg: int
    ny_lg: int
    lam_x: np.ndarray       # fringe lambda(x), (nx,)
    hbot: np.ndarray
    htop: np.ndarray
    d2hbot: np.ndarray
    d2htop: np.ndarray


def dpdz(grid: Grid, d: np.ndarray, u: np.ndarray, p: int) -> np.ndarray:
    """dpdz (src/derivatives.f90:135-158) on a single column: the DCT path for n > 31,
    else matmul(d, u) applied once whatever p is (the reference's loop re-applies d
    to u, not to the previous result)."""
    if grid.nzp > 31:
        return dct_diff_apply(u, grid.gf, grid.xl, p)
    return d @ u


def dealias_sizes(nx: int, ny: int):
    """nx_lg, ny_lg of setup_dealiasing (src/dealiasing.f90:133-154), nproch = 1."""
    if nx % 2 == 0 and nx % 4 == 0:
        nx_lg = 3 * nx // 2
    elif nx % 3 == 0:
        nx_lg = 5 * nx // 3
    elif nx % 5 == 0:
        nx_lg = 8 * nx // 5
    else:
        nx_lg = 2 * nx
    if ny % 2 == 0:
        ny_lg = 3 * ny // 2
    elif ny % 3 == 0:
        ny_lg = 5 * ny // 3
    elif ny % 5 == 0:
        ny_lg = 8 * ny // 5
    else:
        ny_lg = 2 * ny
    return nx_lg, ny_lg


def fringe_lambda(cfg: LsbConfig, grid: Grid) -> np.ndarray:
    """lambda(x) of force() (src/navierstokes.f90:123-186), ftype = 1."""
    nx = grid.nx
    xpts = grid.xpts
    epsx = 1.0e-5
    sfs = cfg.sfsize * cfg.fsize
    lfs = cfg.lfsize * cfg.fsize
    rfsize = cfg.fsize - sfs - lfs
    dxs = sfs * grid.xlen
    dxl = lfs * grid.xlen
    dxr = rfsize * grid.xlen
    dxf = dxs + dxl + dxr
    kappa = 2.0 * cfg.u0 / dxf * (-math.log(epsx))
    r = np.zeros(nx)
    for i in range(nx):
        eta0 = (xpts[i] - (xpts[nx - 1] - dxf + dxs)) / (dxs / 2.0)
        eta = (xpts[i] - (xpts[nx - 1] - dxl)) / (dxl / 2.5)
        s0 = math.exp(-eta0 ** 2)
        s = math.exp(-eta ** 2)
        if eta0 > 0.0 and eta < 0.0:
            s0 = 1.0
        if eta < 0.0:
            s = 0.0
        if eta >= 0.0:
            s0 = 0.0
        r[i] = kappa * (s0 + s)
    xshift = 0
    for i in range(1, nx // 4 + 1):
        if xpts[i - 1] < xpts[0] + dxl / 1.5:
            xshift = i
    lam = np.zeros(nx)
    if xshift > 1:
        lam[xshift:nx] = r[0:nx - xshift]
        lam[0:xshift] = r[nx - xshift:nx]
    else:
        lam[:] = r
    return lam


def lift_functions(cfg: LsbConfig, grid: Grid, wbar, wbarpp):
    """hbot, htop, d2hbot, d2htop of solve_nhom_helmholtz (src/helmholtz.f90:239-307)."""
    zpts = grid.zpts
    nzp = grid.nzp
    if cfg.mapping == 0:
        width = zpts[0] - zpts[nzp - 1]
        htop = (zpts - zpts[nzp - 1]) / width
        hbot = -(zpts - zpts[0]) / width
        d2htop = np.zeros(nzp)
        d2hbot = np.zeros(nzp)
    elif cfg.mapping == 1:
        bbot = 50.0
        htop = np.zeros(nzp)
        d2htop = np.zeros(nzp)
        hbot = np.exp(-bbot * zpts)
        hbot[0] = 0.0
        d2hbot = bbot ** 2.0 * hbot
    elif cfg.mapping == 2:
        h = zpts[0] - zpts[nzp - 1]
        bbot = 5.0
        hbot = np.exp(-bbot * zpts) - np.exp(bbot * (zpts - 2.0 * h))
        hbot = hbot / (1.0 - math.exp(-2.0 * bbot * h))
        d2hbot = bbot ** 2 * hbot
        htop = wbar / wbar[0]
        htop[nzp - 1] = 0.0
        d2htop = wbarpp / wbar[0]
    else:
        btop = bbot = 50.0
        h = zpts[0] - zpts[nzp - 1]
        hbot = np.exp(-bbot * zpts) - np.exp(bbot * (zpts - 2.0 * h))
        hbot = hbot / (1.0 - math.exp(-2.0 * bbot * h))
        d2hbot = bbot ** 2.0 * hbot
        htop = np.exp(btop * (zpts - h)) * (1.0 - np.exp(-2.0 * btop * zpts))
        htop = htop / (1.0 - math.exp(-2.0 * btop * h))
        d2htop = btop ** 2.0 * htop
    return hbot, htop, d2hbot, d2htop


def make_setup(cfg: LsbConfig) -> Setup:
    """initialize() for nstart = 0 (src/init.f90:91-106), without the field IC."""
    grid = setup_grid(cfg)
    dor, d, d2 = cheb_d(grid)
    if cfg.nz > 31:
        dz1 = dct_diff_matrix(grid, 1)
        dz2 = dct_diff_matrix(grid, 2)
    else:
        dz1, dz2 = d.copy(), d2.copy()
    nz = cfg.nz
    lam, E, Ei = diagonalize(d2[1:nz, 1:nz])
    # setup_ic, ic = 0 branch (src/init.f90:333-424)
    okr = math.sqrt(cfg.x0 * cfg.xnu / cfg.u0)
    bz = grid.zpts / okr
    ubar, wbar, its = blasfl(1.0e-11, 100, 0.33, bz, dor, d * okr, (d * okr) @ (d * okr))
    ubar = cfg.u0 * ubar
    wbar = wbar * math.sqrt(cfg.xnu * cfg.u0 / cfg.x0)
    wbar[0] = wbar[1]
    wbar[-1] = 0.0
    ubarp = dpdz(grid, d, ubar, 1)
    ubarpp = dpdz(grid, d, ubar, 2)
    wbarp = dpdz(grid, d, wbar, 1)
    wbarpp = dpdz(grid, d, wbar, 2)
    # dt from cfl with zero perturbation (src/init.f90:451); setdt gives the same value
    dt = cfg.cfl * grid.dx / max(np.max(np.abs(ubar)), 1.0)
    if cfg.dt_fixed is not None:
        dt = float(cfg.dt_fixed)
    nx_lg, ny_lg = dealias_sizes(cfg.nx, cfg.ny)
    if cfg.dealiasflag != 1:
        nx_lg, ny_lg = cfg.nx, cfg.ny
    lam_x = fringe_lambda(cfg, grid)
    hbot, htop, d2hbot, d2htop = lift_functions(cfg, grid, wbar, wbarpp)
    return Setup(cfg, grid, dor, d, d2, dz1, dz2, lam, E, Ei, ubar, ubarp, ubarpp,
                 wbar, wbarp, wbarpp, its, dt, nx_lg, ny_lg, lam_x, hbot, htop, d2hbot, d2htop)
