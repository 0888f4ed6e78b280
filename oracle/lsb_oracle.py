"""FP64 CPU oracle of LSBFLOW's per-time-step hot path (test infrastructure only).

This module is the checker the tests, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` compare the CUDA library against.  It is never part
of the product path.  It restates the reference Fortran (one MPI rank, nproch = 1)
in NumPy, routine by routine; each function cites the lines it follows.

Array layout: numpy C order [k, j, i] equals the reference's Fortran (i, j, k):

* spectral fields ``(nzp, ny, nx)`` -- i odd/even = Re/Im of kx = (i//2)*alpha,
  ky in FFT order, k = 0 the ceiling, k = nzp-1 the wall;
* physical fields ``(nzp, ny, nxpp)`` with nxpp = nx + 2 (two pad columns).

Third-party arithmetic: FFTW 3.3.x (r2c/c2r/c2c and REDFT00) is replaced by
numpy/scipy pocketfft; LAPACK by numpy.linalg (set-up only, see hostsetup).
The temperature equation is carried as identically zero: with the reference's
setup_ic (tbar = 0, T = 0, src/init.f90:353-355,429) every temperature term is
exactly 0.0 for all steps, so skipping it changes no bit of u, v, w, p.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import scipy.fft

from lsbflow_b200.hostsetup import Setup

PI = 4.0 * math.atan(1.0)

# z-derivative algorithm for nz > 31: "dct" follows the reference (dct_diff, FFTW
# REDFT00); "dense" applies the same operator as its dense matrix (what the device
# contraction does).  Both are the same linear map; they differ only in rounding.
ZDER = "dct"
# threads used by scipy.fft (the timed CPU baseline sets this to the host's cores)
WORKERS = 1


def _fft(x, axis):
    return scipy.fft.fft(x, axis=axis, workers=WORKERS)


def _ifft(x, axis):
    return scipy.fft.ifft(x, axis=axis, workers=WORKERS)


def _rfft(x, axis):
    return scipy.fft.rfft(x, axis=axis, workers=WORKERS)


def _irfft(x, n, axis):
    return scipy.fft.irfft(x, n=n, axis=axis, workers=WORKERS)


def _zmat(m, f):
    """m (nzp x nzp) applied along axis 0 of f (z, ...)."""
    sh = f.shape
    return (m @ f.reshape(sh[0], -1)).reshape((m.shape[0],) + sh[1:])


# ----------------------------------------------------------------------------- FFTs
def to_complex(af: np.ndarray) -> np.ndarray:
    return af[..., 0::2] + 1j * af[..., 1::2]


def to_real(cf: np.ndarray) -> np.ndarray:
    out = np.empty(cf.shape[:-1] + (2 * cf.shape[-1],))
    out[..., 0::2] = cf.real
    out[..., 1::2] = cf.imag
    return out


def horfft_fwd(a: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """horfft(is=-1) (src/horfft.f90:94-119): x r2c, drop the kx Nyquist, y c2c, /(nx ny)."""
    xh = _rfft(a[..., :nx], axis=-1)[..., : nx // 2]
    c = _fft(xh, axis=-2) * (1.0 / float(nx * ny))
    return to_real(c)


def c2r(X: np.ndarray, n: int) -> np.ndarray:
    """FFTW c2r of n/2+1 modes (imaginary parts of DC and Nyquist ignored), unnormalised."""
    X = np.array(X, dtype=np.complex128, copy=True)
    X[..., 0] = X[..., 0].real
    if X.shape[-1] > n // 2:
        X[..., n // 2] = X[..., n // 2].real
    return _irfft(X, n=n, axis=-1) * n


def horfft_inv(af: np.ndarray, nx: int, ny: int) -> np.ndarray:
    """horfft(is=+1) (src/horfft.f90:121-144): y c2c backward, x c2r; pad columns 0."""
    c = _ifft(to_complex(af), axis=-2) * ny
    full = np.zeros(c.shape[:-1] + (nx // 2 + 1,), dtype=np.complex128)
    full[..., : nx // 2] = c
    out = np.zeros(af.shape[:-1] + (nx + 2,))
    out[..., :nx] = c2r(full, nx)
    return out


def norm(fields, ny: int):
    """norm (src/horfft.f90:153-224) on spectral fields, in place."""
    nyh = ny // 2
    for f in fields:
        f[:, 0, 1] = 0.0
        if ny > 2:
            for j in range(2, nyh + 1):
                jp = ny + 2 - j
                f[:, j - 1, 0] = 0.5 * (f[:, j - 1, 0] + f[:, jp - 1, 0])
                f[:, j - 1, 1] = 0.5 * (f[:, j - 1, 1] - f[:, jp - 1, 1])
            for j in range(2, nyh + 1):
                jp = ny + 2 - j
                f[:, jp - 1, 0] = f[:, j - 1, 0]
                f[:, jp - 1, 1] = -f[:, j - 1, 1]
            f[:, nyh, :] = 0.0


# ------------------------------------------------------------------ derivatives
def dfdx(st: Setup, uf):
    """dfdx (src/derivatives.f90:261-280)."""
    w = st.grid.wavx[0::2]
    out = np.empty_like(uf)
    out[..., 0::2] = -w * uf[..., 1::2]
    out[..., 1::2] = w * uf[..., 0::2]
    return out


def dfdy(st: Setup, uf):
    """dfdy (src/derivatives.f90:283-303)."""
    w = st.grid.wavy[:, None]
    out = np.empty_like(uf)
    out[..., 0::2] = -w * uf[..., 1::2]
    out[..., 1::2] = w * uf[..., 0::2]
    return out


def divuv(st: Setup, uf, vf):
    """divuv (src/derivatives.f90:394-409)."""
    wx = st.grid.wavx[0::2]
    wy = st.grid.wavy[:, None]
    out = np.empty_like(uf)
    out[..., 0::2] = -wx * uf[..., 1::2] - wy * vf[..., 1::2]
    out[..., 1::2] = wx * uf[..., 0::2] + wy * vf[..., 0::2]
    return out


def _dct_diff_z(st: Setup, y, p):
    """dct_diff (src/chebyshev.f90:204-270) along z (axis 0)."""
    g = st.grid
    n = y.shape[0]
    half = 0.5 * g.xl
    nlog = 2 * (n - 1)
    beta = np.array(y, copy=True)
    shape = (n,) + (1,) * (y.ndim - 1)
    gf = g.gf.reshape(shape)
    for _ in range(p):
        alpha = scipy.fft.dct(beta, type=1, axis=0, workers=WORKERS)
        alpha[1:n - 1] = alpha[1:n - 1] / half
        beta = np.zeros_like(alpha)
        beta[n - 2] = 2.0 * (n - 1.0) * alpha[n - 1]
        for k in range(n - 1, 1, -1):
            beta[k - 2] = beta[k] + 2.0 * (k - 1.0) * alpha[k - 1]
        alpha = scipy.fft.dct(beta, type=1, axis=0, workers=WORKERS)
        beta = alpha * gf / nlog
    return beta


def dfdz(st: Setup, uf):
    """dfdz (src/derivatives.f90:112-132): DCT path for nz > 31, else matmul(d, .)."""
    if st.cfg.nz > 31:
        return _dct_diff_z(st, uf, 1) if ZDER == "dct" else _zmat(st.dz1, uf)
    return _zmat(st.d, uf)


def d2fdz2(st: Setup, uf):
    """d2fdz2 (src/derivatives.f90:161-188)."""
    if st.cfg.nz > 31:
        return _dct_diff_z(st, uf, 2) if ZDER == "dct" else _zmat(st.dz2, uf)
    return _zmat(st.d2, uf)


def wav2(st: Setup):
    wx2 = st.grid.wavx ** 2
    wy2 = st.grid.wavy ** 2
    return wx2[None, :] + wy2[:, None]  # (ny, nx)


# ------------------------------------------------------------------ Helmholtz
def solve_helmholtz(st: Setup, rhs, dtnui):
    """solve_helmholtz (src/helmholtz.f90:130-208), n = nzm; rhs in place."""
    nz = st.cfg.nz
    q = rhs[1:nz]                                       # (nzm, ny, nx)
    dfac = -wav2(st) - dtnui                             # (ny, nx)
    trhs = _zmat(st.Ei, q)
    trhs = trhs / (st.lam[:, None, None] + dfac[None])
    q = _zmat(st.E, trhs)
    rhs[1:nz] = q
    rhs[0] = 0.0
    rhs[nz] = 0.0
    return rhs


def solve_nhom_helmholtz(st: Setup, rhs, bc, dtnui):
    """solve_nhom_helmholtz (src/helmholtz.f90:211-358); rhs in place."""
    nzp = st.cfg.nzp
    w2 = wav2(st)
    hb, ht, d2hb, d2ht = st.hbot, st.htop, st.d2hbot, st.d2htop
    for k in range(nzp):
        abot = d2hb[k] + (-w2 - dtnui) * hb[k]
        rhs[k] = rhs[k] - abot * bc[nzp - 1]
        atop = d2ht[k] + (-w2 - dtnui) * ht[k]
        rhs[k] = rhs[k] - atop * bc[0]
    solve_helmholtz(st, rhs, dtnui)
    for k in range(nzp):
        rhs[k] = rhs[k] + hb[k] * bc[nzp - 1] + ht[k] * bc[0]
    return rhs


# ------------------------------------------------------------------ dealiasing
def dealias_product(st: Setup, a, b, layout: str):
    """dealiasing_2d_fftw (src/dealiasing.f90:262-447), nproch = 1.

    layout "ref": the spanwise spectrum is copied to rows 1..ny of the padded array
    and truncated from rows 1..ny (src/dealiasing.f90:329-330,435), as the reference
    does; "correct": negative ky go to the top rows of the padded spectrum.
    """
    nx, ny = st.cfg.nx, st.cfg.ny
    nxl, nyl = st.nx_lg, st.ny_lg
    af = to_complex(horfft_fwd(a, nx, ny))
    bf = to_complex(horfft_fwd(b, nx, ny))

    def pad(cf):
        out = np.zeros(cf.shape[:-2] + (nyl, nxl // 2 + 1), dtype=np.complex128)
        if layout == "ref":
            out[..., :ny, : nx // 2] = cf
        else:
            h = ny // 2
            out[..., :h, : nx // 2] = cf[..., :h, :]
            out[..., nyl - h:, : nx // 2] = cf[..., h:, :]
        out = _ifft(out, axis=-2) * nyl
        return c2r(out, nxl)

    prod = pad(af) * pad(bf)
    xh = _rfft(prod, axis=-1)
    c = _fft(xh, axis=-2) * (1.0 / (float(nxl) * float(nyl)))
    if layout == "ref":
        t = c[..., :ny, : nx // 2]
    else:
        h = ny // 2
        t = np.concatenate([c[..., :h, : nx // 2], c[..., nyl - h:, : nx // 2]], axis=-2)
    return horfft_inv(to_real(t), nx, ny)


# ------------------------------------------------------------------ filters
def specfilter_exp_xy(st: Setup, uf):
    """specfilter_exp_xy with filtery = 1 (src/filters.f90:281-360), incl. the
    magnitude/phase round trip of the reference."""
    c = st.cfg
    g = st.grid
    nxh, nyh = c.nx // 2, c.ny // 2
    akmax = math.sqrt((nxh * g.alpha) ** 2 + (nyh * g.beta) ** 2)
    akc = akmax * c.kc
    ak = np.sqrt(wav2(st)[:, 0::2])                      # (ny, nx/2)
    theta = (np.abs(ak) - akc) / (akmax - akc)
    with np.errstate(invalid="ignore"):
        filt = np.where(np.abs(ak) >= akc, np.exp(-c.filt_amp * np.power(theta, 2 * c.filt_order)), 1.0)
    fr = uf[..., 0::2]
    fi = uf[..., 1::2]
    fmag = np.sqrt(fr * fr + fi * fi)
    nz_ = fmag != 0.0
    with np.errstate(invalid="ignore", divide="ignore"):
        cosc = np.where(nz_, fr / np.where(nz_, fmag, 1.0), 0.0)
        sinc = np.where(nz_, fi / np.where(nz_, fmag, 1.0), 0.0)
        cosc = np.clip(cosc, -1.0, 1.0)
        phase = np.where(sinc >= 0.0, np.arccos(cosc), -np.arccos(cosc))
    fmagf = fmag * filt[None]
    out = np.empty_like(uf)
    out[..., 0::2] = np.where(nz_, fmagf * np.cos(phase), 0.0)
    out[..., 1::2] = np.where(nz_, fmagf * np.sin(phase), 0.0)
    return out


def zfilter_coeffs(st: Setup, a, b):
    """az, bz, cz of filter_q_3pt with interpflag = 1 (src/filters.f90:398-443)."""
    zp = st.grid.zpts
    n = zp.shape[0]
    az = np.zeros(n)
    bz = np.zeros(n)
    cz = np.zeros(n)
    if st.cfg.mapping in (1, 2):
        for k in range(1, n - 1):
            dltm = zp[k] - zp[k - 1]
            dltp = zp[k + 1] - zp[k]
            az[k] = a * 2.0 * dltm / (dltp + dltm)
            bz[k] = a * 2.0 * (1.0 - dltm / dltp) + b
            cz[k] = a * 2.0 * dltm * dltm / (dltp * (dltp + dltm))
        if st.cfg.mapping == 1:
            az[1], bz[1], cz[1] = 0.0, 2.0 * a + b, 0.0
    else:
        m = (n + 1) // 2
        for k in range(2, m):                           # Fortran k = 2..(nzp+1)/2-1
            dltm = zp[k - 1] - zp[k - 2]
            dltp = zp[k] - zp[k - 1]
            az[k - 1] = a * 2.0 * dltm / (dltp + dltm)
            bz[k - 1] = a * 2.0 * (1.0 - dltm / dltp) + b
            cz[k - 1] = a * 2.0 * dltm * dltm / (dltp * (dltp + dltm))
        for k in range(m + 1, n):                       # Fortran k = (nzp+1)/2+1..nzp-1
            dltm = zp[k - 1] - zp[k - 2]
            dltp = zp[k] - zp[k - 1]
            az[k - 1] = a * 2.0 * dltp * dltp / (dltm * (dltm + dltp))
            bz[k - 1] = a * 2.0 * (1.0 - dltp / dltm) + b
            cz[k - 1] = a * 2.0 * dltp / (dltm + dltp)
        az[m - 1], bz[m - 1], cz[m - 1] = a, b, a
    return az, bz, cz


def filter_q_3pt(st: Setup, q, a, b):
    """filter_q_3pt + filtery_q_3pt (src/filters.f90:363-613), one process.

    ``q`` has shape (..., nzp, ny, nxpp); the x pad columns of the result are 0
    (in the reference they hold uninitialised memory that nothing reads).
    """
    nx, ny = st.cfg.nx, st.cfg.ny
    s = 2.0 * a + b
    x = q[..., :nx]
    qh = (a * np.roll(x, 1, axis=-1) + b * x + a * np.roll(x, -1, axis=-1)) / s
    # y: periodic wrap on one process
    if ny > 2:
        qy = (a * np.roll(qh, 1, axis=-2) + b * qh + a * np.roll(qh, -1, axis=-2)) / s
    else:
        qpad = np.concatenate([qh[..., ny - 1:ny, :], qh, qh[..., 0:1, :]], axis=-2)
        qy = (a * qpad[..., 0:ny, :] + b * qpad[..., 1:ny + 1, :] + a * qpad[..., 2:ny + 2, :]) / s
    az, bz, cz = zfilter_coeffs(st, a, b)
    out = np.array(qy, copy=True)
    n = qy.shape[-3]
    for k in range(1, n - 1):
        out[..., k, :, :] = (az[k] * qy[..., k - 1, :, :] + bz[k] * qy[..., k, :, :]
                             + cz[k] * qy[..., k + 1, :, :]) / s
    res = np.zeros(q.shape)
    res[..., :nx] = out
    return res


def modecut(st: Setup, q, a, b):
    """modecutFC (src/filters.f90:617-654): sum of 6 iterated filters with binomial
    coefficients (6, -15, 20, -15, 6, -1)."""
    coef = (6.0, -15.0, 20.0, -15.0, 6.0, -1.0)
    qb = np.zeros_like(q)
    cur = q
    for c in coef:
        cur = filter_q_3pt(st, cur, a, b)
        qb = qb + c * cur
    return qb


# ------------------------------------------------------------------ SGS
def delta_dyn(st: Setup):
    g = st.grid
    zp = g.zpts
    n = zp.shape[0]
    dz = np.empty(n)
    dz[0] = zp[0] - zp[1]
    dz[1:n - 1] = 0.5 * (zp[0:n - 2] - zp[2:n])
    dz[n - 1] = zp[n - 2] - zp[n - 1]
    return (g.dx * g.dy * dz) ** (1.0 / 3.0)


def static_smagorinsky(st: Setup, duidxj):
    """static_smagorinsky (src/sgsterm.f90:39-120).  duidxj[l][m] = du_l/dx_m.

    delta(nzp) is never assigned in the reference; its factor (1-exp(-z+/25)) is 0
    at the wall, so the wall plane gets nu_sgs = 0 for any finite value."""
    g = st.grid
    nx = st.cfg.nx
    xnu = st.cfg.xnu
    zp = g.zpts
    n = zp.shape[0]
    wall = [k for k in range(n) if zp[k] == 0.0 or abs(zp[k]) == 0.5]
    utau = np.zeros(duidxj[0][2].shape[1:])
    for k in wall:
        utau = utau + xnu * duidxj[0][2][k]
    utau = utau / len(wall)
    utau_avg = np.sum(utau[:, :nx]) / (nx * st.cfg.ny)
    utau_avg = math.sqrt(abs(utau_avg))
    zplus = zp * utau_avg / xnu
    sn = np.zeros_like(duidxj[0][0])
    for j in range(3):
        for i in range(3):
            sn = sn + (0.5 * (duidxj[i][j] + duidxj[j][i])) ** 2
    sn = np.sqrt(2.0 * sn)
    delta = np.zeros(n)
    for k in range(1, n - 1):
        dz = (zp[k - 1] - zp[k + 1]) / 2.0
        delta[k] = (g.dx * g.dy * dz) ** (1.0 / 3.0)
    dz = abs(zp[n - 1] - zp[n - 2])
    delta[0] = (g.dx * g.dy * dz) ** (1.0 / 3.0)
    delta[n - 1] = 0.0
    nu = -((st.cfg.CS * delta * (1.0 - np.exp(-zplus / 25.0))) ** 2)[:, None, None] * sn
    return [[nu * 0.5 * (duidxj[i][j] + duidxj[j][i]) for j in range(3)] for i in range(3)]


def dynamic_smagorinsky(st: Setup, ui, uiuj, duidxj):
    """dynamic_smagorinsky (src/sgsterm.f90:123-280)."""
    a, b = st.cfg.a, st.cfg.b
    nx = st.cfg.nx
    delta = delta_dyn(st)[:, None, None]
    cd = 2.0 * delta
    sij = np.array([[0.5 * (duidxj[l][m] + duidxj[m][l]) for m in range(3)] for l in range(3)])
    snorm = np.sqrt(np.sum(2.0 * sij * sij, axis=(0, 1)))
    sijhat = filter_q_3pt(st, sij, a, b)
    snormhat = np.sqrt(np.sum(2.0 * sijhat * sijhat, axis=(0, 1)))
    lij = delta * delta * snorm * sij
    sijhat = cd * cd * snormhat * sijhat
    mij = filter_q_3pt(st, lij, a, b)
    mij = 2.0 * (mij - sijhat)
    uihat = filter_q_3pt(st, np.array(ui), a, b)
    uu = np.array([[uiuj[l][m] for m in range(3)] for l in range(3)])
    lij = filter_q_3pt(st, uu, a, b)
    lij = lij - uihat[:, None] * uihat[None, :]
    numc = np.sum(mij * lij, axis=(0, 1))
    denomc = np.sum(mij * mij, axis=(0, 1))
    ctot = filter_q_3pt(st, numc, 1.0, 1.0)
    cdd = filter_q_3pt(st, denomc, 1.0, 1.0)
    with np.errstate(invalid="ignore", divide="ignore"):
        c = ctot[..., :nx] / cdd[..., :nx]
    c = np.where((c < 0.0) | np.isnan(c), 0.0, c)
    cmax = 0.2 ** 2
    c = np.where(c > cmax, cmax, c)
    ctot[..., :nx] = c
    nu = ctot * delta * delta * snorm
    return [[-2.0 * nu * sij[l, m] for m in range(3)] for l in range(3)]


def sigma_model(st: Setup, duidxj):
    """sigma_model (src/sgsterm.f90:283-423); its debug print has no effect on results."""
    g = st.grid
    nx = st.cfg.nx
    gij = np.array([[duidxj[l][m][..., :nx] for m in range(3)] for l in range(3)])  # (3,3,...)
    G = np.einsum("kl...,km...->lm...", gij, gij)            # G = g^T g
    G2 = np.einsum("lk...,km...->lm...", G, G)
    i1 = G[0, 0] + G[1, 1] + G[2, 2]
    i2 = 0.5 * (i1 ** 2 - (G2[0, 0] + G2[1, 1] + G2[2, 2]))
    i3 = (G[0, 0] * (G[1, 1] * G[2, 2] - G[1, 2] * G[2, 1])
          - G[0, 1] * (G[1, 0] * G[2, 2] - G[1, 2] * G[2, 0])
          + G[0, 2] * (G[1, 0] * G[2, 1] - G[1, 1] * G[2, 0]))
    a1 = i1 ** 2 / 9.0 - i2 / 3.0
    a2 = i1 ** 3 / 27.0 - i1 * i2 / 6.0 + 0.5 * i3
    a1 = np.abs(a1)
    with np.errstate(invalid="ignore", divide="ignore"):
        pre = a2 / np.sqrt(a1) ** 3.0
        a3 = np.where((pre >= 1.0) | np.isnan(pre), 0.0,
                      np.where(pre <= -1.0, PI / 3.0, np.arccos(np.clip(pre, -1.0, 1.0)) / 3.0))
    sq = np.sqrt(a1)
    s1 = np.sqrt(np.abs(i1 / 3.0 + 2.0 * sq * np.cos(a3)))
    s2 = np.sqrt(np.abs(i1 / 3.0 - 2.0 * sq * np.cos(PI / 3.0 + a3)))
    s3 = np.sqrt(np.abs(i1 / 3.0 - 2.0 * sq * np.cos(PI / 3.0 - a3)))
    ds = s3 * (s1 - s2) * (s2 - s3)
    with np.errstate(invalid="ignore", divide="ignore"):
        ds = np.where(s1 != 0.0, ds / np.where(s1 != 0.0, s1, 1.0) ** 2, ds)
    ds = np.where((ds < 0.0) | np.isnan(ds), 0.0, ds)
    zp = g.zpts
    n = zp.shape[0]
    dz = np.empty(n)
    dz[0] = zp[0] - zp[1]
    dz[n - 1] = zp[n - 2] - zp[n - 1]
    dz[1:n - 1] = 0.5 * (zp[0:n - 2] - zp[2:n])
    delta = (g.dx * g.dy * dz) ** (1.0 / 3.0)
    nu = np.zeros(duidxj[0][0].shape)
    nu[..., :nx] = -((1.35 * delta) ** 2)[:, None, None] * ds
    return [[2.0 * nu * 0.5 * (duidxj[l][m] + duidxj[m][l]) for m in range(3)] for l in range(3)]


def interscale_model(st: Setup, ui):
    """interscale_model (src/sgsterm.f90:426-467); tau is not symmetric."""
    a, b = st.cfg.a, st.cfg.b
    u = np.array(ui)
    ub = filter_q_3pt(st, u, a, b)
    ub2 = filter_q_3pt(st, ub, a, b)
    uibuj = ub[:, None] * u[None, :]
    uibujbar = filter_q_3pt(st, uibuj, a, b)
    tau = uibujbar - ub2[:, None] * ub2[None, :] - ub[:, None] * (u[None, :] - ub[None, :])
    return [[tau[l, m] for m in range(3)] for l in range(3)]


def tau_sgs(st: Setup, ui, uiuj, duidxj):
    """tau_sgs (src/sgsterm.f90:10-37); sgsmodel 4 (TNS) gives tau = 0."""
    m = st.cfg.sgsmodel
    if m == 0:
        return static_smagorinsky(st, duidxj)
    if m == 1:
        return dynamic_smagorinsky(st, ui, uiuj, duidxj)
    if m == 2:
        return sigma_model(st, duidxj)
    if m == 3:
        return interscale_model(st, ui)
    z = np.zeros_like(ui[0])
    return [[z for _ in range(3)] for _ in range(3)]


# ------------------------------------------------------------------ forcing, BCs
def force(st: Setup, ui):
    """force (src/navierstokes.f90:92-211): lambda(x) (ubar - u), -lambda v, -lambda w."""
    nx = st.cfg.nx
    lam = np.zeros(nx + 2)
    lam[:nx] = st.lam_x
    ub = st.ubar[:, None, None]
    return [lam * (ub - ui[0]), lam * (0.0 - ui[1]), lam * (0.0 - ui[2])]


def bound(st: Setup, t: float):
    """bound (src/navierstokes.f90:214-355): spectral w BC, only planes k=1, nzp used.

    bctype 3 is the dipole w(x, ceiling) = A (x - xc)/s exp(-((x - xc)/s)^2),
    xc = xpts(1) + bc3_xc; nothing at the wall."""
    c = st.cfg
    g = st.grid
    nx, ny, nzp = c.nx, c.ny, c.nzp
    bc = np.zeros((nzp, ny, nx + 2))
    x = g.xpts
    if c.bctype == 1:
        h = g.zpts[0]
        xloc = 1.0e5 * c.xnu / c.u0
        if x[nx // 2 - 1] < xloc:
            xloc = c.x0 + 3.0 / 7.0 * c.xlen
        xwidth = 0.24 * h
        amp = c.samp * c.u0 / (0.24 * math.sqrt(PI))
        bamp = c.samp / 2.25
        ref_time = c.xlen / c.u0
        if t - c.istartbound <= ref_time:
            s = math.sin(0.5 * PI * (t - c.istartbound) / ref_time) ** 2.0
            amp, bamp = amp * s, bamp * s
        elif t - c.istartbound > ref_time:
            pass
        else:
            amp = bamp = 0.0
        bwidth = xwidth * 2.25
        x1 = x[nx - 1] - 2.0 * bwidth
        eta = (x - xloc) / xwidth
        bc[0, :, :nx] = amp * np.exp(-eta ** 2.0)
        eta0 = (x - x1) / bwidth
        bc[nzp - 1, :, :nx] = bamp * np.exp(-eta0 ** 4.0)
    elif c.bctype == 2:
        A = 0.002 * c.u0
        A_half = 0.0001 * c.u0
        phi = 0.0
        x1 = 1.655e5 * c.xnu / c.u0
        x2 = 1.81e5 * c.xnu / c.u0
        xm = (x1 + x2) / 2.0
        ref_time = c.x0 / c.u0
        omega = 1.24e-4 * ref_time
        lambda_y = 0.151367188 * c.x0
        theta = t - c.istartbound
        for j in range(ny):
            for i in range(nx):
                eta = 0.0
                if x1 <= x[i] <= xm:
                    eta = (x[i] - x1) / (xm - x1)
                if xm <= x[i] <= x2:
                    eta = (x2 - x[i]) / (x2 - xm)
                if x1 <= x[i] <= x2:
                    f = 15.1875 * eta ** 5 - 35.4375 * eta ** 4 + 20.25 * eta ** 3
                    if x[i] > xm:
                        f = -f
                    gg = math.cos(2.0 * PI * g.ypts[j] / lambda_y)
                    bc[nzp - 1, j, i] = A * f * math.sin(omega * theta) + A_half * f * gg * math.cos(omega / 2.0 * theta + phi)
    elif c.bctype == 3:
        xc = x[0] + c.bc3_xc
        e = (x - xc) / c.bc3_s
        bc[0, :, :nx] = c.bc3_amp * e * np.exp(-e * e)
    bcf = horfft_fwd(bc, nx, ny)
    if c.bctype == 1:
        amp_ = bcf[0, 0, 0]
        bamp_ = bcf[nzp - 1, 0, 0]
        bfac = amp_ / bamp_ if bamp_ != 0 else 0.0
        bcf[nzp - 1] = bfac * bcf[nzp - 1]
    return bcf


# ------------------------------------------------------------------ the step
def nlterm_skewsym(st: Setup, uif, return_parts=False):
    """nlterm_skewsym (src/navierstokes.f90:658-855), velocity part."""
    c = st.cfg
    nx, ny = c.nx, c.ny
    du = [[None] * 3 for _ in range(3)]
    for l in range(3):
        du[l][0] = dfdx(st, uif[l])
        du[l][1] = dfdy(st, uif[l])
        du[l][2] = dfdz(st, uif[l])
    dphys = [[horfft_inv(du[l][m], nx, ny) for m in range(3)] for l in range(3)]
    ui = [horfft_inv(uif[m], nx, ny) for m in range(3)]
    ui[0] = ui[0] + st.ubar[:, None, None]
    dphys[0][2] = dphys[0][2] + st.ubarp[:, None, None]
    nlt = [np.zeros_like(ui[0]) for _ in range(3)]
    uiuj = [[None] * 3 for _ in range(3)]
    for l in range(3):
        for m in range(3):
            if c.dealiasflag == 1:
                p = dealias_product(st, ui[m], dphys[l][m], c.dealias_layout)
                nlt[l] = nlt[l] - 0.5 * p
                uiuj[m][l] = dealias_product(st, ui[m], ui[l], c.dealias_layout)
            else:
                nlt[l] = nlt[l] - 0.5 * ui[m] * dphys[l][m]
                uiuj[m][l] = ui[m] * ui[l]
    if c.forcing == 1:
        fi = force(st, ui)
        for l in range(3):
            nlt[l] = nlt[l] + fi[l]
    if c.sgsflag == 1:
        tau = tau_sgs(st, ui, uiuj, dphys)
    else:
        tau = None
    h = [[0.5 * uiuj[l][m] + (tau[l][m] if tau is not None else 0.0) for m in range(3)] for l in range(3)]
    nltf = [horfft_fwd(nlt[m], nx, ny) for m in range(3)]
    hf = [[horfft_fwd(h[l][m], nx, ny) for m in range(3)] for l in range(3)]
    for l in range(3):
        nltf[l] = nltf[l] - dfdx(st, hf[l][0]) - dfdy(st, hf[l][1]) - dfdz(st, hf[l][2])
    if return_parts:
        return nltf, dict(ui=ui, duidxj=dphys, uiuj=uiuj, tau=tau)
    return nltf


def abcoef(nstart, istep):
    """abcoef (src/navierstokes.f90:1500-1542); variable-dt AB is commented out there."""
    if nstart == 0 and istep == 1:
        return (1.0, 0.0, 0.0)
    if nstart == 0 and istep == 2:
        return (2.0, -1.0, 0.0)
    return (3.0, -3.0, 1.0)


def bdfcoef(nstart, istep, dt1, dt2, dt3):
    """bdfcoef (src/navierstokes.f90:1545-1662): returns (bdf1, bdf2, bdf3), bdfv."""
    if nstart == 0 and istep == 1:
        return (1.0, 0.0, 0.0), 1.0
    if nstart == 0 and istep == 2:
        return (2.0, -0.5, 0.0), 2.0 / 3.0
    if dt1 != dt2 or dt2 != dt3:
        d12, d23, d123 = dt1 + dt2, dt2 + dt3, dt1 + dt2 + dt3
        v = 1.0 + dt1 / d12 + dt1 / d123
        b1 = -(-1.0 - dt1 / dt2 - dt1 / d123 - dt1 * dt1 / (d123 * dt2) - dt1 * dt1 * d12 / (d123 * d23 * dt2))
        b2 = -(dt1 * dt1 / (d12 * dt2) + dt1 * dt1 / (dt2 * d123) + dt1 * dt1 * d12 / (dt2 * d23 * d123)
               + dt1 * dt1 * d12 / (dt3 * d23 * d123))
        b3 = -(-dt1 * dt1 * d12 / (dt3 * d23 * d123))
        return (b1, b2, b3), 1.0 / v
    return (3.0, -1.5, 1.0 / 3.0), 6.0 / 11.0


@dataclass
class State:
    """The reference's module ``core`` (src/common.f90:162-175) minus temperature."""
    uf: np.ndarray
    vf: np.ndarray
    wf: np.ndarray
    pf: np.ndarray
    pnf: np.ndarray
    unif: list
    unmif: list
    nlnif: list
    nlnmif: list
    t: float = 0.0
    dt: float = 0.0
    dt2: float = 0.0
    dt3: float = 0.0
    istep: int = 0
    nstart: int = 0
    abfac: tuple = (0.0, 0.0, 0.0)
    bdf: tuple = (0.0, 0.0, 0.0)
    bdfv: float = 0.0
    tavg: list = None

    @staticmethod
    def zeros_like(st: Setup, uf, vf, wf, dt):
        z = np.zeros_like(uf)
        return State(uf.copy(), vf.copy(), wf.copy(), z.copy(), z.copy(),
                     [z.copy() for _ in range(3)], [z.copy() for _ in range(3)],
                     [z.copy() for _ in range(3)], [z.copy() for _ in range(3)],
                     0.0, dt, dt, dt)

    def copy(self):
        import copy
        return copy.deepcopy(self)


def navierstokes_update(st: Setup, s: State):
    """navierstokes_update (src/navierstokes.f90:1157-1496); s.istep is the current step."""
    c = st.cfg
    nz = c.nz
    nzp = c.nzp
    istep = s.istep
    dt = s.dt
    uif = [s.uf.copy(), s.vf.copy(), s.wf.copy()]
    nlin = uif
    if c.dealiasflag >= 2:
        nlin = [specfilter_exp_xy(st, q) for q in uif]
    nltermif = nlterm_skewsym(st, nlin)
    if c.dealiasflag == 2:
        uif = [s.uf.copy(), s.vf.copy(), s.wf.copy()]
    elif c.dealiasflag >= 2:
        uif = nlin
    tmp = [q.copy() for q in nltermif]
    if istep <= 3 or dt != s.dt2 or s.dt2 != s.dt3:
        s.abfac = abcoef(s.nstart, istep)
    ab = s.abfac
    nlt = [ab[0] * nltermif[l] + ab[1] * s.nlnif[l] + ab[2] * s.nlnmif[l] for l in range(3)]
    if istep <= 3 or dt != s.dt2 or s.dt2 != s.dt3:
        s.bdf, s.bdfv = bdfcoef(s.nstart, istep, dt, s.dt2, s.dt3)
    bdf, bdfv = s.bdf, s.bdfv
    dtnui = 1.0 / (c.xnu * dt)
    rhsf = [-dtnui * (dt * nlt[l] + bdf[0] * uif[l] + bdf[1] * s.unif[l] + bdf[2] * s.unmif[l]) for l in range(3)]
    if np.sum(np.abs(st.ubarpp)) > 0.0:
        du0 = np.zeros((nzp, c.ny, c.nx + 2))
        du0[:, :, : c.nx] = st.ubarpp[:, None, None]
        rhsf[0] = rhsf[0] - horfft_fwd(du0, c.nx, c.ny)
    s.nlnmif = s.nlnif
    s.unmif = s.unif
    s.nlnif = tmp
    s.unif = [q.copy() for q in uif]
    if istep == 1:
        pfac = (0.0, 0.0)
    elif istep == 2:
        pfac = (1.0, 0.0)
    else:
        pfac = (2.0, -1.0)
    psf = pfac[0] * s.pf + pfac[1] * s.pnf
    s.pnf = s.pf.copy()
    dpf = dfdx(st, psf)
    uif[0][nzp - 1] = dt * bdfv * dpf[nzp - 1]
    w2 = wav2(st)
    for l in range(2):
        uif[l][0] = -rhsf[l][0] / (w2 + dtnui / bdfv)
    dwdzf = d2fdz2(st, uif[2])
    active = c.bctype > 0 and s.t >= c.istartbound
    if active:
        uif[2] = bound(st, s.t)
        uif[2][0] = uif[2][0] + c.xnu * dt * bdfv * dwdzf[0]
    else:
        uif[2][0] = c.xnu * dt * bdfv * dwdzf[0]
        uif[2][nzp - 1] = c.xnu * dt * bdfv * dwdzf[nzp - 1]
    dpf = dfdy(st, psf)
    uif[1][nzp - 1] = dt * bdfv * dpf[nzp - 1]
    if c.bctype == 3 and getattr(c, "bc3_top", 0) == 1:
        # extension (no reference counterpart): the free stream on the ceiling, u' = v = 0
        # in the velocity solves
        uif[0][0] = 0.0
        uif[1][0] = 0.0
    for l in range(3):
        if active or c.forcing == 1:
            solve_nhom_helmholtz(st, rhsf[l], uif[l], dtnui / bdfv)
        else:
            solve_helmholtz(st, rhsf[l], dtnui / bdfv)
    uf, vf, wf = rhsf[0], rhsf[1], rhsf[2]
    dpf = dfdz(st, uf)
    dwdzf = dfdz(st, vf)
    divdzf = divuv(st, dpf, dwdzf)
    divf = divuv(st, uf, vf)
    rhs3 = -divdzf - w2[None] * wf
    if active:
        wf = bound(st, s.t)
    else:
        wf = wf.copy()
        wf[0] = 0.0
        wf[nzp - 1] = 0.0
    solve_nhom_helmholtz(st, rhs3, wf, 0.0)
    wf = rhs3
    dwdzf = dfdz(st, wf)
    with np.errstate(divide="ignore", invalid="ignore"):
        pf = np.where(w2[None] == 0.0, 0.0, -(dwdzf + divf) / (w2[None] * dt * bdfv))
    uf = uf - dt * bdfv * dfdx(st, pf)
    vf = vf - dt * bdfv * dfdy(st, pf)
    s.uf, s.vf, s.wf, s.pf = uf, vf, wf, pf


def timestep(st: Setup, s: State):
    """timestep (src/navierstokes.f90:10-90) for istep = s.istep + 1 (ifilt hooks
    in ``filter_hook``; dtadapt handled by ``maxcalc``)."""
    c = st.cfg
    s.istep += 1
    if c.ifilt >= 1 and c.modfilt > 0 and s.istep % c.modfilt == 0:
        filter_hook(st, s)
    navierstokes_update(st, s)
    norm([s.uf, s.vf, s.wf], c.ny)
    if c.ifrz == 1:
        for f in (s.uf, s.vf, s.wf):
            f[:, 0, 0:2] = 0.0
    s.t = s.t + s.dt
    s.dt3 = s.dt2
    s.dt2 = s.dt
    if c.dtadapt == 1 and (s.istep % c.iomod == 0 or s.istep % 5 == 0):
        maxcalc(st, s)


def main_step(st: Setup, s: State):
    """One pass of the main loop body (src/main.f90:64-76): timestep, then the
    on-the-fly average q_tavg += q/iomod while its > istartavg."""
    timestep(st, s)
    c = st.cfg
    if c.otfavg == 1 and s.istep > c.istartavg:
        if s.tavg is None:
            s.tavg = [np.zeros_like(s.uf) for _ in range(4)]
        for a, q in zip(s.tavg, (s.uf, s.vf, s.wf, s.pf)):
            a += q / c.iomod


def filter_hook(st: Setup, s: State):
    """The ifilt branch of timestep (src/navierstokes.f90:33-40)."""
    c = st.cfg
    nx, ny = c.nx, c.ny
    if c.sgsflag == 1 and c.sgsmodel == 4:
        q = np.array([horfft_inv(f, nx, ny) for f in (s.uf, s.vf, s.wf, s.pf)])
        q2kc = modecut(st, q, 1.0, 6.0)
        qf = modecut(st, q, 1.0, 2.0)
        e1 = np.sum((q[:3, :, :, :nx] - qf[:3, :, :, :nx]) ** 2, axis=(0, 2, 3)) / (ny * nx)
        e2 = np.sum((q[:3, :, :, :nx] - q2kc[:3, :, :, :nx]) ** 2, axis=(0, 2, 3)) / (ny * nx)
        zp = st.grid.zpts
        ih = idel = 0.0
        for k in range(c.nz - 1, -1, -1):
            dz = zp[k] - zp[k + 1]
            ih += 0.5 * (e2[k] + e2[k + 1]) * dz
            idel += 0.5 * (e1[k] + e1[k + 1]) * dz
        if ih / idel > 0.007:
            s.uf, s.vf, s.wf, s.pf = (horfft_fwd(q2kc[i], nx, ny) for i in range(4))
        return ih / idel
    q = np.array([horfft_inv(f, nx, ny) for f in (s.uf, s.vf, s.wf, s.pf)])
    qf = modecut(st, q, c.a, c.b)
    s.uf, s.vf, s.wf, s.pf = (horfft_fwd(qf[i], nx, ny) for i in range(4))
    return None


def maxcalc(st: Setup, s: State, dtmax: float = 1.0):
    """maxcalc (src/navierstokes.f90:358-511).

    Returns the diagnostics; updates s.dt / s.dt2 like the reference
    (dt2 = dt3 then dt2 = dt, so dt3 is left alone)."""
    c = st.cfg
    g = st.grid
    nx, ny, nz = c.nx, c.ny, c.nz
    u = horfft_inv(s.uf, nx, ny)[..., :nx] + st.ubar[:, None, None]
    v = horfft_inv(s.vf, nx, ny)[..., :nx]
    w = horfft_inv(s.wf, nx, ny)[..., :nx]
    zp = g.zpts
    wc = np.empty_like(w)
    for k in range(nz):
        wc[k] = w[k] * s.dt / (zp[k] - zp[k + 1])
    wc[0] = wc[0] * s.dt / (zp[0] - zp[1])
    wc[nz] = w[nz] * s.dt / (zp[nz - 1] - zp[nz])
    # the reference's maxima run over the two pad columns too, which hold
    # 0 + ubar(k) for u and 0 for v, w (horfft zero-fills them)
    umax_abs = max(np.max(np.abs(u)), np.max(np.abs(st.ubar)))
    cflx = umax_abs * s.dt / g.dx
    cfly = max(np.max(np.abs(v)), 0.0) * s.dt / g.dy
    if s.t > c.istartbound:
        findex = int((1.0 - 0.8 * c.fsize) * nx)
        cflz = np.max(np.abs(wc[..., :findex]))
    else:
        cflz = np.max(np.abs(wc))
    exceed = cflz > 0.45 or cflx > 0.25 or cfly > 0.25
    below = cflz < 0.25 and cflx < 0.10 and cfly < 0.12 and s.dt < dtmax
    if exceed or below:
        cdt = 1.25 if exceed else 1.0 / 1.25
        s.dt2 = s.dt
        s.dt = s.dt / cdt
    return dict(umax=max(u.max(), st.ubar.max()), umin=min(u.min(), st.ubar.min()),
                vmax=max(v.max(), 0.0), vmin=min(v.min(), 0.0), wmax=max(w.max(), 0.0), wmin=min(w.min(), 0.0),
                cflx=cflx, cfly=cfly, cflz=cflz, changed=exceed or below)


def divcheck(st: Setup, uf, vf, wf):
    """divcheck (src/derivatives.f90:348-392): mean |div u| over the physical grid."""
    c = st.cfg
    d = dfdx(st, uf) + dfdy(st, vf) + dfdz(st, wf)
    p = horfft_inv(d, c.nx, c.ny)
    return np.sum(np.abs(p[..., : c.nx])) / (c.nx * c.ny * c.nzp)


def spanwise_stats(st: Setup, uf, vf, wf, pf):
    """Spanwise mean (run/spanwiseavg.m:1-7: sum over y / ny, per (x, z)) of u + ubar, v, w,
    p on the physical grid, and the rms about it; two arrays (4, nzp, nx)."""
    c = st.cfg
    ph = [horfft_inv(f, c.nx, c.ny)[..., : c.nx] for f in (uf, vf, wf, pf)]
    ph[0] = ph[0] + st.ubar[:, None, None]
    mean = np.stack([np.sum(f, axis=1) / float(c.ny) for f in ph])
    rms = np.stack([np.sqrt(np.sum((f - m[:, None, :]) ** 2, axis=1) / float(c.ny)) for f, m in zip(ph, mean)])
    return mean, rms


def ener(st: Setup, uf, vf, wf, itot: int):
    """ener (src/orrsomm.f90:625-666)."""
    c = st.cfg
    nx, ny, nz = c.nx, c.ny, c.nz
    u = horfft_inv(uf, nx, ny)[..., :nx]
    v = horfft_inv(vf, nx, ny)[..., :nx]
    w = horfft_inv(wf, nx, ny)[..., :nx]
    if itot == 1:
        u = u + st.ubar[:, None, None]
    ee = np.sum(0.5 * (u ** 2.0 + v ** 2.0 + w ** 2.0), axis=(1, 2))
    zp = st.grid.zpts
    en = 0.0
    for k in range(nz - 1, 0, -1):   # Fortran k = nz .. 2
        en = en + 0.5 * (ee[k + 1] + ee[k]) * (zp[k] - zp[k + 1])
    return en


def lintest(st: Setup, s: State):
    """lintest (src/orrsomm.f90:566-622) energies: (E_total, E_perturbation)."""
    en1 = ener(st, s.uf, s.vf, s.wf, 1)
    up, vp, wp = s.uf.copy(), s.vf.copy(), s.wf.copy()
    for f in (up, vp, wp):
        f[:, 0, 0:2] = 0.0
    en2 = ener(st, up, vp, wp, 0)
    return en1, en2
