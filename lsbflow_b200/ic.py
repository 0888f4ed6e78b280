"""Seeded divergence-free perturbation fields (``ic = 2``).

The reference has no seeded noise IC (src/init.f90:426-440 leaves u = v = w = 0 and
its random seeding reads /dev/urandom, src/common.f90:245-293).  This builds a
reproducible one in spectral space, in the reference's spectral layout:

1. a random vector potential psi with seeded random phases on the modes
   |kx| <= nx/3, |ky| <= ny/3 (kx < nx/2 stored, ky in FFT order), times the
   z envelope (xi (1 - xi))^2 so psi and d psi/dz vanish at both boundaries;
2. u = curl psi with the spectral x/y derivatives and the Chebyshev D matrix
   (d/dx, d/dy and D commute column by column, so div u = 0 to round-off);
3. the boundary planes k = 1 and k = nzp are set to zero and the reference's
   ``norm`` symmetrisation (src/horfft.f90:153-224) is applied;
4. the result is scaled so that the rms over all grid points of the three
   perturbation components together is ``amp * u0``.
"""
from __future__ import annotations

import numpy as np

from .hostsetup import Setup


def _norm_inplace(fields, ny):
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


def _phys_rms(fields, nx, ny):
    tot = 0.0
    for f in fields:
        c = f[..., 0::2] + 1j * f[..., 1::2]
        y = np.fft.ifft(c, axis=-2) * ny
        full = np.zeros(c.shape[:-1] + (nx // 2 + 1,), dtype=np.complex128)
        full[..., : nx // 2] = y
        full[..., 0] = full[..., 0].real
        p = np.fft.irfft(full, n=nx, axis=-1) * nx
        tot += float(np.mean(p * p))
    return np.sqrt(tot / 3.0)


def seeded_noise(st: Setup, seed: int, amp: float):
    """Returns (uf, vf, wf) spectral arrays of shape (nzp, ny, nx)."""
    cfg = st.cfg
    nx, ny, nzp = cfg.nx, cfg.ny, cfg.nzp
    g = st.grid
    rng = np.random.default_rng(seed)
    kx = np.arange(nx // 2)
    ky = np.fft.fftfreq(ny, 1.0 / ny).astype(int)
    mask = (kx[None, :] <= nx // 3) & (np.abs(ky)[:, None] <= ny // 3)
    xi = (g.zpts - g.zpts[-1]) / (g.zpts[0] - g.zpts[-1])
    env = (xi * (1.0 - xi)) ** 2
    psi = []
    for _ in range(3):
        ph = rng.uniform(0.0, 2.0 * np.pi, size=(nzp, ny, nx // 2))
        mag = rng.standard_normal(size=(nzp, ny, nx // 2))
        c = mag * np.exp(1j * ph) * mask[None] * env[:, None, None]
        c[:, 0, 0] = 0.0
        f = np.empty((nzp, ny, nx))
        f[..., 0::2] = c.real
        f[..., 1::2] = c.imag
        psi.append(f)
    # smooth psi in z with the Chebyshev basis: apply D once and integrate back is
    # unnecessary; the envelope already makes psi vanish at the boundaries.
    wx = g.wavx[0::2][None, None, :]
    wy = g.wavy[None, :, None]

    def ddx(f):
        o = np.empty_like(f)
        o[..., 0::2] = -wx * f[..., 1::2]
        o[..., 1::2] = wx * f[..., 0::2]
        return o

    def ddy(f):
        o = np.empty_like(f)
        o[..., 0::2] = -wy * f[..., 1::2]
        o[..., 1::2] = wy * f[..., 0::2]
        return o

    def ddz(f):
        return np.einsum("km,mji->kji", st.d, f)

    u = ddy(psi[2]) - ddz(psi[1])
    v = ddz(psi[0]) - ddx(psi[2])
    w = ddx(psi[1]) - ddy(psi[0])
    for f in (u, v, w):
        f[0] = 0.0
        f[-1] = 0.0
    _norm_inplace([u, v, w], ny)
    rms = _phys_rms([u, v, w], nx, ny)
    s = amp * cfg.u0 / rms if rms > 0 else 0.0
    return u * s, v * s, w * s
