"""Run configuration for the LSBFLOW time step.

The fields mirror the reference's Fortran namelists ``&dimen``, ``&run``,
``&param`` and ``&sgsin`` (src/common.f90:20,78,92,107) with the defaults of
run/input.dat, plus the explicit extensions this implementation adds:

* ``dt_fixed``      -- a fixed time step (the reference only derives dt from
                       ``cfl``, src/init.f90:451,647-689); used with dtadapt=0.
* ``bctype = 3``    -- a zero-net-flux dipole on the ceiling,
                       w(x, z=zlen) = A (x-xc)/s exp(-((x-xc)/s)^2), with xc measured
                       from the domain inlet xpts(1).
* ``dealias_layout``-- "ref" reproduces the spanwise padding of
                       src/dealiasing.f90:329-330,435 bit for bit (negative ky modes
                       land at positive frequencies); "correct" is the textbook 3/2 rule.
* ``ic = 2``        -- start from caller-supplied (seeded) perturbation fields.
* ``bc3_top``       -- the ceiling condition for u, v with bctype 3.  0: the reference's
                       u, v = -rhs/(k^2 + sigma/beta) on the ceiling row
                       (src/navierstokes.f90:1340-1347), which lets the boundary values
                       evolve by the momentum equation without z diffusion -- an outflow
                       condition; where the zero-net-flux dipole blows fluid in, it is
                       ill-posed and perturbations grow there until the run diverges (the
                       oracle and the device alike, at any dt).  1 (default): the free
                       stream, u' = v = 0 on the ceiling in the velocity Helmholtz solves
                       (the projection then leaves a slip of dt beta grad p there).  The
                       wall's Zang-Hussaini form (src/navierstokes.f90:1338) on the ceiling
                       row is not used: with the pressure extrapolated there it diverges.
* ``precision``     -- 0: FP64 throughout (the reference's arithmetic); 1: the mixed form,
                       with the nonlinear-term transforms, products and SGS model in FP32
                       and the z derivatives of the nonlinear term and the velocity
                       Helmholtz solves on the int8 tensor cores (five int8 digits per
                       operand, exact int32 accumulation); the Poisson solve, the pressure
                       and the state stay FP64.

Sizes follow the reference's axes: x streamwise Fourier (nx), y spanwise Fourier
(ny), z vertical Chebyshev with nzp = nz+1 points, k=1 the ceiling, k=nzp the wall.
"""
from __future__ import annotations

import dataclasses
import math
import re
from dataclasses import dataclass, field


@dataclass
class LsbConfig:
    # &dimen
    nx: int = 64
    ny: int = 16
    nz: int = 64
    # &flaglist
    nstart: int = 0
    # &run
    cfl: float = 0.1
    dtadapt: int = 0
    nsteps: int = 200
    iomod: int = 1000000
    mapping: int = 2
    blfac: float = 8.0
    ic: int = 0
    bctype: int = 0
    istartbound: float = 0.0
    samp: float = 0.3
    forcing: int = 0
    fsize: float = 0.15
    lfsize: float = 0.25
    sfsize: float = 0.70
    linstab: int = 0
    astar: float = 0.8
    ifrz: int = 0
    sgsflag: int = 0
    ifilt: int = 0
    modfilt: int = 0
    dealiasflag: int = 2
    otfavg: int = 0
    istartavg: int = 0
    # &param
    xlen: float = 333.3333
    ylen: float = 20.0
    zlen: float = 33.3333
    x0: float = 8.3333
    u0: float = 1.0
    xnu: float = 0.001
    cguess: complex = 0.36 + 0.0j
    # &sgsin
    sgsmodel: int = 3
    a: float = 1.0
    b: float = 6.0
    CS: float = 0.1
    kc: float = 0.6
    filt_order: float = 1.0
    filt_amp: float = 20.0
    # extensions (see module docstring)
    dt_fixed: float | None = None
    bc3_amp: float = 0.3
    bc3_xc: float = 40.0
    bc3_s: float = 7.5
    dealias_layout: str = "ref"
    precision: int = 0      # 0: FP64 throughout; 1: mixed form (FP32 nonlinear-term transforms)
    bc3_top: int = 1        # bctype 3 ceiling for u, v: 0 the reference's outflow row, 1 free stream
    debug: int = 0

    @property
    def nzp(self) -> int:
        return self.nz + 1

    def replace(self, **kw) -> "LsbConfig":
        return dataclasses.replace(self, **kw)


_NML_KEYS = {f.name.lower(): f.name for f in dataclasses.fields(LsbConfig)}


def parse_namelist(text: str, base: LsbConfig | None = None) -> LsbConfig:
    """Parse the reference's input.dat namelist text (run/input.dat layout).

    Unknown keys (``iwrite``, ``prtl`` ...) are accepted and ignored,
    as they do not touch the time-step path.
    """
    cfg = dataclasses.replace(base) if base is not None else LsbConfig()
    body = re.sub(r"!.*", "", text)
    for m in re.finditer(r"([A-Za-z_][A-Za-z_0-9]*)\s*=\s*(\([^)]*\)|[^,/\n&]+)", body):
        key, val = m.group(1).lower(), m.group(2).strip()
        if key not in _NML_KEYS:
            continue
        name = _NML_KEYS[key]
        cur = getattr(cfg, name)
        if val.startswith("("):
            re_, im_ = (float(v) for v in val.strip("()").split(","))
            setattr(cfg, name, complex(re_, im_))
        elif isinstance(cur, int) and not isinstance(cur, bool):
            setattr(cfg, name, int(float(val.replace("d", "e").replace("D", "e"))))
        else:
            setattr(cfg, name, float(val.replace("d", "e").replace("D", "e")))
    return cfg


def delta_star_to_x0(re_dstar: float, xnu: float = 0.001, u0: float = 1.0) -> float:
    """x0 at which the Blasius displacement thickness 1.72 sqrt(nu x/U) gives Re_delta*.

    The reference's delta* constant is src/init.f90:614.
    """
    dstar = re_dstar * xnu / u0
    return (dstar / 1.72) ** 2 * u0 / xnu


def workload(name: str, re_d: float | None = None, bc_amp: float | None = None, bc_xc: float | None = None,
             **over) -> LsbConfig:
    """Named workloads in the reference's axes (x stream, y span, z Chebyshev).

    dns64   : 64 x 16 x 64 (nzp 65) plain DNS, Re_d*=500, fringe 10%, dipole ceiling BC.
    os128   : 128 x 4 x 96 (nzp 97) Orr-Sommerfeld linear test, Re_d*=1000 (displacement
              thickness), alpha d* = 0.25: the domain is one wavelength (linstab = 1).
    les256  : 256 x 64 x 128 (nzp 129) dynamic-Smagorinsky LES with the 3/2 rule.
    ens128  : 128 x 32 x 64 (nzp 65) sigma-model LES member.
    Lengths are 200/20/20 displacement thicknesses (xlen/ylen/zlen).  ``re_d``, ``bc_amp``
    and ``bc_xc`` (dipole centre in displacement thicknesses, default 80) override the
    workload's Re_delta*, ceiling-dipole amplitude and position.
    """
    if name == "dns64":
        re_d_default, amp, nx, ny, nz, sgs, model, dal = 500.0, 0.3, 64, 16, 64, 0, 0, 1
        dt = 0.01
    elif name == "os128":
        re_d_default, amp, nx, ny, nz, sgs, model, dal = 1000.0, 0.0, 128, 4, 96, 0, 0, 0
        dt = 0.005
    elif name == "les256":
        re_d_default, amp, nx, ny, nz, sgs, model, dal = 800.0, 0.35, 256, 64, 128, 1, 1, 1
        dt = 0.005
    elif name == "ens128":
        re_d_default, amp, nx, ny, nz, sgs, model, dal = 500.0, 0.3, 128, 32, 64, 1, 2, 1
        dt = 0.005
    else:
        raise ValueError(f"unknown workload {name!r}")
    re_d = re_d if re_d is not None else re_d_default
    amp = bc_amp if bc_amp is not None else amp
    xc = bc_xc if bc_xc is not None else 80.0
    xnu, u0 = 0.001, 1.0
    dstar = re_d * xnu / u0
    cfg = LsbConfig(
        nx=nx, ny=ny, nz=nz, xnu=xnu, u0=u0,
        x0=delta_star_to_x0(re_d, xnu, u0),
        xlen=200.0 * dstar, ylen=20.0 * dstar, zlen=20.0 * dstar,
        mapping=2, blfac=8.0, dtadapt=0, dt_fixed=dt,
        bctype=3 if amp > 0 else 0, bc3_amp=amp, bc3_xc=xc * dstar, bc3_s=15.0 * dstar,
        forcing=1 if name != "os128" else 0, fsize=0.1, lfsize=0.25, sfsize=0.70,
        sgsflag=sgs, sgsmodel=model, dealiasflag=dal, dealias_layout="correct",
        a=1.0, b=6.0, ic=2,
    )
    if name == "os128":
        # one wavelength 2 pi / alpha; astar is the reference's alpha * 6.02 sqrt(nu x0 / U)
        alpha = 0.25 / dstar
        cfg = dataclasses.replace(cfg, linstab=1, astar=alpha * 6.02 * math.sqrt(xnu * cfg.x0 / u0),
                                  cguess=0.36 + 0.0j, zlen=20.0 * dstar, nsteps=500)
    return dataclasses.replace(cfg, **over)


def ensemble_configs(n: int, seed: int, base: str = "ens128", **over) -> list:
    """Ensemble members of one grid: Re_delta* ~ U[300, 800], ceiling-dipole amplitude
    A ~ U[0.1, 0.4] and centre x0 ~ U[60, 100] displacement thicknesses, drawn from a
    seeded generator (member m's noise seed is the caller's, e.g. seed + m)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        re_d, amp, xc = rng.uniform(300.0, 800.0), rng.uniform(0.1, 0.4), rng.uniform(60.0, 100.0)
        out.append(workload(base, re_d=float(re_d), bc_amp=float(amp), bc_xc=float(xc), **over))
    return out
