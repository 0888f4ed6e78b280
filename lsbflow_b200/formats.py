"""The reference's on-disk formats, so device runs restart from and write the same files.

* restart ``start*.dat`` (mpi_write_restart_file / mpi_read_restart_file,
  src/mpi_io.f90:9-161, 164-300): native float32; a 9-value header
  [isum, t, dt, dt2, dt3, nx, ny, nzp, nxpl], then 20 variables of nx*ny*nzp values each:
  u, v, w, T, uni(1:3), unmi(1:3), nlni(1:3), nlnmi(1:3), tn, tnm, nltn, nltnm.  Each rank
  writes its x slab (nxpl spectral reals) as one block with the spectral index i slowest,
  then j, then k fastest; blocks follow rank order, so the file is the global (i, j, k)
  array whatever the rank count.  The reference's writer stores nlni again in variables
  14-16 (src/mpi_io.f90:62); ``write_restart(..., ref_bug=True)`` reproduces that, and its
  reader loads 14-16 into nlnmi.
* snapshot ``q*.dat`` / ``qavg*.dat`` (mpi_snapshot, src/mpi_io.f90:303-472): float32,
  a 7-value header [isum, t, dt, nx, ny, nzp, nypl], then 5 physical variables
  (u + ubar, v, w, T + Tbar, p) of nx*ny*nzp values, each rank's y slab ordered
  (y, z, x) with x fastest; over ranks the file is the global (y, z, x) array.
* ``grid.dat`` / ``paral.dat`` (write_grid / write_paral, src/io.f90:110-131, 251-275):
  Fortran sequential unformatted records (4-byte length markers), int32 sizes and float64
  arrays.

Arrays on the Python side use the device layout [nzp][ny][nx] (spectral: nx interleaved
re/im kx reals; physical: nx points).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass, field

import numpy as np

RESTART_VARS = ["u", "v", "w", "T", "uni0", "uni1", "uni2", "unmi0", "unmi1", "unmi2",
                "nlni0", "nlni1", "nlni2", "nlnmi0", "nlnmi1", "nlnmi2", "tn", "tnm", "nltn", "nltnm"]


@dataclass
class Restart:
    isum: int
    t: float
    dt: float
    dt2: float
    dt3: float
    nx: int
    ny: int
    nzp: int
    nxpl: int
    fields: dict = field(default_factory=dict)   # name -> [nzp][ny][nx] float64


def write_restart(path: str, r: Restart, ref_bug: bool = True) -> None:
    head = np.array([r.isum, r.t, r.dt, r.dt2, r.dt3, r.nx, r.ny, r.nzp, r.nxpl], dtype=np.float32)
    zero = np.zeros((r.nzp, r.ny, r.nx))
    with open(path, "wb") as f:
        head.tofile(f)
        for name in RESTART_VARS:
            src = name
            if ref_bug and name.startswith("nlnmi"):
                src = "nlni" + name[-1]
            a = r.fields.get(src, zero)
            # [nzp][ny][nx] -> file order (i, j, k), k fastest
            np.ascontiguousarray(np.transpose(a, (2, 1, 0)), dtype=np.float32).tofile(f)


def read_restart(path: str, nx: int | None = None, ny: int | None = None, nzp: int | None = None) -> Restart:
    raw = np.fromfile(path, dtype=np.float32)
    if raw.size < 9:
        raise ValueError(f"{path}: no restart header")
    h = raw[:9]
    isum, t, dt, dt2, dt3 = int(round(float(h[0]))), float(h[1]), float(h[2]), float(h[3]), float(h[4])
    fnx, fny, fnzp, fnxpl = (int(round(float(x))) for x in h[5:9])
    if (nx, ny, nzp) != (None, None, None) and (fnx, fny, fnzp) != (nx, ny, nzp):
        # src/mpi_io.f90:233-242 stops the run on a dimension mismatch
        raise ValueError(f"restart dimension mismatch: file ({fnx} {fny} {fnzp}) vs run ({nx} {ny} {nzp})")
    res = fnx * fny * fnzp
    if raw.size < 9 + 20 * res:
        raise ValueError(f"{path}: truncated restart file ({raw.size} values, need {9 + 20 * res})")
    r = Restart(isum, t, dt, dt2, dt3, fnx, fny, fnzp, fnxpl)
    for v, name in enumerate(RESTART_VARS):
        blk = raw[9 + v * res: 9 + (v + 1) * res].reshape(fnx, fny, fnzp)
        r.fields[name] = np.ascontiguousarray(np.transpose(blk, (2, 1, 0)), dtype=np.float64)
    return r


def restart_from_state(state: dict, isum: int, nxpl: int | None = None) -> Restart:
    """A Restart from ``Solver.download()`` output (u, v, w and the four histories)."""
    uf = state["uf"]
    nzp, ny, nx = uf.shape
    f = {"u": uf, "v": state["vf"], "w": state["wf"]}
    for key, name in (("unif", "uni"), ("unmif", "unmi"), ("nlnif", "nlni"), ("nlnmif", "nlnmi")):
        for l in range(3):
            f[f"{name}{l}"] = state[key][l]
    return Restart(isum, state["t"], state["dt"], state["dt2"], state["dt3"], nx, ny, nzp,
                   nx if nxpl is None else nxpl, f)


def upload_args(r: Restart) -> dict:
    """Keyword arguments of ``Solver.upload`` for a restart (p and p^(n-1) are not in the
    file and start at zero, as after mpi_read_restart_file)."""
    f = r.fields
    return dict(uf=f["u"], vf=f["v"], wf=f["w"],
                unif=np.array([f[f"uni{l}"] for l in range(3)]),
                unmif=np.array([f[f"unmi{l}"] for l in range(3)]),
                nlnif=np.array([f[f"nlni{l}"] for l in range(3)]),
                nlnmif=np.array([f[f"nlnmi{l}"] for l in range(3)]),
                t=r.t, dt=r.dt, dt2=r.dt2, dt3=r.dt3)


@dataclass
class Snapshot:
    isum: int
    t: float
    dt: float
    nx: int
    ny: int
    nzp: int
    nypl: int
    u: np.ndarray
    v: np.ndarray
    w: np.ndarray
    T: np.ndarray
    p: np.ndarray


def write_snapshot(path: str, s: Snapshot) -> None:
    head = np.array([s.isum, s.t, s.dt, s.nx, s.ny, s.nzp, s.nypl], dtype=np.float32)
    with open(path, "wb") as f:
        head.tofile(f)
        for a in (s.u, s.v, s.w, s.T, s.p):
            # [nzp][ny][nx] -> (y, z, x), x fastest
            np.ascontiguousarray(np.transpose(a, (1, 0, 2)), dtype=np.float32).tofile(f)


def read_snapshot(path: str) -> Snapshot:
    raw = np.fromfile(path, dtype=np.float32)
    if raw.size < 7:
        raise ValueError(f"{path}: no snapshot header")
    h = raw[:7]
    nx, ny, nzp, nypl = (int(round(float(x))) for x in h[3:7])
    res = nx * ny * nzp
    if raw.size < 7 + 5 * res:
        raise ValueError(f"{path}: truncated snapshot ({raw.size} values, need {7 + 5 * res})")
    out = []
    for v in range(5):
        blk = raw[7 + v * res: 7 + (v + 1) * res].reshape(ny, nzp, nx)
        out.append(np.ascontiguousarray(np.transpose(blk, (1, 0, 2)), dtype=np.float64))
    return Snapshot(int(round(float(h[0]))), float(h[1]), float(h[2]), nx, ny, nzp, nypl, *out)


def snapshot_from_spectral(solver, st, uf, vf, wf, pf, isum: int, t: float, dt: float, add_base: bool = True,
                           tempf=None) -> Snapshot:
    """What mpi_snapshot writes for spectral fields: horfft(+1) of each (on the device,
    through ``solver.horfft``), ubar added to u unless ``add_base`` is False (the
    q_ref.dat case, name = 2)."""
    c = st.cfg

    def phys(f):
        return solver.horfft(None, f, 1)[..., : c.nx]

    u, v, w, p = phys(uf), phys(vf), phys(wf), phys(pf)
    T = np.zeros_like(u) if tempf is None else phys(tempf)
    if add_base:
        u = u + st.ubar[:, None, None]
    return Snapshot(isum, t, dt, c.nx, c.ny, c.nzp, c.ny, u, v, w, T, p)


# ---------------------------------------------------------------- Fortran sequential records
def read_records(path: str) -> list:
    b = open(path, "rb").read()
    i, out = 0, []
    while i < len(b):
        n = struct.unpack("<i", b[i:i + 4])[0]
        n2 = struct.unpack("<i", b[i + 4 + n:i + 8 + n])[0]
        if n2 != n:
            raise ValueError(f"{path}: bad record markers at byte {i}")
        out.append(b[i + 4:i + 4 + n])
        i += 8 + n
    return out


def write_records(path: str, recs) -> None:
    with open(path, "wb") as f:
        for r in recs:
            f.write(struct.pack("<i", len(r)))
            f.write(r)
            f.write(struct.pack("<i", len(r)))


def write_grid(path: str, grid) -> None:
    recs = [np.array([grid.nx, grid.ny, grid.nzp], "<i4").tobytes(),
            np.array([grid.x0, grid.xl, grid.xlen, grid.ylen, grid.zlen], "<f8").tobytes(),
            np.asarray(grid.xpts, "<f8").tobytes(), np.asarray(grid.ypts, "<f8").tobytes(),
            np.asarray(grid.zpts, "<f8").tobytes(), np.asarray(grid.gf, "<f8").tobytes()]
    write_records(path, recs)


def read_grid(path: str) -> dict:
    r = read_records(path)
    nx, ny, nzp = np.frombuffer(r[0], "<i4")
    x0, xl, xlen, ylen, zlen = np.frombuffer(r[1], "<f8")
    return dict(nx=int(nx), ny=int(ny), nzp=int(nzp), x0=x0, xl=xl, xlen=xlen, ylen=ylen, zlen=zlen,
                xpts=np.frombuffer(r[2], "<f8").copy(), ypts=np.frombuffer(r[3], "<f8").copy(),
                zpts=np.frombuffer(r[4], "<f8").copy(), gf=np.frombuffer(r[5], "<f8").copy())


PARAL_VARS = ["ubar", "ubarp", "ubarpp", "wbar", "wbarp", "wbarpp", "tbar", "tbarp", "tbarpp"]


def write_paral(path: str, st) -> None:
    nzp = st.grid.nzp
    recs = [np.array([nzp], "<i4").tobytes()]
    for name in PARAL_VARS:
        a = getattr(st, name, None)
        recs.append(np.asarray(a if a is not None else np.zeros(nzp), "<f8").tobytes())
    write_records(path, recs)


def read_paral(path: str) -> dict:
    r = read_records(path)
    out = {"nzp": int(np.frombuffer(r[0], "<i4")[0])}
    for name, rec in zip(PARAL_VARS, r[1:]):
        out[name] = np.frombuffer(rec, "<f8").copy()
    return out
