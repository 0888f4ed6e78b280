"""The reference's file formats: restart start*.dat, snapshot q*.dat, grid.dat and
paral.dat (src/mpi_io.f90, src/io.f90), written and read back, and their layouts
checked against an independent per-rank statement of the reference's writers."""
import os

import numpy as np
import pytest

from lsbflow_b200 import formats as F
from lsbflow_b200 import hostsetup as hs
from lsbflow_b200.config import LsbConfig

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_run.npz"))


def fields(nzp, ny, nx, seed):
    rng = np.random.default_rng(seed)
    return {n: rng.standard_normal((nzp, ny, nx)) for n in F.RESTART_VARS}


def rank_blocks_restart(a, nprocs):
    """mpi_write_restart_file's per-rank loop (i, j, k; k fastest) over x slabs."""
    nzp, ny, nx = a.shape
    nxpl = nx // nprocs
    out = []
    for r in range(nprocs):
        for i in range(r * nxpl, (r + 1) * nxpl):
            for j in range(ny):
                out.extend(a[:, j, i])
    return np.array(out, dtype=np.float32)


def test_restart_layout_independent_of_ranks(tmp_path):
    nx, ny, nzp = 8, 4, 5
    fl = fields(nzp, ny, nx, 1)
    r = F.Restart(40, 1.25, 0.01, 0.01, 0.009, nx, ny, nzp, nx, fl)
    p = tmp_path / "start.dat"
    F.write_restart(str(p), r, ref_bug=False)
    raw = np.fromfile(p, np.float32)
    assert raw.size == 9 + 20 * nx * ny * nzp
    res = nx * ny * nzp
    for v, name in enumerate(F.RESTART_VARS):
        for P in (1, 2, 4):
            assert np.array_equal(raw[9 + v * res: 9 + (v + 1) * res], rank_blocks_restart(fl[name], P))


def test_restart_round_trip_and_ref_bug(tmp_path):
    nx, ny, nzp = 8, 4, 5
    fl = fields(nzp, ny, nx, 2)
    r = F.Restart(40, 1.25, 0.01, 0.011, 0.012, nx, ny, nzp, nx, fl)
    p = str(tmp_path / "start.dat")
    F.write_restart(p, r, ref_bug=True)
    back = F.read_restart(p, nx, ny, nzp)
    assert (back.isum, back.nx, back.ny, back.nzp, back.nxpl) == (40, nx, ny, nzp, nx)
    assert np.float32(back.dt2) == np.float32(0.011)
    for name in F.RESTART_VARS:
        src = "nlni" + name[-1] if name.startswith("nlnmi") else name
        assert np.array_equal(back.fields[name], fl[src].astype(np.float32).astype(np.float64))
    with pytest.raises(ValueError, match="mismatch"):
        F.read_restart(p, nx, ny, nzp + 2)


def test_snapshot_layout_and_round_trip(tmp_path):
    nx, ny, nzp = 6, 4, 3
    rng = np.random.default_rng(3)
    q = [rng.standard_normal((nzp, ny, nx)) for _ in range(5)]
    s = F.Snapshot(20, 0.5, 0.025, nx, ny, nzp, 2, *q)
    p = str(tmp_path / "q00002.dat")
    F.write_snapshot(p, s)
    raw = np.fromfile(p, np.float32)
    res = nx * ny * nzp
    # mpi_snapshot's per-rank loop (j, k, i; i fastest) over y slabs of nypl = 2
    for v in range(5):
        ref = []
        for r in range(ny // 2):
            for j in range(r * 2, r * 2 + 2):
                for k in range(nzp):
                    ref.extend(q[v][k, j, :])
        assert np.array_equal(raw[7 + v * res: 7 + (v + 1) * res], np.array(ref, np.float32))
    back = F.read_snapshot(p)
    assert (back.isum, back.nx, back.ny, back.nzp, back.nypl) == (20, nx, ny, nzp, 2)
    assert np.array_equal(back.w, q[2].astype(np.float32).astype(np.float64))


def test_snapshot_header_matches_shipped_files():
    # the shipped prev_q0000{1,2}.dat headers (extracted into the golden fixture)
    for step in (10, 20):
        h = GOLD[f"q{step}_header"]
        assert int(h[0]) == step and tuple(int(x) for x in h[3:6]) == (224, 24, 33)


def test_grid_and_paral_round_trip(tmp_path):
    cfg = LsbConfig(nx=16, ny=4, nz=16)
    st = hs.make_setup(cfg)
    gp = str(tmp_path / "grid.dat")
    F.write_grid(gp, st.grid)
    g = F.read_grid(gp)
    assert (g["nx"], g["ny"], g["nzp"]) == (16, 4, 17)
    assert np.array_equal(g["zpts"], st.grid.zpts) and g["xlen"] == st.grid.xlen
    pp = str(tmp_path / "paral.dat")
    F.write_paral(pp, st)
    pr = F.read_paral(pp)
    assert pr["nzp"] == 17 and np.array_equal(pr["ubarpp"], st.ubarpp)
    assert np.all(pr["tbar"] == 0)


def test_grid_reader_on_shipped_layout(tmp_path):
    # rebuild the shipped grid.dat from the golden fixture, read it back
    gd, gpar = GOLD["grid_dims"], GOLD["grid_params"]
    recs = [gd.astype("<i4").tobytes(), gpar.astype("<f8").tobytes()] + \
        [GOLD[k].astype("<f8").tobytes() for k in ("xpts", "ypts", "zpts", "gf")]
    p = str(tmp_path / "grid.dat")
    F.write_records(p, recs)
    g = F.read_grid(p)
    assert (g["nx"], g["ny"], g["nzp"]) == (224, 24, 33)
    assert np.array_equal(g["gf"], GOLD["gf"])
