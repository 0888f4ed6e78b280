"""Restart through the reference's start.dat format: a device run is written to a float32
restart file, read back into a new handle with nstart = 1 (BDF3 from the first step,
src/navierstokes.f90:1500-1590) and continued; the oracle continues from the same file."""
import numpy as np
import pytest

from lsbflow_b200 import formats as F
from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import ic
from lsbflow_b200.config import workload
from oracle import lsb_oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b)


@pytest.mark.parametrize("ref_bug", [True, False])
def test_restart_continuation(tmp_path, ref_bug):
    from lsbflow_b200 import lib
    cfg = workload("dns64", nx=32, ny=8, nz=32, dealiasflag=1, dealias_layout="correct")
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 21, 2e-2)
    s1 = lib.Solver(st)
    s1.upload(u, v, w, dt=st.dt)
    s1.step(6)
    state = s1.download()
    s1.close()
    path = str(tmp_path / "start.dat")
    F.write_restart(path, F.restart_from_state(state, isum=6), ref_bug=ref_bug)
    r = F.read_restart(path, cfg.nx, cfg.ny, cfg.nzp)
    assert r.isum == 6

    st2 = hs.make_setup(cfg.replace(nstart=1))
    s2 = lib.Solver(st2)
    s2.upload(**F.upload_args(r), istep=0)
    s2.step(4)
    got = s2.download()
    s2.close()

    a = F.upload_args(r)
    ost = O.State(a["uf"], a["vf"], a["wf"], np.zeros_like(a["uf"]), np.zeros_like(a["uf"]),
                  list(a["unif"]), list(a["unmif"]), list(a["nlnif"]), list(a["nlnmif"]),
                  r.t, r.dt, r.dt2, r.dt3, istep=0, nstart=1)
    old = O.ZDER
    O.ZDER = "dense"
    try:
        for _ in range(4):
            O.timestep(st2, ost)
    finally:
        O.ZDER = old
    for key, ref in (("uf", ost.uf), ("vf", ost.vf), ("wf", ost.wf), ("pf", ost.pf)):
        assert rel(got[key], ref) < 1e-10, (key, rel(got[key], ref))
    assert got["istep"] == 4
