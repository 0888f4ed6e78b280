"""The native driver lsb_run continues a run from a restart file on the device, as the
reference's main loop does, and writes the q files and the final restart file that the
Python path writes for the same run: the restart byte for byte, the q files to float32
rounding of the oracle's transform of the same state.  (Named to run after the other GPU
parity tests.)"""
import os
import subprocess

import numpy as np
import pytest

from lsbflow_b200 import build
from lsbflow_b200 import formats as F
from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import ic
from lsbflow_b200.config import workload
from oracle import lsb_oracle as O

pytestmark = pytest.mark.gpu


def test_driver_continues_a_restart_like_the_python_path(tmp_path):
    from lsbflow_b200 import lib
    driver = build.build_driver()
    cfg = workload("dns64", nx=32, ny=8, nz=32, dealiasflag=1)
    st0 = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st0, 31, 2e-2)
    s = lib.Solver(st0)
    try:
        s.upload(u, v, w, dt=st0.dt)
        s.step(6)
        start = str(tmp_path / "start.dat")
        F.write_restart(start, F.restart_from_state(s.download(), isum=6), ref_bug=True)
    finally:
        s.close()

    # restarted runs: BDF3 from the first step (nstart = 1, src/navierstokes.f90:1500-1590)
    st = hs.make_setup(cfg.replace(nstart=1))
    lib.write_setup_file(str(tmp_path / "setup.bin"), st)
    out_dir = tmp_path / "out"
    os.makedirs(out_dir)
    res = subprocess.run([driver, str(tmp_path / "setup.bin"), start, "6", "3", str(out_dir)],
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    assert res.stdout.count("step ") == 2

    r = F.read_restart(start, cfg.nx, cfg.ny, cfg.nzp)
    s2 = lib.Solver(st)
    try:
        s2.upload(**F.upload_args(r), istep=0)
        for isum in (9, 12):
            s2.step(3)
            d = s2.download()
            q = F.read_snapshot(str(out_dir / f"q{isum:05d}.dat"))
            assert (q.isum, q.nx, q.ny, q.nzp) == (isum, cfg.nx, cfg.ny, cfg.nzp)
            assert abs(q.t - d["t"]) <= 1e-6 * max(1.0, abs(d["t"]))
            want = [O.horfft_inv(d[k], cfg.nx, cfg.ny)[..., : cfg.nx] for k in ("uf", "vf", "wf", "pf")]
            want[0] = want[0] + st.ubar[:, None, None]
            for name, a, b in zip("uvwp", (q.u, q.v, q.w, q.p), want):
                b32 = b.astype(np.float32).astype(np.float64)
                assert np.abs(a - b32).max() <= 1e-6 * np.abs(b32).max(), (isum, name)
        expect = str(tmp_path / "expect.dat")
        F.write_restart(expect, F.restart_from_state(d, isum=12), ref_bug=True)
    finally:
        s2.close()
    with open(out_dir / "end.dat", "rb") as a, open(expect, "rb") as b:
        assert a.read() == b.read()
