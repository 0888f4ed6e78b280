"""Asynchronous q-file snapshots (lsb_snapshot_async + SnapshotWriter) hold what mpi_snapshot
writes for the state at that step -- horfft(+1) of u (+ ubar), v, w, p, here from the oracle's
transform of the same state downloaded from a second run -- while the run keeps stepping
after each write."""
import numpy as np
import pytest

from lsbflow_b200 import formats
from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import ic
from lsbflow_b200.config import workload
from lsbflow_b200.snapwriter import SnapshotWriter
from oracle import lsb_oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_async_snapshots_match_synchronous_ones(tmp_path, precision):
    import torch
    from lsbflow_b200 import lib

    cfg = workload("les256", nx=128, ny=16, nz=32, precision=precision)
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 12, 1e-2)
    stream = torch.cuda.Stream()
    s = lib.Solver(st)
    ref = lib.Solver(st)
    try:
        s.upload(u, v, w, dt=st.dt)
        ref.upload(u, v, w, dt=st.dt)
        wr = SnapshotWriter(s, str(tmp_path), stream)
        expected = {}
        for isum in (4, 8, 12):
            s.step(4)
            wr.write(isum, t=isum * st.dt, dt=st.dt)   # queued; stepping goes on
            ref.step(4)
            d = ref.download()
            phys = [O.horfft_inv(d[k], cfg.nx, cfg.ny)[..., : cfg.nx] for k in ("uf", "vf", "wf", "pf")]
            phys[0] = phys[0] + st.ubar[:, None, None]
            expected[isum] = phys
        s.step(3)
        wr.close()
        s.synchronize()
    finally:
        s.close()
        ref.close()
    for isum, e in expected.items():
        got = formats.read_snapshot(str(tmp_path / f"q{isum:05d}.dat"))
        assert (got.isum, got.nx, got.ny, got.nzp) == (isum, cfg.nx, cfg.ny, cfg.nzp)
        for name, a, b in zip("uvwp", (got.u, got.v, got.w, got.p), e):
            b32 = b.astype(np.float32).astype(np.float64)
            assert np.abs(a - b32).max() <= 1e-6 * np.abs(b32).max(), (isum, name)
        assert not got.T.any()
