"""The double-buffered snapshot writer's host logic, with a stand-in for the device copy:
files are written in the reference's q-file layout, buffers alternate, and a buffer is
reused only after its file is written."""
import threading

import numpy as np

from lsbflow_b200 import formats
from lsbflow_b200.config import workload
from lsbflow_b200.snapwriter import SnapshotWriter


class FakeSolver:
    def __init__(self, cfg):
        self.cfg = cfg
        self.k = 0
        self.addrs = []
        self.bufs = {}

    def fields(self, k):
        c = self.cfg
        rng = np.random.default_rng(k)
        return rng.standard_normal((4, c.nzp, c.ny, c.nx))

    def snapshot_async(self, addr):
        self.addrs.append(addr)
        self.bufs[addr][:] = self.fields(self.k).ravel()
        self.k += 1


class SlowEvent:
    """Stands for a CUDA event the writer thread waits on."""
    def __init__(self, gate):
        self.gate = gate

    def synchronize(self):
        self.gate.wait(5.0)


def test_writes_reference_layout_and_alternates_buffers(tmp_path):
    cfg = workload("dns64", nx=16, ny=4, nz=8)
    sol = FakeSolver(cfg)
    gate = threading.Event()

    def alloc(n):
        a = np.zeros(n)
        sol.bufs[a.ctypes.data] = a
        return a

    w = SnapshotWriter(sol, str(tmp_path), alloc=alloc, record_event=lambda: SlowEvent(gate))
    f0 = w.write(10, 0.1, 0.01)
    f1 = w.write(20, 0.2, 0.01)
    assert not f0.done() and not f1.done()     # queued: the copies have not "arrived" yet
    assert sol.addrs[0] != sol.addrs[1]        # two buffers
    gate.set()
    w.write(30, 0.3, 0.01)                     # reuses buffer 0 once file 10 is written
    assert sol.addrs[2] == sol.addrs[0]
    w.close()
    for k, (isum, t) in enumerate(((10, 0.1), (20, 0.2), (30, 0.3))):
        s = formats.read_snapshot(str(tmp_path / f"q{isum:05d}.dat"))
        q = sol.fields(k).astype(np.float32).astype(np.float64)
        assert (s.isum, s.nx, s.ny, s.nzp, s.nypl) == (isum, cfg.nx, cfg.ny, cfg.nzp, cfg.ny)
        assert abs(s.t - t) < 1e-6 and abs(s.dt - 0.01) < 1e-9
        for got, want in zip((s.u, s.v, s.w, s.p), q):
            assert np.array_equal(got, want)
        assert not s.T.any()
