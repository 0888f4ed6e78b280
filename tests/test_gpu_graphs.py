"""Steady steps replayed from CUDA graphs give the results of ordinary launches, bit for bit.

lsb_step captures one graph per rotation of the history buffers once the step is steady
(after the start-up steps, constant dt, no timers) and replays it; lsb_graphs(h, 0) turns
that off.  Both runs start from the same state and must agree exactly, through the start-up
steps, the captures and many replays (more than one full rotation of 6 steps).
"""
import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import ic
from lsbflow_b200.config import workload

pytestmark = pytest.mark.gpu

CASES = [
    ("les", dict(nx=128, ny=16, nz=32, sgsflag=1, sgsmodel=1, dealiasflag=1)),
    ("les_mixed", dict(nx=128, ny=16, nz=32, sgsflag=1, sgsmodel=1, dealiasflag=1, precision=1)),
    ("dns_avg", dict(nx=64, ny=16, nz=32, dealiasflag=1, otfavg=1, istartavg=5)),
]


@pytest.mark.parametrize("name,over", CASES, ids=[c[0] for c in CASES])
def test_graph_replay_matches_launches(name, over):
    from lsbflow_b200 import lib
    cfg = workload("dns64", **over)
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 21, 1e-2)
    out = []
    for graphs in (False, True):
        s = lib.Solver(st)
        s.graphs(graphs)
        s.upload(u, v, w, dt=st.dt)
        k0 = lib.kernel_launches()
        s.step(5)
        for _ in range(4):
            s.step(3)      # single calls and blocks, so replays start at every rotation phase
        s.step(1)
        s.synchronize()
        out.append((s.download(), lib.kernel_launches() - k0, s.tavg() if cfg.otfavg else None))
        s.close()
    (a, na, ta), (b, nb, tb) = out
    for k in ("uf", "vf", "wf", "pf", "pnf", "unif", "unmif", "nlnif", "nlnmif"):
        assert np.array_equal(a[k], b[k]), k
    assert a["istep"] == b["istep"] == 18 and a["t"] == b["t"]
    # replays count the kernels they run
    assert na == nb
    if ta is not None:
        for x, y in zip(ta, tb):
            assert np.array_equal(x, y)
