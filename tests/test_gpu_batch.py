"""Ensembles stepped together (lsb_batch_*) give each member the result it reaches alone.

A batch advances every member by one time step per ensemble step; once every member is
steady the members' steps run as parallel branches of one CUDA graph.  Members here differ
in Re_delta*, ceiling-dipole amplitude and position (the ensemble draws), in precision and
in grid.  Each member stepped in the batch must equal, bit for bit, the same member stepped
alone through lsb_step, through the start-up steps, the ensemble captures and more than one
rotation of replays, and work issued on a member afterwards must follow the batch's steps.
"""
import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import ic
from lsbflow_b200.config import ensemble_configs, workload

pytestmark = pytest.mark.gpu

KEYS = ("uf", "vf", "wf", "pf", "pnf", "unif", "unmif", "nlnif", "nlnmif")


def members():
    # the mixed form needs register-plan transform lengths: padded x/2 = 96 = 32 x 3
    cfgs = ensemble_configs(3, seed=5, nx=128, ny=16, nz=32)          # sigma-model LES draws
    cfgs.append(cfgs[0].replace(precision=1))                         # mixed form of member 0
    cfgs.append(workload("dns64", nx=32, ny=8, nz=32, dealiasflag=1))  # another grid
    out = []
    for m, cfg in enumerate(cfgs):
        st = hs.make_setup(cfg)
        out.append((st, ic.seeded_noise(st, 40 + m, 1e-2)))
    return out


PATTERN = [5, 3, 3, 3, 3, 1]  # 18 steps: captures and replays at every rotation phase


@pytest.mark.parametrize("ens_graphs", [True, False], ids=["ensemble_graphs", "member_by_member"])
def test_batch_matches_members_alone(ens_graphs):
    from lsbflow_b200 import lib
    mem = members()

    alone, n_alone = [], 0
    for st, (u, v, w) in mem:
        s = lib.Solver(st)
        s.upload(u, v, w, dt=st.dt)
        k0 = lib.kernel_launches()
        for n in PATTERN:
            s.step(n)
        s.synchronize()
        n_alone += lib.kernel_launches() - k0
        s.step(2)
        alone.append(s.download())
        s.close()

    sols = []
    for st, (u, v, w) in mem:
        s = lib.Solver(st)
        s.upload(u, v, w, dt=st.dt)
        sols.append(s)
    b = lib.Batch(sols)
    try:
        b.graphs(ens_graphs)
        k0 = lib.kernel_launches()
        for n in PATTERN:
            b.step(n)
        b.synchronize()
        n_batch = lib.kernel_launches() - k0
        for s in sols:
            s.step(2)      # on the member's own stream, after the batch's steps
        got = [s.download() for s in sols]
    finally:
        b.close()
        for s in sols:
            s.close()

    assert n_batch == n_alone  # replays count the kernels they run
    for m, (a, g) in enumerate(zip(alone, got)):
        assert g["istep"] == a["istep"] == sum(PATTERN) + 2 and g["t"] == a["t"], m
        for k in KEYS:
            assert np.array_equal(g[k], a[k]), (m, k, np.abs(g[k] - a[k]).max())


def test_batch_rejects_bad_members():
    from lsbflow_b200 import lib
    st, (u, v, w) = members()[4]
    s = lib.Solver(st)
    try:
        with pytest.raises(lib.LsbError):
            lib.Batch([s, s])
        with pytest.raises(lib.LsbError):
            lib.Batch([])
    finally:
        s.close()
