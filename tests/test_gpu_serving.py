"""Continuous batching on the device: runs of different grids and models, arriving while
others are stepping, give the same result alone and in the mix."""
import numpy as np
import pytest

from lsbflow_b200 import serving as S
from lsbflow_b200.config import workload

pytestmark = pytest.mark.gpu


def requests():
    a = workload("dns64", nx=32, ny=8, nz=32, dealiasflag=1)
    b = workload("ens128", nx=64, ny=16, nz=32)               # sigma-model LES
    c = workload("les256", nx=64, ny=16, nz=32)               # dynamic Smagorinsky
    return [S.RunRequest(0, a, 40, seed=1, amp=1e-2, arrival=0.0),
            S.RunRequest(1, b, 30, seed=2, amp=1e-2, arrival=0.0),
            S.RunRequest(2, c, 25, seed=3, amp=1e-2, arrival=0.02),
            S.RunRequest(3, a, 20, seed=4, amp=1e-2, arrival=0.05)]


def test_results_same_alone_and_in_the_mix():
    reqs = requests()
    srv = S.Server(chunk=5)
    for r in reqs:
        srv.submit(r)
    mixed = {r.rid: r for r in srv.run()}
    summ = S.summary(list(mixed.values()), srv.elapsed)
    assert summ["runs"] == 4 and summ["p99"] >= summ["p50"] > 0
    for r in reqs:
        alone = S.Server(chunk=r.nsteps)
        r2 = S.RunRequest(r.rid, r.cfg, r.nsteps, r.seed, r.amp, 0.0)
        alone.submit(r2)
        ref = alone.run()[0].state
        got = mixed[r.rid].state
        assert got["istep"] == r.nsteps
        for k in ("uf", "vf", "wf", "pf"):
            assert np.array_equal(got[k], ref[k]), (r.rid, k, np.abs(got[k] - ref[k]).max())


def test_grouped_cohorts_same_as_alone():
    """Same-shape runs stepped as one ensemble batch (runs 0 and 3 share a grid; 3 joins
    while 0 is stepping) reach the results they reach alone."""
    reqs = requests()
    srv = S.Server(chunk=5, group=True)
    for r in reqs:
        srv.submit(r)
    grouped = {r.rid: r for r in srv.run()}
    for r in reqs:
        alone = S.Server(chunk=r.nsteps)
        alone.submit(S.RunRequest(r.rid, r.cfg, r.nsteps, r.seed, r.amp, 0.0))
        ref = alone.run()[0].state
        got = grouped[r.rid].state
        assert got["istep"] == r.nsteps
        for k in ("uf", "vf", "wf", "pf"):
            assert np.array_equal(got[k], ref[k]), (r.rid, k, np.abs(got[k] - ref[k]).max())
