"""Launch schedules (lsb_set_schedule) change speed only: every schedule gives the results
of the built-in models bit for bit, and the tuner stores a valid schedule per grid."""
import numpy as np
import pytest

from lsbflow_b200 import autotune as A
from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import ic
from lsbflow_b200.config import workload

pytestmark = pytest.mark.gpu

KEYS = ("uf", "vf", "wf", "pf", "pnf", "unif", "nlnif")


def run(st, u, v, w, sched, n=12):
    from lsbflow_b200 import lib
    s = lib.Solver(st)
    try:
        s.set_schedule(sched)
        assert s.schedule() == {"gemm_warps": sched.get("gemm_warps", 0),
                                "filter_zchunks": sched.get("filter_zchunks", 0),
                                "y_staging": sched.get("y_staging", 0),
                                "filter_staging": sched.get("filter_staging", 0)}
        s.upload(u, v, w, dt=st.dt)
        s.step(n)
        return s.download()
    finally:
        s.close()


@pytest.mark.parametrize("precision", [0, 1], ids=["fp64", "mixed"])
def test_schedules_are_bit_identical(precision):
    # dynamic model (filtered); padded x/2 = 96 = 32 x 3 as the mixed form's transforms need
    cfg = workload("les256", nx=128, ny=16, nz=32, precision=precision)
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 8, 1e-2)
    ref = run(st, u, v, w, {})
    zmax = max(1, (cfg.nzp + 3) // 4)
    for sched in ({"gemm_warps": 4}, {"gemm_warps": 7, "filter_zchunks": 1},
                  {"gemm_warps": 8, "filter_zchunks": zmax}, {"filter_zchunks": 2},
                  {"y_staging": 2}, {"y_staging": 1, "gemm_warps": 5}, {"filter_staging": 1},
                  {"filter_staging": 2, "filter_zchunks": 3}):
        got = run(st, u, v, w, sched)
        for k in KEYS:
            assert np.array_equal(got[k], ref[k]), (sched, k)


def test_set_schedule_rejects_out_of_range():
    from lsbflow_b200 import lib
    st = hs.make_setup(workload("dns64", nx=32, ny=8, nz=32))
    s = lib.Solver(st)
    try:
        for bad in ({"gemm_warps": 3}, {"gemm_warps": 9}, {"filter_zchunks": -1},
                    {"filter_zchunks": (st.cfg.nzp + 3) // 4 + 1}, {"y_staging": 3}, {"filter_staging": 3},
                    {"filter_staging": -1}):
            with pytest.raises(lib.LsbError):
                s.set_schedule(bad)
        assert s.schedule() == {"gemm_warps": 0, "filter_zchunks": 0, "y_staging": 0, "filter_staging": 0}
    finally:
        s.close()
    # TMA row loads need rows of a multiple of 128 bytes: 8 FP64 points are 64 bytes
    s = lib.Solver(hs.make_setup(workload("les256", nx=8, ny=8, nz=16)))
    try:
        with pytest.raises(lib.LsbError):
            s.set_schedule({"filter_staging": 2})
    finally:
        s.close()


def test_tune_and_store(tmp_path):
    st = hs.make_setup(workload("les256", nx=64, ny=16, nz=32))
    path = str(tmp_path / "schedules.json")
    res = A.tune_and_store(st, path, steps=3, reps=1)
    got = A.lookup(st.cfg, path, res["device"])
    assert got == res["schedule"]
    c = A.candidates(st.cfg)
    assert got["gemm_warps"] in c["gemm_warps"] and got["filter_zchunks"] in c["filter_zchunks"]
    assert got["y_staging"] in c["y_staging"] and got["filter_staging"] in c["filter_staging"]
    assert res["ms_per_step"] <= res["model_ms_per_step"] and res["ms_per_step"] > 0


@pytest.mark.parametrize("grid", [dict(nx=256, ny=64, nz=128), dict(nx=64, ny=16, nz=64, sgsflag=0),
                                  dict(nx=32, ny=8, nz=16, sgsflag=0), dict(nx=128, ny=24, nz=32, precision=1)],
                         ids=["les256", "nz64", "nz16", "mixed"])
def test_fused_helmholtz_solves_are_bit_identical(grid):
    # the velocity and Poisson solves as one launch each (the models' widths, 4 or 6 warps:
    # E^-1 and E_ext with the intermediate in registers, E_ext's wall row as the edge row)
    # against the two separate contractions (gemm_warps 5): the same products and sums in
    # the same order, with the lifted right-hand side of the non-homogeneous solves; in the
    # mixed form only the Poisson solve has FP64 contractions to fuse
    cfg = workload("les256", **grid)
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 13, 5e-3)
    ref = run(st, u, v, w, {"gemm_warps": 5}, n=6)
    got = run(st, u, v, w, {}, n=6)
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k


@pytest.mark.parametrize("grid", [dict(nx=256, ny=64, nz=128), dict(nx=64, ny=16, nz=64, sgsflag=0),
                                  dict(nx=64, ny=16, nz=16, dealias_layout="ref"), dict(nx=64, ny=16, nz=32, dealiasflag=0)],
                         ids=["les256", "dns64", "ref-layout", "no-dealias"])
def test_tma_staged_spanwise_passes_are_bit_identical(grid):
    # the FP64 spanwise tiles staged by TMA tile loads (y_staging 2): the same arithmetic as
    # the cp.async staging, so the same state bit for bit, on the padded textbook layout (the
    # two-box split), the reference's padded layout, and the unpadded grid
    cfg = workload("les256", **grid)
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 9, 5e-3)
    ref = run(st, u, v, w, {"y_staging": 1}, n=6)
    got = run(st, u, v, w, {"y_staging": 2}, n=6)
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k


@pytest.mark.parametrize("grid", [dict(nx=256, ny=64, nz=128), dict(nx=128, ny=24, nz=32),
                                  dict(nx=16, ny=8, nz=16), dict(nx=512, ny=8, nz=16, precision=1),
                                  dict(nx=128, ny=24, nz=32, precision=1)],
                         ids=["les256", "partial-block", "one-block", "mixed-512", "mixed-partial"])
def test_tma_staged_filter_ring_is_bit_identical(grid):
    # the dynamic model's 3-point test filter with its plane ring filled by TMA row loads
    # (filter_staging 2; two boxes per row where a row is wider than 256 points, the periodic
    # y halo rows wrapped, a last block of fewer rows) gives the cp.async ring's state bit for bit
    cfg = workload("les256", **grid)
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 10, 5e-3)
    ref = run(st, u, v, w, {"filter_staging": 1}, n=4)
    got = run(st, u, v, w, {"filter_staging": 2}, n=4)
    for k in KEYS:
        assert np.array_equal(got[k], ref[k]), k
