"""The bench's side sections (tuned schedule, long-run profiles, serving, ensemble) run their
host logic end to end with stand-ins for the device, so a slip in them shows here and not
first in a GPU run."""
import types

import numpy as np
import pytest

import bench
from lsbflow_b200 import autotune as A
from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import lib
from lsbflow_b200 import serving as S
from lsbflow_b200.config import workload


class FakeSolver:
    def __init__(self, st):
        self.st = st
        self.cfg = st.cfg
        self.sched = {}

    def set_stream(self, s):
        pass

    def set_schedule(self, s):
        self.sched = dict(s)

    def upload(self, *a, **k):
        pass

    def step(self, n):
        pass

    def download(self):
        c = self.cfg
        return {k: np.ones((c.nzp, c.ny, c.nx)) * (1.0 + 1e-7 * c.precision) for k in ("uf", "vf", "wf", "pf")}

    def device_bytes(self):
        return 1 << 20

    def diag(self):
        self.ndiag = getattr(self, "ndiag", 0) + 1
        return {"nonfinite": 0, "umax": 1.0, "energy_pert": float(np.exp(1e-3 * self.ndiag))}

    def spanwise_stats(self):
        c = self.cfg
        m = np.ones((4, c.nzp, c.nx)) * (1.0 + 1e-7 * c.precision)
        return m, 2.0 * m

    def close(self):
        pass


class FakeBatch:
    def __init__(self, members):
        self.members = members

    def set_stream(self, s):
        pass

    def step(self, n):
        pass

    def close(self):
        pass


class FakeEvent:
    def __init__(self, enable_timing=False):
        pass

    def record(self, s=None):
        pass

    def elapsed_time(self, other):
        return 10.0


@pytest.fixture
def small_st():
    return hs.make_setup(workload("dns64", nx=32, ny=8, nz=16))


def test_tune_schedule_applies_only_checked_schedules(monkeypatch, small_st):
    monkeypatch.setattr(lib, "Solver", FakeSolver)
    faster = {"gemm_warps": 6, "filter_zchunks": 0, "y_staging": 0, "filter_staging": 0}
    monkeypatch.setattr(A, "gpu_measurer",
                        lambda st, steps, reps: (lambda s: 1.0 if s == faster else 2.0, lambda: None))
    sol = FakeSolver(small_st)
    out = bench.tune_schedule(types.SimpleNamespace(no_tune=False), small_st, sol)
    assert out["schedule"] == faster and out["applied"] and out["bit_identical_to_model"]
    assert sol.sched == faster
    assert bench.tune_schedule(types.SimpleNamespace(no_tune=True), small_st, sol) is None


def test_profiles_compare_the_two_forms(monkeypatch, small_st):
    monkeypatch.setattr(lib, "Solver", FakeSolver)
    out = bench.run_profiles(types.SimpleNamespace(profile_steps=100), small_st, None, None, None,
                             types.SimpleNamespace(cuda_stream=0))
    assert out["steps"] == 100 and out["target"] == 1e-4
    assert out["max_rel_err_mean_velocity"] == pytest.approx(1e-7, rel=1e-3)
    assert set(out["rel_err_rms"]) == set("uvwp")


def test_profiles_report_a_nonfinite_run(monkeypatch, small_st):
    class Diverging(FakeSolver):
        def diag(self):
            return {"nonfinite": 1, "umax": 1.0, "energy_pert": 0.0}

    monkeypatch.setattr(lib, "Solver", Diverging)
    out = bench.run_profiles(types.SimpleNamespace(profile_steps=200), small_st, None, None, None,
                             types.SimpleNamespace(cuda_stream=0))
    assert out["first_nonfinite_step"] == {"fp64": 100} and "error" in out


def test_os_growth_section(monkeypatch):
    monkeypatch.setattr(lib, "Solver", FakeSolver)
    out = bench.run_os_growth(types.SimpleNamespace(), types.SimpleNamespace(cuda_stream=0))
    assert out["steps"] == 500 and out["omega_i"] > 0
    # E grows by exp(1e-3) per step: <dE/dt> = (1 - exp(-1e-3)) / (2 dt)
    g = (1.0 - np.exp(-1e-3)) / (2 * 0.005)
    for form in ("fp64", "mixed"):
        assert out[form]["mean_growth"] == pytest.approx(g, rel=1e-9)
    assert out["mixed_rel_err_vs_fp64"] == pytest.approx(0.0, abs=1e-12)


def test_serving_section(monkeypatch):
    from test_serving_cpu import PreparingBackend

    class Backend(PreparingBackend):
        def __init__(self, schedules=None):
            assert schedules is None
            super().__init__(free=10 ** 12, lag=1)

    monkeypatch.setattr(S, "DeviceBackend", Backend)
    out = bench.run_serving(types.SimpleNamespace(serve_runs=4), 0)
    for form in ("fp64", "mixed", "fp64_grouped"):
        assert out[form]["runs"] == 4 and "error" not in out[form]
        assert out[form]["p99_s"] >= out[form]["p50_s"] > 0
    assert out["horizon_steps"] == [300, 3000]


def test_stream_requests_draw_the_survey_mix():
    reqs = S.stream_requests(300, 4.0, 5, precision=1)
    grids = {(r.cfg.nx, r.cfg.ny, r.cfg.nzp) for r in reqs}
    assert grids == {(64, 16, 65), (128, 32, 97), (256, 64, 129)}
    models = {(r.cfg.sgsflag, r.cfg.sgsmodel if r.cfg.sgsflag else None) for r in reqs}
    assert models == {(0, None), (1, 0), (1, 1), (1, 2), (1, 3)}
    assert all(r.cfg.precision == 1 for r in reqs)
    assert min(r.nsteps for r in reqs) >= 300 and max(r.nsteps for r in reqs) <= 3000
    t = [r.arrival for r in reqs]
    assert all(b > a for a, b in zip(t, t[1:])) and 50 < t[-1] < 100  # about 300 / 4 s


def test_ensemble_section(monkeypatch):
    import torch
    monkeypatch.setattr(lib, "Solver", FakeSolver)
    monkeypatch.setattr(lib, "Batch", FakeBatch)
    monkeypatch.setattr(torch.cuda, "mem_get_info", lambda: (100 << 30, 180 << 30))
    monkeypatch.setattr(torch.cuda, "Event", FakeEvent)
    monkeypatch.setattr(torch.cuda, "synchronize", lambda: None)
    args = types.SimpleNamespace(members=3, steps=300, warmup=5)
    out = bench.run_ensemble(args, 0, 1, types.SimpleNamespace(cuda_stream=0), lambda x: x, lambda: None)
    assert out["members"] == 3
    for form in ("fp64", "mixed"):
        assert out[form]["gain_vs_one_member"] == pytest.approx(3.0)
        assert out[form]["timed_steps"] == 30
    per = out["mixed_rel_err_velocity_per_member"]
    assert len(per["members"]) == 3 and per["max"] == pytest.approx(1e-7, rel=1e-6)


def test_clock_sampler_summary_inside_the_timed_region():
    c = bench.ClockSampler(0)
    c.samples = [(0.5, 1000.0, 1965.0, set()), (1.5, 1960.0, 1965.0, {"sw_power_cap"}),
                 (2.5, 1965.0, 1965.0, set()), (9.0, 500.0, 1965.0, {"hw_slowdown"})]
    c.t_start, c.t_end = 1.0, 3.0
    s = c.summary()
    assert s["samples"] == 2 and s["sm_mhz"] == 1962.5 and s["reasons"] == ["sw_power_cap"]
    c.t_start, c.t_end = 3.0, 4.0
    assert c.summary()["reasons"] == ["unsampled"]
