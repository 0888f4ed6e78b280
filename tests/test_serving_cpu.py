"""The serving loop's admission and scheduling, with a fake device backend."""
import threading

import pytest

from lsbflow_b200 import serving as S
from lsbflow_b200.config import workload


class FakeBackend:
    """Each launch completes after ``lag`` polls; records the device bytes in use."""

    def __init__(self, free=10_000_000, lag=2, nbytes=None):
        self.free = free
        self.lag = lag
        self.nbytes = nbytes or {}
        self.in_use = 0
        self.peak = 0
        self.log = []
        self.runs_by_rid = {}

    def free_bytes(self):
        return self.free

    def start(self, req):
        b = self.nbytes.get(req.rid, S.estimate_bytes(req.cfg))
        self.in_use += b
        self.peak = max(self.peak, self.in_use)
        self.log.append(("start", req.rid))
        run = {"rid": req.rid, "steps": 0, "polls": 0, "bytes": b}
        self.runs_by_rid[req.rid] = run
        return run

    def launch(self, run, n):
        run["steps"] += n
        run["polls"] = self.lag

    def ready(self, run):
        if run["polls"] > 0:
            run["polls"] -= 1
            return False
        return True

    def abort(self, run):
        assert not run.get("in_group"), "a run was freed while its cohort's batch held it"
        self.in_use -= run["bytes"]
        self.log.append(("abort", run["rid"]))

    def finish(self, run):
        assert not run.get("in_group"), "a run was finished while its cohort's batch held it"
        self.in_use -= run["bytes"]
        self.log.append(("finish", run["rid"]))
        return {"steps": run["steps"]}

    # cohorts (Server(group=True)): one launch advances every member
    def new_group(self):
        return {"members": (), "polls": 0, "batches": 0}

    def launch_group(self, g, runs, n):
        ids = tuple(r["rid"] for r in runs)
        if g["members"] != ids:
            self.close_group(g)
            g["members"] = ids
            g["batches"] += 1
            for r in runs:
                r["in_group"] = True
        for r in runs:
            assert "polls" not in r or r["polls"] == 0
            r["steps"] += n
        g["polls"] = self.lag
        self.log.append(("group", ids, n))

    def group_ready(self, g):
        if g["polls"] > 0:
            g["polls"] -= 1
            return False
        return True

    def close_group(self, g):
        self.log.append(("close", g["members"]))
        g["members"] = ()
        # members of a closed batch may be finished
        for r in self.runs_by_rid.values():
            r["in_group"] = False


def cfg(nx):
    return workload("dns64", nx=nx, ny=8, nz=16)


def test_all_runs_complete_with_their_steps():
    be = FakeBackend()
    srv = S.Server(backend=be, memory_budget=10_000_000, chunk=7)
    for i in range(5):
        srv.submit(S.RunRequest(i, cfg(32), nsteps=10 + 3 * i, arrival=0.001 * i))
    res = srv.run()
    assert [r.rid for r in res] == list(range(5))
    assert [r.state["steps"] for r in res] == [10 + 3 * i for i in range(5)]
    s = S.summary(res, srv.elapsed)
    assert s["runs"] == 5 and s["p50"] <= s["p99"]


def test_admission_respects_memory_budget_and_order():
    one = S.estimate_bytes(cfg(32))
    be = FakeBackend()
    srv = S.Server(backend=be, memory_budget=int(2.5 * one), chunk=5)
    for i in range(6):
        srv.submit(S.RunRequest(i, cfg(32), nsteps=20, arrival=0.0))
    srv.run()
    assert be.peak <= 2 * one                      # never three resident at once
    starts = [rid for ev, rid in be.log if ev == "start"]
    assert starts == sorted(starts)                 # first come, first admitted


def test_measured_footprint_replaces_estimate():
    be = FakeBackend(nbytes={0: 1000})
    srv = S.Server(backend=be, memory_budget=10_000_000)
    srv.submit(S.RunRequest(0, cfg(32), nsteps=3))
    srv.run()
    assert srv.footprints[S.shape_key(cfg(32))] == 1000


def test_oversize_request_rejected():
    srv = S.Server(backend=FakeBackend(), memory_budget=1000)
    with pytest.raises(ValueError, match="budget"):
        srv.submit(S.RunRequest(0, cfg(64), nsteps=3))


def test_poisson_requests_are_seeded():
    shapes = [cfg(32), cfg(64)]
    a = S.poisson_requests(8, 4.0, 7, shapes)
    b = S.poisson_requests(8, 4.0, 7, shapes)
    assert [(r.arrival, r.nsteps, r.cfg.nx) for r in a] == [(r.arrival, r.nsteps, r.cfg.nx) for r in b]
    assert all(x.arrival < y.arrival for x, y in zip(a, a[1:]))


def test_grouped_cohorts_step_together_and_finish_after_their_batch():
    be = FakeBackend()
    srv = S.Server(backend=be, memory_budget=100_000_000, chunk=7, group=True)
    horizons = [10, 16, 13, 9, 20]
    shapes = [cfg(32), cfg(32), cfg(64), cfg(32), cfg(64)]
    for i, (n, c) in enumerate(zip(horizons, shapes)):
        srv.submit(S.RunRequest(i, c, nsteps=n, arrival=0.0))
    res = srv.run()
    assert [r.rid for r in res] == list(range(5))
    assert [r.state["steps"] for r in res] == horizons          # each run does exactly its steps
    groups = [e for e in be.log if e[0] == "group"]
    # runs of one shape advance together; the two shapes never share a launch
    assert any(set(ids) == {0, 1, 3} for _, ids, _ in groups)
    assert any(set(ids) == {2, 4} for _, ids, _ in groups)
    assert all(set(ids) <= {0, 1, 3} or set(ids) <= {2, 4} for _, ids, _ in groups)
    # a chunk never overshoots a member's horizon
    assert all(n <= 7 for _, _, n in groups)
    assert be.in_use == 0


def test_grouped_admission_respects_budget_and_late_arrivals_join():
    one = S.estimate_bytes(cfg(32))
    be = FakeBackend()
    t = [0.0]

    def clock():
        t[0] += 0.001
        return t[0]

    srv = S.Server(backend=be, memory_budget=int(2.5 * one), chunk=5, group=True)
    for i in range(5):
        srv.submit(S.RunRequest(i, cfg(32), nsteps=12, arrival=0.004 * i))
    res = srv.run(clock=clock, idle_sleep=0.0)
    assert [r.state["steps"] for r in res] == [12] * 5
    assert be.peak <= 2 * one
    starts = [rid for ev, rid, *_ in be.log if ev == "start"]
    assert starts == sorted(starts)
    sizes = {len(ids) for ev, ids, *_ in be.log if ev == "group"}
    assert 2 in sizes                                  # a later arrival joined a running cohort


class PreparingBackend(FakeBackend):
    """A backend whose host set-up runs ahead of admission on helper threads."""

    def __init__(self, **kw):
        super().__init__(**kw)
        self.prepared = []
        self.lock = threading.Lock()

    def prepare(self, req):
        with self.lock:
            self.prepared.append((req.rid, threading.current_thread() is threading.main_thread()))
        return ("setup", req.rid)

    def start(self, req, prepared=None):
        assert prepared == ("setup", req.rid)
        return super().start(req)


@pytest.mark.parametrize("group", [False, True])
def test_host_setup_runs_ahead_on_helper_threads(group):
    be = PreparingBackend()
    srv = S.Server(backend=be, memory_budget=100_000_000, chunk=4, group=group)
    for i in range(6):
        srv.submit(S.RunRequest(i, cfg(32), nsteps=9, arrival=0.002 * i))
    res = srv.run()
    assert [r.state["steps"] for r in res] == [9] * 6
    assert sorted(rid for rid, _ in be.prepared) == list(range(6))   # each prepared once
    assert not any(on_main for _, on_main in be.prepared)             # never on the loop's thread


@pytest.mark.parametrize("group", [False, True])
def test_cancelled_runs_leave_at_a_step_boundary(group):
    be = FakeBackend(lag=1)
    t = [0.0]
    srv = S.Server(backend=be, memory_budget=100_000_000, chunk=3, group=group)

    def clock():
        t[0] += 0.001
        if abs(t[0] - 0.010) < 5e-4:
            srv.cancel(1)            # active by now: leaves at its next boundary
        return t[0]

    for i in range(4):
        srv.submit(S.RunRequest(i, cfg(32), nsteps=30, arrival=0.0 if i < 3 else 0.5))
    srv.cancel(3)                    # still queued: never started
    res = {r.rid: r for r in srv.run(clock=clock, idle_sleep=0.0)}
    assert res[3].cancelled and res[3].nsteps == 0 and res[3].state is None
    assert ("start", 3) not in be.log
    assert res[1].cancelled and 0 < res[1].nsteps < 30 and ("abort", 1) in be.log
    assert [res[i].state["steps"] for i in (0, 2)] == [30, 30] and not res[0].cancelled
    assert be.in_use == 0
    s = S.summary(list(res.values()), srv.elapsed)
    assert s["runs"] == 2 and s["cancelled"] == 2
    pts = [r.points for r in res.values()][0]
    # throughput of completed runs only; the cancelled run's partial steps apart
    assert s["pt_steps_per_s"] * srv.elapsed == pytest.approx(pts * 60)
    assert s["cancelled_pt_steps_per_s"] * srv.elapsed == pytest.approx(pts * res[1].nsteps)
