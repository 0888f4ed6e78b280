"""Request loop for ensemble runs on one GPU (continuous batching of independent runs).

Each admitted run is one library handle on its own CUDA stream; its state stays resident in
HBM from admission to result.  The loop works at step boundaries:

* admission -- queued requests that have arrived are admitted, oldest first, while the
  sum of device footprints stays inside the memory budget and a slot is free.  The
  footprint of a (grid, model) shape is the measured ``lsb_device_bytes`` of the first
  handle of that shape; before one exists it is estimated as 64 spectral fields.
* stepping -- every active run has at most one chunk of ``chunk`` steps in flight on its
  stream; when a chunk's event has completed the next chunk is queued, so runs of
  different sizes advance concurrently and kernels of different streams overlap.
* completion -- a run that has done its steps is downloaded, its handle freed, and its
  slot and memory go to the next arrival.
* set-up ahead of admission -- when a backend has ``prepare`` (the host-only part of
  starting a run: grid, matrices, base flow, initial field), arrived requests are prepared
  on helper threads while the loop keeps stepping, so admission only creates the handle
  and uploads the state.

With ``group=True`` the runs of one shape (grid, model, dealiasing, averaging) form a
cohort stepped through one ensemble batch (``lsb_batch_step``: one CUDA graph launch per
ensemble step once the members are steady): at each cohort boundary finished runs leave,
newly admitted runs of that shape join, and the cohort advances by the smallest of the
chunk and its members' remaining steps.  A change of membership makes a new batch, whose
ensemble graphs are captured over its next steps.

Results do not depend on what else runs: handles share no device memory and every kernel
of a run is on that run's stream.  ``percentiles`` gives p50/p99 of time-to-result
(completion minus arrival) and the loop reports runs per hour and grid-point-steps/s.
"""
from __future__ import annotations

import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .config import LsbConfig


@dataclass
class RunRequest:
    rid: int
    cfg: LsbConfig
    nsteps: int
    seed: int = 0
    amp: float = 1e-3
    arrival: float = 0.0          # seconds after the loop starts


@dataclass
class RunResult:
    rid: int
    state: dict
    arrival: float
    admitted: float
    done: float
    nsteps: int                 # steps done (fewer than requested for a cancelled run)
    points: int
    cancelled: bool = False     # stopped by Server.cancel; state is None

    @property
    def time_to_result(self) -> float:
        return self.done - self.arrival


def shape_key(cfg: LsbConfig):
    return (cfg.nx, cfg.ny, cfg.nz, cfg.dealiasflag, cfg.sgsflag, cfg.sgsmodel, cfg.otfavg)


def estimate_bytes(cfg: LsbConfig) -> int:
    return 64 * cfg.nx * cfg.ny * cfg.nzp * 8


class DeviceBackend:
    """Handles and streams on the current CUDA device (the library's C ABI).  With
    ``schedules`` (a JSON file of lsbflow_b200.autotune) each run gets the launch schedule
    tuned for its shape on this device, if there is one."""

    def __init__(self, schedules: str | None = None):
        import torch  # device plumbing: streams and events
        from . import lib
        self.torch = torch
        self.lib = lib
        self._free, _ = torch.cuda.mem_get_info()
        self.schedules = schedules
        self.device = torch.cuda.get_device_name() if schedules else None

    def schedule_for(self, cfg):
        if not self.schedules:
            return None
        from . import autotune
        return autotune.lookup(cfg, self.schedules, self.device)

    def free_bytes(self) -> int:
        return int(self._free)

    @staticmethod
    def prepare(req: RunRequest):
        """Host-only set-up of a run (grid, matrices, base flow, initial field); no device
        work, so it can run on a helper thread while the loop steps other runs."""
        from . import hostsetup as hs
        from . import ic
        st = hs.make_setup(req.cfg)
        return st, ic.seeded_noise(st, req.seed, req.amp)

    def start(self, req: RunRequest, prepared=None):
        st, (u, v, w) = prepared if prepared is not None else self.prepare(req)
        s = self.lib.Solver(st)
        sched = self.schedule_for(req.cfg)
        if sched:
            s.set_schedule(sched)
        stream = self.torch.cuda.Stream()
        s.set_stream(stream.cuda_stream)
        s.upload(u, v, w, dt=st.dt)
        return {"solver": s, "stream": stream, "event": None, "bytes": s.device_bytes()}

    def launch(self, run, nsteps: int):
        run["solver"].step(nsteps)
        ev = self.torch.cuda.Event()
        ev.record(run["stream"])
        run["event"] = ev

    def ready(self, run) -> bool:
        return run["event"] is None or run["event"].query()

    # ---- cohorts of same-shape runs stepped as one ensemble batch
    def new_group(self):
        return {"batch": None, "members": (), "event": None, "stream": self.torch.cuda.Stream()}

    def launch_group(self, g, runs, nsteps: int):
        ids = tuple(id(r) for r in runs)
        if g["members"] != ids:
            self.close_group(g)
            g["batch"] = self.lib.Batch([r["solver"] for r in runs])
            g["batch"].set_stream(g["stream"].cuda_stream)
            g["members"] = ids
        g["batch"].step(nsteps)
        ev = self.torch.cuda.Event()
        ev.record(g["stream"])
        g["event"] = ev

    def group_ready(self, g) -> bool:
        return g["event"] is None or g["event"].query()

    def close_group(self, g):
        """Release the cohort's batch (before any member is finished and freed)."""
        if g["batch"] is not None:
            g["batch"].close()
            g["batch"] = None
            g["members"] = ()

    def abort(self, run):
        """Free a cancelled run's handle without downloading its state."""
        run["stream"].synchronize()
        run["solver"].close()

    def finish(self, run) -> dict:
        run["stream"].synchronize()
        state = run["solver"].download()
        run["solver"].close()
        return state


@dataclass
class _Active:
    req: RunRequest
    run: dict
    admitted: float
    remaining: int
    nbytes: int


@dataclass
class Server:
    backend: object = None
    memory_budget: int | None = None     # bytes; default 90% of free device memory
    max_active: int = 32
    chunk: int = 10
    footprints: dict = field(default_factory=dict)
    group: bool = False                  # step same-shape runs as one ensemble batch
    prefetch: int = 2                    # helper threads preparing arrived runs (0: none)
    schedules: str | None = None         # tuned launch schedules (autotune JSON) for new runs

    def __post_init__(self):
        if self.backend is None:
            self.backend = DeviceBackend(schedules=self.schedules)
        if self.memory_budget is None:
            self.memory_budget = int(0.9 * self.backend.free_bytes())
        self.queue: list = []
        self._cancel: set = set()
        self._cancel_lock = threading.Lock()

    def cancel(self, rid: int):
        """Stop run ``rid`` (safe from another thread): a queued run is dropped, an active
        one leaves at its next step boundary and its handle is freed without a download.
        Its result has ``cancelled`` set, ``state`` None and the steps it did."""
        with self._cancel_lock:
            self._cancel.add(rid)

    def _cancelled(self, rid: int) -> bool:
        with self._cancel_lock:
            return rid in self._cancel

    def _drop_cancelled(self, queue, results, now):
        """Cancelled requests still waiting leave the queue with an empty result."""
        for req in [r for r in queue if self._cancelled(r.rid)]:
            queue.remove(req)
            fut = self._prepared.pop(req.rid, None)
            if fut is not None:
                fut.cancel()
            c = req.cfg
            results.append(RunResult(req.rid, None, req.arrival, now, now, 0, c.nx * c.ny * c.nzp, True))

    def _abort(self, a, results, now):
        self.backend.abort(a.run)
        c = a.req.cfg
        results.append(RunResult(a.req.rid, None, a.req.arrival, a.admitted, now, a.req.nsteps - a.remaining,
                                 c.nx * c.ny * c.nzp, True))

    def submit(self, req: RunRequest):
        if req.nsteps <= 0:
            raise ValueError("a run needs at least one step")
        need = self.footprints.get(shape_key(req.cfg), estimate_bytes(req.cfg))
        if need > self.memory_budget:
            raise ValueError(f"run {req.rid} needs {need} bytes, more than the budget {self.memory_budget}")
        self.queue.append(req)

    def _prefetch(self, queue, now):
        """Queue the host set-up of every arrived request not yet being prepared."""
        if self._pool is None:
            return
        for req in queue:
            if req.arrival > now:
                break
            if req.rid not in self._prepared:
                self._prepared[req.rid] = self._pool.submit(self.backend.prepare, req)

    def _start(self, req):
        fut = self._prepared.pop(req.rid, None)
        if fut is None:
            return self.backend.start(req)
        return self.backend.start(req, fut.result())

    def _admit(self, queue, now, n_active, used, t0, clock):
        """Admits arrived requests, oldest first, no overtaking, while a slot and the memory
        budget allow (one run is always admitted when none is active); yields each admitted
        run as an _Active.  ``used`` and ``n_active`` are the caller's totals on entry."""
        self._prefetch(queue, now)
        while queue and queue[0].arrival <= now and n_active < self.max_active:
            req = queue[0]
            need = self.footprints.get(shape_key(req.cfg), estimate_bytes(req.cfg))
            if used + need > self.memory_budget and n_active:
                break
            queue.pop(0)
            run = self._start(req)
            nb = int(run.get("bytes") or need)
            self.footprints[shape_key(req.cfg)] = nb
            used += nb
            n_active += 1
            yield _Active(req, run, clock() - t0, req.nsteps, nb)

    def _result(self, a: _Active, state: dict, done: float) -> RunResult:
        c = a.req.cfg
        return RunResult(a.req.rid, state, a.req.arrival, a.admitted, done, a.req.nsteps, c.nx * c.ny * c.nzp)

    def _wait(self, progressed, busy, queue, clock, t0, idle_sleep):
        if progressed:
            return
        if not busy and queue:
            wait = queue[0].arrival - (clock() - t0)
            if wait > 0:
                time.sleep(min(wait, 0.05))
        else:
            time.sleep(idle_sleep)

    def _run_grouped(self, clock, idle_sleep) -> list:
        queue = sorted(self.queue, key=lambda r: (r.arrival, r.rid))
        self.queue = []
        cohorts: dict = {}   # shape -> {"runs": [...], "joining": [...], "g": backend group}
        results = []
        used = 0
        t0 = clock()

        def n_active():
            return sum(len(c["runs"]) + len(c["joining"]) for c in cohorts.values())

        try:
            while queue or n_active():
                self._drop_cancelled(queue, results, clock() - t0)
                for a in self._admit(queue, clock() - t0, n_active(), used, t0, clock):
                    used += a.nbytes
                    key = shape_key(a.req.cfg)
                    if key not in cohorts:
                        cohorts[key] = {"runs": [], "joining": [], "g": self.backend.new_group()}
                    cohorts[key]["joining"].append(a)
                progressed = False
                for c in cohorts.values():
                    if not (c["runs"] or c["joining"]) or not self.backend.group_ready(c["g"]):
                        continue
                    stop = [a for a in c["runs"] + c["joining"] if self._cancelled(a.req.rid)]
                    done = [a for a in c["runs"] if a.remaining == 0 and a not in stop]
                    if done or stop:
                        self.backend.close_group(c["g"])
                        for a in done:
                            results.append(self._result(a, self.backend.finish(a.run), clock() - t0))
                        for a in stop:
                            self._abort(a, results, clock() - t0)
                        for a in done + stop:
                            (c["runs"] if a in c["runs"] else c["joining"]).remove(a)
                            used -= a.nbytes
                    c["runs"] += c["joining"]
                    c["joining"] = []
                    if c["runs"]:
                        k = min(self.chunk, min(a.remaining for a in c["runs"]))
                        self.backend.launch_group(c["g"], [a.run for a in c["runs"]], k)
                        for a in c["runs"]:
                            a.remaining -= k
                    progressed = progressed or bool(done) or bool(stop) or bool(c["runs"])
                self._wait(progressed, n_active() > 0, queue, clock, t0, idle_sleep)
        finally:
            for c in cohorts.values():
                self.backend.close_group(c["g"])
        self.elapsed = clock() - t0
        return sorted(results, key=lambda r: r.rid)

    def run(self, clock=time.perf_counter, idle_sleep: float = 1e-4) -> list:
        self._prepared = {}
        self._pool = None
        if self.prefetch > 0 and hasattr(self.backend, "prepare"):
            from concurrent.futures import ThreadPoolExecutor
            self._pool = ThreadPoolExecutor(max_workers=self.prefetch)
        try:
            if self.group:
                return self._run_grouped(clock, idle_sleep)
            return self._run_plain(clock, idle_sleep)
        finally:
            if self._pool is not None:
                self._pool.shutdown(wait=True)
            self._pool = None

    def _run_plain(self, clock, idle_sleep) -> list:
        queue = sorted(self.queue, key=lambda r: (r.arrival, r.rid))
        self.queue = []
        active: list = []
        results = []
        used = 0
        t0 = clock()
        while queue or active:
            self._drop_cancelled(queue, results, clock() - t0)
            # admission at a step boundary, oldest arrival first, no overtaking
            for a in self._admit(queue, clock() - t0, len(active), used, t0, clock):
                used += a.nbytes
                active.append(a)
            progressed = False
            for a in list(active):
                if not self.backend.ready(a.run):
                    continue
                if self._cancelled(a.req.rid):
                    self._abort(a, results, clock() - t0)
                    active.remove(a)
                    used -= a.nbytes
                    progressed = True
                elif a.remaining > 0:
                    k = min(self.chunk, a.remaining)
                    self.backend.launch(a.run, k)
                    a.remaining -= k
                    progressed = True
                else:
                    results.append(self._result(a, self.backend.finish(a.run), clock() - t0))
                    active.remove(a)
                    used -= a.nbytes
                    progressed = True
            self._wait(progressed, bool(active), queue, clock, t0, idle_sleep)
        self.elapsed = clock() - t0
        return sorted(results, key=lambda r: r.rid)


def percentiles(results, qs=(50, 99)) -> dict:
    """p50/p99 of time-to-result over the runs that completed (cancelled runs excluded)."""
    ttr = np.array([r.time_to_result for r in results if not r.cancelled])
    if ttr.size == 0:
        return {f"p{q}": float("nan") for q in qs}
    return {f"p{q}": float(np.percentile(ttr, q)) for q in qs}


def summary(results, elapsed: float) -> dict:
    """runs, runs/h, p50/p99 and pt_steps_per_s count completed runs only; the grid-point
    steps that cancelled runs took before they stopped are reported apart
    (cancelled_pt_steps_per_s)."""
    out = percentiles(results)
    done = [r for r in results if not r.cancelled]
    out["runs"] = len(done)
    out["cancelled"] = len(results) - len(done)
    out["runs_per_hour"] = len(done) / elapsed * 3600.0
    out["pt_steps_per_s"] = sum(r.points * r.nsteps for r in done) / elapsed
    out["cancelled_pt_steps_per_s"] = sum(r.points * r.nsteps for r in results if r.cancelled) / elapsed
    out["elapsed_s"] = elapsed
    return out


# the serving mix of the survey's stream: grids (reference nx x ny x nzp) and SGS models
STREAM_GRIDS = (("dns64", {}), ("ens128", {"nz": 96}), ("les256", {}))   # 64x16x65, 128x32x97, 256x64x129
STREAM_MODELS = ((0, 0), (1, 0), (1, 1), (1, 2), (1, 3))  # (sgsflag, sgsmodel): none, static, dynamic, sigma,
                                                          # interscale (src/sgsterm.f90:21-35)


def stream_requests(n: int, rate: float, seed: int, precision: int = 0, steps_range=(300, 3000)) -> list:
    """Poisson arrivals at ``rate`` per second of runs with the grid drawn uniformly from
    64 x 16 x 65, 128 x 32 x 97 and 256 x 64 x 129, the SGS model from none, static and
    dynamic Smagorinsky, sigma and interscale, Re_delta* ~ U[300, 800], ceiling-dipole
    amplitude A ~ U[0.1, 0.4] and centre x0 ~ U[60, 100] displacement thicknesses, and a
    horizon drawn uniformly from ``steps_range``; every run in ``precision`` (0 FP64, 1 mixed)."""
    from .config import workload
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        base, over = STREAM_GRIDS[int(rng.integers(len(STREAM_GRIDS)))]
        sgsflag, sgsmodel = STREAM_MODELS[int(rng.integers(len(STREAM_MODELS)))]
        re_d, amp, xc = rng.uniform(300.0, 800.0), rng.uniform(0.1, 0.4), rng.uniform(60.0, 100.0)
        nsteps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        cfg = workload(base, re_d=float(re_d), bc_amp=float(amp), bc_xc=float(xc), sgsflag=sgsflag,
                       sgsmodel=sgsmodel, precision=precision, **over)
        out.append(RunRequest(i, cfg, nsteps, seed=1000 + i, amp=1e-3, arrival=t))
    return out


def poisson_requests(n: int, rate: float, seed: int, shapes, steps_range=(300, 3000)) -> list:
    """Poisson arrivals at ``rate`` per second, each drawing a grid/model from ``shapes``
    and a horizon uniformly from ``steps_range``."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        cfg = shapes[int(rng.integers(len(shapes)))]
        out.append(RunRequest(i, cfg, int(rng.integers(steps_range[0], steps_range[1] + 1)), seed=1000 + i,
                              amp=1e-3, arrival=t))
    return out
