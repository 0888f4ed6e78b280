#!/usr/bin/env python
"""Throughput of the LSBFLOW time step on B200, in grid-point-steps per second.

Workload: the 256 x 129 x 64 dynamic-Smagorinsky LES (reference axes: nx = 256
streamwise, ny = 64 spanwise, nz = 128 -> nzp = 129 Chebyshev points), 3/2-rule
dealiased products (padded grid 384 x 96), fringe forcing, ceiling dipole suction,
FP64, fixed dt = 0.005, seeded divergence-free noise of amplitude 5e-3 (synthetic:
the reference ships no restart file for this case).  One "step" is one call of the
reference's timestep(); value = nx*ny*nzp*steps*N / (max over ranks of the device
time), inputs resident in HBM (the state, 24 FP64 fields = 405 MB, is larger than L2).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With N > 1 (torchrun) every rank advances its own independent run (replicas: the
path has no exchange step), so the job's throughput is the sum over ranks.

Beside the headline the line carries the mixed-precision form of the same workload, a
Poisson serving stream, and the batched ensemble (64 sigma-model members at 128 x 32 x 65
with their own Re_delta*, dipole amplitude and position, stepped together with one CUDA
graph launch per ensemble step) in both precisions.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from lsbflow_b200 import hostsetup as hs  # noqa: E402
from lsbflow_b200 import ic  # noqa: E402
from lsbflow_b200.config import workload  # noqa: E402

WORKLOAD = "les256"
METRIC = "grid-point-steps/s (FP64 dynamic-Smagorinsky LES time step; mixed form beside it)"
UNIT = "pt-steps/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """SM clock and throttle-reason samples taken during the timed region: NVML read every
    5 ms from a helper thread when the library is there, else nvidia-smi every 20 ms.  Both
    only read the GPU's state."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    # NVML clock-event reason bits of those names
    BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20, "sw_power_cap": 0x4}

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (time, sm_mhz, sm_max_mhz, set of active reason names)
        self._stop = threading.Event()
        self._proc = None
        self._t = None
        self.source = None

    def __enter__(self):
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.index)
            mx = float(N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM))
            get_reasons = getattr(N, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                N.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while not self._stop.is_set():
                    try:
                        sm = float(N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM))
                        bits = int(get_reasons(h))
                        act = {n for n, b in self.BITS.items() if bits & b}
                        self.samples.append((time.perf_counter(), sm, mx, act))
                    except Exception:
                        pass
                    time.sleep(0.005)

            self._t = threading.Thread(target=poll, daemon=True)
            self._t.start()
            self.source = "nvml, every 5 ms"
            return self
        except Exception:
            pass
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "20"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            self.source = "nvidia-smi, every 20 ms"
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                try:
                    sm, mx = float(parts[1]), float(parts[2])
                except ValueError:
                    continue
                act = {n for n, v in zip(self.NAMES, parts[5:9]) if v.lower() == "active"}
                self.samples.append((time.perf_counter(), sm, mx, act))

    def wait_first(self, timeout_s: float = 5.0):
        """Block until the first sample arrived, so the timed region is covered."""
        t0 = time.perf_counter()
        while self._t is not None and not self.samples and time.perf_counter() - t0 < timeout_s:
            time.sleep(0.002)

    def mark(self, start: bool):
        if start:
            self.t_start = time.perf_counter()
        else:
            self.t_end = time.perf_counter()

    def __exit__(self, *exc):
        self._stop.set()
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._t is not None:
            self._t.join(timeout=2)

    def summary(self):
        t0, t1 = getattr(self, "t_start", 0.0), getattr(self, "t_end", float("inf"))
        inside = [s for s in self.samples if t0 <= s[0] <= t1]
        if not inside:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "source": self.source}
        sm = [s[1] for s in inside]
        reasons = sorted(set().union(*[s[3] for s in inside]))
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(s[2] for s in inside), "reasons": reasons,
                "samples": len(inside), "source": self.source}


CPU_KIND = "port"
CPU_WHAT = "the C++/OpenMP restatement of the reference's FP64 step (oracle/cpu_step.cpp)"


def cpu_reference_step_time(cfg, max_steps: int, budget_s: float, warmup: int, threads: int):
    """Seconds per step of the C++/OpenMP restatement of the reference's FP64 step
    (oracle/cpu_step.cpp, parity-tested against the NumPy oracle) on ``threads`` host
    threads, and the steps timed: a bounded sample of at most ``max_steps`` steps, fewer
    when a probe step says they would take longer than ``budget_s``."""
    from oracle import cpu_baseline as CB
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 0, 5e-3)
    probe, _ = CB.run(st, u, v, w, max(1, warmup), threads, want_state=False)
    per = probe / max(1, warmup)
    n = int(max(1, min(max_steps, budget_s / max(per, 1e-9))))
    sec, _ = CB.run(st, u, v, w, n, threads, want_state=False)
    return sec / n, n


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    pts = cfg.nx * cfg.ny * cfg.nzp
    warm = max(1, min(args.warmup, 3))
    t_step, n = cpu_reference_step_time(cfg, args.steps, 120.0, warm, threads)
    val = pts / t_step
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": n, "warmup": warm, "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{WORKLOAD}: 256x64x129 (ref nx,ny,nzp), padded 384x96, dyn-Smagorinsky LES, "
                               f"dealias 3/2, fringe, dipole BC, dt={cfg.dt_fixed}"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": CPU_KIND,
                         "sample": f"{n} full time steps of the same workload with {CPU_WHAT} on {threads} threads"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (Fortran + MPI + FFTW + LAPACK) cannot be built here; its restatement is timed",
    }
    print(json.dumps(line), flush=True)


ROW_NL_PROFILE = os.path.join(ROOT, "profiles", "row_nl_les256_fp64.txt")


def profiled_traffic(path: str):
    """DRAM bytes per launch of the dominant kernel from its committed ncu summary."""
    try:
        with open(path) as f:
            for line in f:
                if line.startswith("dram_bytes_per_launch:"):
                    return float(line.split(":", 1)[1].split()[0])
    except OSError:
        pass
    return None


def same_results(st, sched, nsteps=4):
    """Whether ``sched`` and the built-in models give identical states after a few steps from
    the same seeded field on this grid (every schedule should: none reorders a sum)."""
    from lsbflow_b200 import lib

    u, v, w = ic.seeded_noise(st, 99, 5e-3)
    out = []
    for s_ in ({}, sched):
        s = lib.Solver(st)
        try:
            s.set_schedule(s_)
            s.upload(u, v, w, dt=st.dt)
            s.step(nsteps)
            out.append(s.download())
        finally:
            s.close()
    return all(np.array_equal(out[0][k], out[1][k]) for k in ("uf", "vf", "wf", "pf"))


def tune_schedule(args, st, sol):
    """Times the launch-schedule candidates on this GPU (lsbflow_b200.autotune) and applies
    the fastest to ``sol`` once it is shown to give the models' results bit for bit on this
    grid; returns what was found, or why not."""
    if args.no_tune:
        return None
    try:
        from lsbflow_b200 import autotune as A
        measure, close = A.gpu_measurer(st, steps=10, reps=2)
        try:
            res = A.tune(st.cfg, measure)
        finally:
            close()
        out = {"schedule": res["schedule"], "model_ms_per_step": round(res["model_ms_per_step"], 4),
               "tuned_ms_per_step": round(res["ms_per_step"], 4), "trials": len(res["trials"])}
        if any(res["schedule"].values()):
            out["bit_identical_to_model"] = same_results(st, res["schedule"])
            if not out["bit_identical_to_model"]:
                out["applied"] = False
                return out
        sol.set_schedule(res["schedule"])
        out["applied"] = True
        return out
    except Exception as e:  # the models' schedule stays
        return {"error": f"{type(e).__name__}: {e}"}


def run_serving(args, rank):
    """The survey's serving stream through the request loop: Poisson arrivals (4/s) of runs
    on 64x16x65, 128x32x97 and 256x64x129 grids with no SGS model or the static, dynamic,
    sigma or interscale model, Re_delta*, dipole amplitude and position drawn per run, and
    horizons of 300-3000 steps; the same stream in FP64 and in the mixed form, each run on
    its own stream, and the FP64 stream again with same-shape runs stepped as one ensemble
    batch."""
    from lsbflow_b200 import serving as S

    def one(precision, group=False):
        reqs = S.stream_requests(args.serve_runs, 4.0, 11 + rank, precision=precision)
        srv = S.Server(chunk=50, group=group)
        for r in reqs:
            srv.submit(r)
        res = srv.run()
        summ = S.summary(res, srv.elapsed)
        return {"runs": summ["runs"], "runs_per_hour": round(summ["runs_per_hour"], 1),
                "p50_s": round(summ["p50"], 4), "p99_s": round(summ["p99"], 4),
                "pt_steps_per_s": summ["pt_steps_per_s"], "elapsed_s": round(summ["elapsed_s"], 3)}

    serving = {"arrivals": "Poisson 4/s, seeded",
               "mix": "grids 64x16x65 / 128x32x97 / 256x64x129 (ref nx,ny,nzp) x SGS none / static / dynamic / "
                      "sigma / interscale, Re_d* ~ U[300,800], A ~ U[0.1,0.4], x0 ~ U[60,100] d*",
               "horizon_steps": [300, 3000]}
    serving["fp64"] = one(0)
    try:
        serving["mixed"] = one(1)
    except Exception as e:  # reported in the line; the FP64 numbers above stand
        serving["mixed"] = {"error": f"{type(e).__name__}: {e}"}
    try:
        serving["fp64_grouped"] = one(0, group=True)
    except Exception as e:
        serving["fp64_grouped"] = {"error": f"{type(e).__name__}: {e}"}
    return serving


def run_profiles(args, st, u, v, w, stream):
    """Spanwise mean and rms profiles of u + ubar, v, w, p (per z and x, as run/spanwiseavg.m
    averages q snapshots over y), averaged in time over the second half of a long run, for
    the FP64 and the mixed form from the same initial field; the relative L2 difference of
    the mixed form's profiles from the FP64 ones per field."""
    from lsbflow_b200 import lib

    nsteps = max(20, args.profile_steps)
    every = 20
    out = {}
    first_nonfinite = {}
    umax = {}
    for prec in (0, 1):
        s = lib.Solver(hs.make_setup(st.cfg.replace(precision=prec)) if prec else st)
        s.set_stream(stream.cuda_stream)
        s.upload(u, v, w, dt=st.dt)
        acc_m = acc_r = None
        n = 0
        done = 0
        bad = None
        while done < nsteps:
            s.step(every)
            done += every
            if done % 100 == 0 or done >= nsteps:
                d = s.diag()  # NaN check of the resident state (maxcalc's reductions)
                umax.setdefault(prec, []).append(round(d["umax"], 4))
                if d["nonfinite"] and bad is None:
                    bad = done
                    break
            if done > nsteps // 2:
                m, r = s.spanwise_stats()
                acc_m = m if acc_m is None else acc_m + m
                acc_r = r if acc_r is None else acc_r + r
                n += 1
        s.close()
        first_nonfinite["fp64" if prec == 0 else "mixed"] = bad
        if bad is not None or n == 0:
            return {"steps": nsteps, "first_nonfinite_step": first_nonfinite, "error": "the run went non-finite"}
        out[prec] = (acc_m / n, acc_r / n, n)
    (m0, r0, n), (m1, r1, _) = out[0], out[1]
    names = ("u", "v", "w", "p")

    def rel(a, b):
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))

    em = {names[k]: rel(m1[k], m0[k]) for k in range(4)}
    er = {names[k]: rel(r1[k], r0[k]) for k in range(4)}
    return {"steps": nsteps, "average": f"steps {nsteps // 2 + every}..{nsteps}, every {every} ({n} samples)",
            "first_nonfinite_step": first_nonfinite,
            "umax_every_100_steps": {"fp64": umax[0][::4], "mixed": umax[1][::4]},
            "rel_err_mean": em, "rel_err_rms": er,
            "max_rel_err_mean_velocity": max(em[k] for k in "uvw"),
            "max_rel_err_rms_velocity": max(er[k] for k in "uvw"), "target": 1e-4}


def run_os_growth(args, stream):
    """The 128 x 4 x 97 Orr-Sommerfeld linear test (Re_delta* = 1000, alpha delta* = 0.25,
    dt = 0.005): the Tollmien-Schlichting mode of the host Orr-Sommerfeld solve stepped
    500 times in FP64 and in the mixed form, the perturbation energy taken every step
    (lintest, src/orrsomm.f90:566-622), and the mean growth rate <dE/dt> of each against
    the mode's omega_i."""
    from lsbflow_b200 import lib
    from lsbflow_b200 import linstab as L

    nsteps = 500
    out = {"grid": "128x4x97 (ref nx,ny,nzp)", "steps": nsteps}
    for prec, name in ((0, "fp64"), (1, "mixed")):
        st = hs.make_setup(workload("os128", precision=prec))
        z = np.zeros((st.grid.nzp, st.cfg.ny, st.cfg.nx))
        uf, vf, wf = z.copy(), z.copy(), z.copy()
        mode = L.setup_linstab(st, uf, vf, wf)
        s = lib.Solver(st)
        s.set_stream(stream.cuda_stream)
        s.upload(uf, vf, wf, dt=st.dt)
        e = []
        for _ in range(nsteps):
            s.step(1)
            e.append(s.diag()["energy_pert"])
        s.close()
        g = L.mean_growth(L.growth_rates(np.array(e), st.dt))
        out["omega_i"] = mode.omega.imag
        out[name] = {"mean_growth": g, "rel_err_vs_omega_i": abs(g - mode.omega.imag) / abs(mode.omega.imag)}
    out["mixed_rel_err_vs_fp64"] = abs(out["mixed"]["mean_growth"] - out["fp64"]["mean_growth"]) / abs(
        out["fp64"]["mean_growth"])
    return out


def run_ensemble(args, rank, world, stream, max_over_ranks, barrier):
    """Members of the 128 x 32 x 64 (nzp 65) sigma-model ensemble (Re_delta* ~ U[300, 800],
    A ~ U[0.1, 0.4], x0 ~ U[60, 100] delta*, noise 1e-3, seeds s0 + m) stepped together
    through lsb_batch_step, in both precisions; beside it one member stepped alone."""
    import torch
    from lsbflow_b200 import lib, replicas
    from lsbflow_b200.config import ensemble_configs

    out = {"members": 0, "grid": "128x32x65 (ref nx,ny,nzp), padded 192x48", "model": "sigma",
           "draws": "Re_d* ~ U[300,800], A ~ U[0.1,0.4], x0 ~ U[60,100] d*, noise 1e-3, seeds s0+m"}
    steps = max(6, min(args.steps, 30))
    for prec, name in ((0, "fp64"), (1, "mixed")):
        cfgs = ensemble_configs(args.members, seed=3000 + rank, precision=prec)
        sols = []
        free = torch.cuda.mem_get_info()[0]
        def prep(m):  # host-only set-up and initial field, on helper threads
            st = hs.make_setup(cfgs[m])
            return st, ic.seeded_noise(st, replicas.replica_seed(5000 + m, rank), 1e-3)

        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as pool:
            prepared = list(pool.map(prep, range(len(cfgs))))
        for m, (st, (u, v, w)) in enumerate(prepared):
            s = lib.Solver(st)
            s.upload(u, v, w, dt=st.dt)
            sols.append(s)
            if m == 0 and s.device_bytes() * len(cfgs) > 0.8 * free:
                raise RuntimeError("ensemble does not fit in device memory")
        pts_m = cfgs[0].nx * cfgs[0].ny * cfgs[0].nzp
        b = lib.Batch(sols)
        b.set_stream(stream.cuda_stream)
        b.step(max(args.warmup, 3) + 6)  # start-up steps, then the 6 ensemble graphs are captured
        torch.cuda.synchronize()
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        n0 = lib.kernel_launches()
        e0.record(stream)
        b.step(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        launches = lib.kernel_launches() - n0
        ms = max_over_ranks(e0.elapsed_time(e1))
        b.close()
        # every member's velocity after the batch's steps, for the mixed form's error per member
        finals = [s_.download() for s_ in sols]
        vel = [np.concatenate([o_[k].ravel() for k in ("uf", "vf", "wf")]) for o_ in finals]
        if prec == 0:
            ref_vel = vel
        else:
            errs = [float(np.linalg.norm(a - b_) / np.linalg.norm(b_)) for a, b_ in zip(vel, ref_vel)]
            out["mixed_rel_err_velocity_per_member"] = {
                "steps": max(args.warmup, 3) + 6 + steps, "max": max(errs), "median": float(np.median(errs)),
                "min": min(errs), "members": [round(e_, 9) for e_ in errs],
                "note": "sigma-model members: the model's trigonometric singular values are ill-conditioned "
                        "near equal singular values, so FP32 inputs move them far more than FP32 rounding"}
        # one member alone on the same stream (its own step graphs)
        s0 = sols[0]
        s0.set_stream(stream.cuda_stream)
        s0.step(6)  # its own 6 step graphs are captured
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        s0.step(steps)
        a1.record(stream)
        torch.cuda.synchronize()
        ms1 = max_over_ranks(a0.elapsed_time(a1))
        for s in sols:
            s.close()
        agg = replicas.job_throughput(pts_m * len(cfgs), steps, world, ms / 1e3)
        one = replicas.job_throughput(pts_m, steps, world, ms1 / 1e3)
        out["members"] = len(cfgs)
        out[name] = {"value": agg, "unit": UNIT, "ms_per_ensemble_step": ms / steps,
                     "single_member_value": one, "gain_vs_one_member": agg / one,
                     "gpu_launches_per_ensemble_step": launches / steps, "timed_steps": steps}
    out["mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=300)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1],
                    help="form of the headline handle: 0 FP64 (the benchmark), 1 the mixed form (for "
                         "profiling the mixed step alone)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--serve-runs", type=int, default=12)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-profiles", action="store_true")
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--profile-steps", type=int, default=2000)
    ap.add_argument("--members", type=int, default=64)
    args = ap.parse_args()
    cfg = workload(args.workload, precision=args.precision) if args.impl != "reference" else workload(args.workload)
    if args.impl == "reference":
        run_reference(args, cfg)
        return

    import torch
    import torch.distributed as dist
    from lsbflow_b200 import lib, replicas

    rank, world, local = replicas.rank_info()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, world, device="cuda")

    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, replicas.replica_seed(1000, rank), 5e-3)
    sol = lib.Solver(st)
    stream = torch.cuda.Stream()
    sol.set_stream(stream.cuda_stream)
    sol.upload(u, v, w, dt=st.dt)
    pts = cfg.nx * cfg.ny * cfg.nzp
    # launch schedule picked by the tuner (part of set-up, like an FFT planner; every
    # schedule gives the same results); the models' choice if tuning is off or fails
    schedules = {"fp64": tune_schedule(args, st, sol)}

    # ---- warm-up
    sol.step(args.warmup)
    torch.cuda.synchronize()

    # ---- device-resident timed region (CUDA events on the library's stream)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        clk.wait_first()
        barrier()
        torch.cuda.synchronize()
        clk.mark(True)
        n0 = lib.kernel_launches()
        ev0.record(stream)
        sol.step(args.steps)
        ev1.record(stream)
        launches = lib.kernel_launches() - n0
        torch.cuda.synchronize()
        clk.mark(False)
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1))
    value = replicas.job_throughput(pts, args.steps, world, ms / 1e3)
    clocks = clk.summary()

    # ---- per kernel-group timing (same workload, separate region with event timers on)
    sol.timers(True)
    sol.step(min(args.steps, 40))
    torch.cuda.synchronize()
    rep = sol.timer_report()
    sol.timers(False)
    # sgs_filter3 runs inside sgs_total: the step total counts it once
    tot = sum(v[1] for k, v in rep.items() if k != "sgs_filter3")
    groups = {k: {"launches": v[0], "ms_total": round(v[1], 4), "share": round(v[1] / tot, 4)}
              for k, v in rep.items()}

    # ---- roofline of the dominant kernel, the fused nonlinear-product row pass (k_row_nl):
    # per (z, y) row of the padded y-intermediate grid it reads 9 rows of kx modes
    # (u_l, du_l/dy, du_l/dz) and writes 9 (3 convective terms, 6 fluxes), nx doubles each
    hbm, hbm_kind = peaks()
    nx, ny, nzp = cfg.nx, cfg.ny, cfg.nzp
    nxl, nyl = st.nx_lg, st.ny_lg
    S8 = nx * ny * nzp * 8
    alg_bytes = 18 * nx * nyl * nzp * 8
    n_nl, ms_nl = rep["row_nl"]
    per_launch_ms = ms_nl / max(n_nl, 1)
    achieved = alg_bytes / (per_launch_ms / 1e3) / 1e9
    roofline = {"kernel": "k_row_nl_r (fused 12 c2r + skew-symmetric products + 9 r2c)", "bound": "hbm",
                "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "peak_kind": hbm_kind, "traffic": profiled_traffic(ROW_NL_PROFILE),
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": round(per_launch_ms, 4),
                "share_of_step": round(ms_nl / tot, 4)}

    # ---- step-level rooflines (the survey's per-grid-point-step figures): compulsory state
    # traffic, 24 FP64 spectral fields read or written once per step (u, v, w, p, p^{n-1},
    # 2 velocity and 2 nonlinear histories read, u, v, w, p, N^n written), and the
    # contraction work, 11 nzp x nzp derivative and 10 nzm x nzm eigenbasis applications per
    # column, against the step time
    nzm = nzp - 2
    state_b = 24 * 8
    flop_c = 2.0 * (11 * nzp + 10 * nzm * nzm / nzp)
    t_step = ms / args.steps / 1e3
    step_roofline = {"state_bytes_per_pt_step": state_b, "contraction_flop_per_pt_step": round(flop_c, 1),
                     "achieved_state_GBs": round(state_b * pts / t_step / 1e9, 1),
                     "state_frac_of_hbm": round(state_b * pts / t_step / 1e9 / hbm, 4),
                     "achieved_contraction_TFLOPs": round(flop_c * pts / t_step / 1e12, 3),
                     "note": "the step moves far more than its state: the padded-grid transforms and "
                             "SGS fields are intermediate traffic; the kernel rooflines explain the time"}

    # ---- end-to-end through the C ABI with host buffers (pinned): per step the velocity
    # (u, v, w) goes host->device, one time step runs, the new velocity comes back.
    hb = [torch.empty(pts, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    for i, f in enumerate((u, v, w)):
        hb[i].copy_(torch.from_numpy(np.ascontiguousarray(f).ravel()))
    e2e_steps = max(3, min(args.steps, 100))
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sol.upload_velocity_ptr(hb[0].data_ptr(), hb[1].data_ptr(), hb[2].data_ptr())
        sol.step(1)
        sol.download_velocity_ptr(hb[0].data_ptr(), hb[1].data_ptr(), hb[2].data_ptr())
    sol.synchronize()
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_val = replicas.job_throughput(pts, e2e_steps, world, e2e_s)

    # ---- the mixed-precision form on the same workload: throughput and its error against
    # the FP64 form after 100 steps from the same initial field
    mixed = None
    if not args.no_mixed:
        cfg_m = cfg.replace(precision=1)
        st_m = hs.make_setup(cfg_m)
        sm = lib.Solver(st_m)
        schedules["mixed"] = tune_schedule(args, st_m, sm)
        sm.set_stream(stream.cuda_stream)
        sm.upload(u, v, w, dt=st.dt)
        sm.step(args.warmup)
        torch.cuda.synchronize()
        barrier()
        em0 = torch.cuda.Event(enable_timing=True)
        em1 = torch.cuda.Event(enable_timing=True)
        em0.record(stream)
        sm.step(args.steps)
        em1.record(stream)
        torch.cuda.synchronize()
        ms_m = max_over_ranks(em0.elapsed_time(em1))
        # per kernel-group timing of the mixed step (event timers on, separate region)
        sm.timers(True)
        sm.step(min(args.steps, 40))
        torch.cuda.synchronize()
        rep_m = sm.timer_report()
        sm.timers(False)
        tot_m = sum(v[1] for k, v in rep_m.items() if k != "sgs_filter3")
        groups_m = {k: {"launches": v[0], "ms_total": round(v[1], 4), "share": round(v[1] / tot_m, 4)}
                    for k, v in rep_m.items()}
        nerr = 100
        sm.upload(u, v, w, dt=st.dt)
        sm.step(nerr)
        got = sm.download()
        sm.close()
        sref = lib.Solver(st)
        sref.set_stream(stream.cuda_stream)
        sref.upload(u, v, w, dt=st.dt)
        sref.step(nerr)
        ref = sref.download()
        sref.close()

        def rel(a, b):
            return float(np.linalg.norm(a - b) / np.linalg.norm(b))

        vg = np.concatenate([got[k].ravel() for k in ("uf", "vf", "wf")])
        vr = np.concatenate([ref[k].ravel() for k in ("uf", "vf", "wf")])
        mixed = {"value": replicas.job_throughput(pts, args.steps, world, ms_m / 1e3), "unit": UNIT,
                 "ms_per_step": ms_m / args.steps, "speedup_vs_fp64": (ms / args.steps) / (ms_m / args.steps),
                 "rel_err_velocity_after_100_steps": rel(vg, vr),
                 "rel_err_components": {k: rel(got[k], ref[k]) for k in ("uf", "vf", "wf", "pf")},
                 "kernel_groups": groups_m,
                 "form": "FP32 transforms, products, physical fields and SGS; z derivatives of the nonlinear "
                         "term and velocity Helmholtz solves on the int8 tensor cores (5 digits per operand, "
                         "exact int32 accumulation); FP64 state, time integration, boundary conditions, "
                         "Poisson solve, pressure and projection"}

    # ---- mean / rms profiles of the mixed form against FP64 after a long run
    profiles = None
    if not args.no_mixed and not args.no_profiles:
        try:
            profiles = run_profiles(args, st, u, v, w, stream)
        except Exception as e:  # reported in the line; the headline stands on its own
            profiles = {"error": f"{type(e).__name__}: {e}"}

    # ---- the Orr-Sommerfeld linear test: growth rate in both forms against omega_i
    os_growth = None
    if not args.no_mixed:
        try:
            os_growth = run_os_growth(args, stream)
        except Exception as e:  # reported in the line; the headline stands on its own
            os_growth = {"error": f"{type(e).__name__}: {e}"}

    # ---- serving: a Poisson stream of ensemble runs (continuous batching on this GPU)
    serving = None
    if not args.no_serving:
        try:
            serving = run_serving(args, rank)
        except Exception as e:  # reported in the line; the headline stands on its own
            serving = {"error": f"{type(e).__name__}: {e}"}

    # ---- batched ensemble: sigma-model LES members of one grid with their own Re_delta*,
    # dipole amplitude and position, stepped together (one graph launch per ensemble step)
    ensemble = None
    if not args.no_ensemble:
        try:
            ensemble = run_ensemble(args, rank, world, stream, max_over_ranks, barrier)
        except Exception as e:  # reported in the line; the headline above stands on its own
            ensemble = {"error": f"{type(e).__name__}: {e}"}

    # ---- the CPU baseline (rank 0, N = 1 only), bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t_step, n = cpu_reference_step_time(cfg, 10, 20.0, 1, threads)
        cpu = {"value": pts / t_step, "unit": UNIT, "cores": threads, "kind": CPU_KIND,
               "sample": f"{n} time step(s) of the same {nx}x{ny}x{nzp} workload with {CPU_WHAT} on "
                         f"{threads} threads"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64" if args.precision == 0 else "mixed (f32 / int8 tensor cores / f64)",
            "data": "synthetic",
            "config": {"workload": f"{args.workload}: {nx}x{ny}x{nzp} (ref nx,ny,nzp), padded {nxl}x{nyl}, "
                                   f"dyn-Smagorinsky LES, dealias 3/2, fringe, dipole BC, dt={st.dt}",
                       "global_batch": world, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (resident state 24 fields x 17 MB = 405 MB)"},
            "roofline": roofline,
            "step_roofline": step_roofline,
            "schedules": schedules,
            "kernel_groups": groups,
            "clocks": clocks,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 3 * S8, "d2h_bytes_per_step": 3 * S8},
            "gpu_launches": launches,
            "cpu_baseline": cpu,
            "mixed": mixed,
            "serving": serving,
            "ensemble": ensemble,
            "profiles": profiles,
            "os_growth": os_growth,
        }
        print(json.dumps(line), flush=True)
    sol.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
