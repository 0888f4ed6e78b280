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
METRIC = "grid-point-steps/s (FP64 dynamic-Smagorinsky LES time step)"
UNIT = "pt-steps/s"


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None
        return self

    def _read(self):
        for line in self._proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self._proc is not None:
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for s in self.samples for n, v in zip(names, s[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def cpu_reference_step_time(cfg, max_steps: int, budget_s: float, warmup: int, threads: int):
    """The FP64 oracle (a NumPy restatement of the reference's step) on the host cores."""
    from oracle import lsb_oracle as O
    O.WORKERS = threads
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 0, 5e-3)
    s = O.State.zeros_like(st, u, v, w, st.dt)
    for _ in range(warmup):
        O.timestep(st, s)
    times = []
    t_all = time.perf_counter()
    for _ in range(max_steps):
        t0 = time.perf_counter()
        O.timestep(st, s)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all > budget_s:
            break
    return float(np.mean(times)), len(times)


def run_reference(args, cfg):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    pts = cfg.nx * cfg.ny * cfg.nzp
    warm = min(args.warmup, 1)
    t_step, n = cpu_reference_step_time(cfg, args.steps, 150.0, warm, threads)
    val = pts / t_step
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": n, "warmup": warm, "ms_per_step": t_step * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{WORKLOAD}: 256x64x129 (ref nx,ny,nzp) dyn-Smagorinsky LES, 3/2 dealias"},
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n} full time steps of the same workload (FP64 NumPy/SciPy oracle, "
                                   f"scipy.fft with {threads} workers, BLAS contractions)"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (Fortran+MPI+FFTW+LAPACK) cannot be built here; its restatement is timed",
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default=WORKLOAD)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    cfg = workload(args.workload)
    if args.impl == "reference":
        run_reference(args, cfg)
        return

    import torch
    import torch.distributed as dist
    from lsbflow_b200 import lib

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 1000 + rank, 5e-3)
    sol = lib.Solver(st)
    stream = torch.cuda.Stream()
    sol.set_stream(stream.cuda_stream)
    sol.upload(u, v, w, dt=st.dt)
    pts = cfg.nx * cfg.ny * cfg.nzp

    # ---- warm-up
    with torch.cuda.stream(stream):
        sol.step(args.warmup)
    torch.cuda.synchronize()

    # ---- device-resident timed region
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        sol.step(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms)
    value = pts * args.steps * world / (ms / 1e3)
    clocks = clk.summary()

    # ---- per kernel-group timing (same workload, separate region with event timers on)
    sol.timers(True)
    with torch.cuda.stream(stream):
        sol.step(args.steps)
    torch.cuda.synchronize()
    rep = sol.timer_report()
    sol.timers(False)
    tot = sum(v[1] for v in rep.values())
    groups = {k: {"launches": v[0], "ms_total": round(v[1], 4), "share": round(v[1] / tot, 4)} for k, v in rep.items()}
    top = max(rep.items(), key=lambda kv: kv[1][1])

    # ---- roofline of the dominant kernel group (HBM-bound FFT / stencil work)
    hbm, hbm_kind = peaks()
    nx, ny, nzp = cfg.nx, cfg.ny, cfg.nzp
    nxl, nyl = st.nx_lg, st.ny_lg
    S8 = nx * ny * nzp * 8
    Yl8 = nx * nyl * nzp * 8
    P8 = nx * ny * nzp * 8
    alg_bytes = {
        # row_nl: 9 y-intermediate rows in, 9 out per launch
        "row_nl": 18 * Yl8,
        # spanwise passes: 9 spectral -> 9 padded intermediates; 9 padded -> 9 spectral
        "yinv_nl": 9 * (S8 // 1) // 1 * 0 + 6 * S8 + 9 * Yl8,
        "yfwd_nl": 9 * Yl8 + 9 * S8,
        # the 3-point filter: one field in, one out per component (counted per launch of 6 fields avg)
        "sgs_filter3": None,
        "gemm_dz": 6 * S8,
        "helmholtz_uvw": 3 * (2 * S8 + 2 * S8),
        "sgs_total": None,
    }
    per_launch_ms = top[1][1] / max(top[1][0], 1)
    ab = alg_bytes.get(top[0])
    if ab is None:
        ab = 2 * P8 * 4  # a conservative 4-field in/out estimate for SGS groups
    achieved = ab / (per_launch_ms / 1e3) / 1e9
    roofline = {"kernel": top[0], "bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
                "frac": round(achieved / hbm, 4), "peak_kind": hbm_kind, "traffic": None,
                "alg_bytes_per_launch": ab, "avg_launch_ms": round(per_launch_ms, 4)}

    # ---- end-to-end through the C ABI with host buffers (pinned): per step the velocity
    # (u, v, w) goes host->device, one time step runs, the new velocity comes back.
    hb = [torch.empty(pts * 3 // 3 * 1, dtype=torch.float64, pin_memory=True) for _ in range(3)]
    for i, f in enumerate((u, v, w)):
        hb[i].copy_(torch.from_numpy(np.ascontiguousarray(f).ravel()))
    e2e_steps = max(3, args.steps // 2)
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sol.upload_velocity_ptr(hb[0].data_ptr(), hb[1].data_ptr(), hb[2].data_ptr())
        sol.step(1)
        sol.download_velocity_ptr(hb[0].data_ptr(), hb[1].data_ptr(), hb[2].data_ptr())
    sol.synchronize()
    e2e_s = time.perf_counter() - t0
    e2e_s = max_over_ranks(e2e_s)
    e2e_val = pts * e2e_steps * world / e2e_s

    # ---- the CPU baseline (rank 0, N = 1 only), bounded sample
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        t_step, n = cpu_reference_step_time(cfg, 2, 40.0, 0, threads)
        cpu = {"value": pts / t_step, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{n} time step(s) of the same workload with the FP64 NumPy oracle"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"{args.workload}: {nx}x{ny}x{nzp} (ref nx,ny,nzp), padded {nxl}x{nyl}, "
                                   f"dyn-Smagorinsky LES, dealias 3/2, fringe, dipole BC, dt={st.dt}",
                       "global_batch": world, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (resident state 24 fields x 17 MB)"},
            "roofline": roofline,
            "kernel_groups": groups,
            "clocks": clocks,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 3 * S8, "d2h_bytes_per_step": 3 * S8},
            "gpu_launches": None,
            "cpu_baseline": cpu,
        }
        line["gpu_launches"] = sum(v[0] for v in rep.values())
        print(json.dumps(line), flush=True)
    sol.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
