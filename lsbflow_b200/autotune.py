"""Launch-schedule tuner for the time step, with its results kept in a JSON file.

The library picks its launch shapes from models: the FP64 z contractions take the CTA
width (4..8 warps of 8 columns) that leaves the least idle in the last wave, and the 3-point
SGS test filter splits each block column into the number of z chunks that minimises
(waves of resident blocks) x (planes per block).  The models ignore what they cannot see
(L2 hits, the overlap of neighbouring kernels, clocks), so the tuner times the step itself:
for each knob in turn it tries every candidate value with the others held, keeps the
fastest (a candidate must beat the incumbent by ``min_gain`` to replace it, so ties keep
the model), and stores the winner per (device, grid, precision, model) key.  A schedule
only moves work between blocks, never the order of a sum, so every schedule gives the
same results bit for bit; the tuner changes speed only.

    sched = autotune.lookup(cfg, path, device)            # None if never tuned
    sched = autotune.tune_and_store(st, path)["schedule"]  # times candidates on the GPU
    solver.set_schedule(sched)

    python -m lsbflow_b200.autotune --workload les256 --out schedules.json   # on a GPU
"""
from __future__ import annotations

import json
import math
import os
from typing import Callable

from .config import LsbConfig

KNOBS = ("gemm_warps", "filter_zchunks", "y_staging", "filter_staging")


def uses_filter3(cfg: LsbConfig) -> bool:
    """Whether the step runs the 3-point test filter (the dynamic model, or the
    filterall3pt hook at the start of timestep)."""
    return (cfg.sgsflag == 1 and cfg.sgsmodel == 1) or (cfg.ifilt >= 1 and cfg.sgsmodel != 4)


def candidates(cfg: LsbConfig) -> dict:
    """Values tried per knob; 0 is the built-in model.  The ranges are the ones
    lsb_set_schedule accepts (gemm_warps 4..8, filter_zchunks 1..(nzp+3)/4, y_staging 1 cp.async
    or 2 TMA for the FP64 spanwise passes -- the built-in choice is TMA on the padded grid and
    cp.async on the unpadded one --, filter_staging 1 cp.async or 2 TMA row loads for the SGS
    filter's plane ring, where a row is a multiple of 128 bytes)."""
    zmax = max(1, (cfg.nzp + 3) // 4)
    zs = [0] + [c for c in (1, 2, 3, 4, 6, 8, 12, 16) if c <= zmax]
    prec = getattr(cfg, "precision", 0)
    row_bytes = cfg.nx * (4 if prec == 1 else 8)
    return {"gemm_warps": [0, 4, 5, 6, 7, 8],
            "filter_zchunks": zs if uses_filter3(cfg) else [0],
            "y_staging": [0, 1, 2] if prec == 0 else [0],
            "filter_staging": [0, 1, 2] if uses_filter3(cfg) and row_bytes % 128 == 0 else [0]}


def schedule_key(cfg: LsbConfig, device: str) -> str:
    return (f"{device}|{cfg.nx}x{cfg.ny}x{cfg.nzp}|prec{getattr(cfg, 'precision', 0)}|"
            f"sgs{cfg.sgsflag}.{cfg.sgsmodel}|dealias{cfg.dealiasflag}|filt{cfg.ifilt}")


def tune(cfg: LsbConfig, measure: Callable[[dict], float], cands: dict | None = None,
         min_gain: float = 0.01) -> dict:
    """Coordinate search over the knobs.  ``measure(schedule)`` returns ms per step.
    Returns the best schedule, its time, the models' time and every trial."""
    cands = cands or candidates(cfg)
    best = {k: 0 for k in KNOBS}
    trials = []
    base_ms = measure(dict(best))
    trials.append((dict(best), base_ms))
    best_ms = base_ms
    for k in KNOBS:
        for v in cands.get(k, [0]):
            if v == best[k]:
                continue
            s = dict(best)
            s[k] = v
            ms = measure(s)
            trials.append((s, ms))
            if ms < best_ms * (1.0 - min_gain):
                best, best_ms = s, ms
    return {"schedule": best, "ms_per_step": best_ms, "model_ms_per_step": base_ms,
            "trials": [{"schedule": s, "ms_per_step": ms} for s, ms in trials]}


def load_cache(path: str) -> dict:
    if not os.path.exists(path):
        return {}
    with open(path) as f:
        return json.load(f)


def save_cache(path: str, cache: dict) -> None:
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(cache, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def lookup(cfg: LsbConfig, path: str, device: str) -> dict | None:
    ent = load_cache(path).get(schedule_key(cfg, device))
    return None if ent is None else dict(ent["schedule"])


def gpu_measurer(st, steps: int = 20, reps: int = 2, seed: int = 0, amp: float = 1e-3):
    """A measure() that times lsb_step on the current CUDA device (steady steps replayed
    from step graphs, CUDA events on the handle's stream; the best of ``reps`` runs of
    ``steps`` steps).  Returns (measure, close)."""
    import torch

    from . import ic, lib

    s = lib.Solver(st)
    stream = torch.cuda.Stream()
    s.set_stream(stream.cuda_stream)
    u, v, w = ic.seeded_noise(st, seed, amp)
    s.upload(u, v, w, dt=st.dt)
    s.step(3)  # start-up steps

    def measure(sched: dict) -> float:
        s.set_schedule(sched)
        s.step(6)  # this schedule's step graphs are captured
        best = math.inf
        for _ in range(reps):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.step(steps)
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1) / steps)
        return best

    return measure, s.close


def tune_and_store(st, path: str, device: str | None = None, steps: int = 20, reps: int = 2) -> dict:
    """Tune the schedule of ``st``'s workload on the current GPU and store it in ``path``."""
    import torch

    device = device or torch.cuda.get_device_name()
    measure, close = gpu_measurer(st, steps=steps, reps=reps)
    try:
        res = tune(st.cfg, measure)
    finally:
        close()
    cache = load_cache(path)
    cache[schedule_key(st.cfg, device)] = {"schedule": res["schedule"], "ms_per_step": res["ms_per_step"],
                                          "model_ms_per_step": res["model_ms_per_step"]}
    save_cache(path, cache)
    res["device"] = device
    return res


def main(argv=None) -> int:
    """python -m lsbflow_b200.autotune --workload les256 [--precision 1] --out schedules.json"""
    import argparse

    from . import hostsetup as hs
    from .config import workload

    ap = argparse.ArgumentParser(description="Tune the launch schedule of a workload on this GPU and store it.")
    ap.add_argument("--workload", default="les256", help="dns64, os128, les256 or ens128")
    ap.add_argument("--precision", type=int, default=0, choices=[0, 1])
    ap.add_argument("--steps", type=int, default=20, help="timed steps per candidate and repetition")
    ap.add_argument("--out", required=True, help="JSON file the schedule is added to")
    args = ap.parse_args(argv)
    st = hs.make_setup(workload(args.workload, precision=args.precision))
    res = tune_and_store(st, args.out, steps=args.steps)
    print(json.dumps({k: res[k] for k in ("device", "schedule", "ms_per_step", "model_ms_per_step")}))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
