"""The schedule tuner's search and its JSON store, with a stand-in for the GPU timer."""
import pytest

from lsbflow_b200 import autotune as A
from lsbflow_b200.config import workload


def surface(best_w=6, best_z=3, tma_gain=0.03, floor=1.0):
    """ms per step: separable, minimal at (best_w, best_z) with TMA staging of the spanwise
    passes (y_staging 2) ``tma_gain`` faster; 0 (the models) is a few % off."""
    def ms(s):
        w = s["gemm_warps"] or 8
        z = s["filter_zchunks"] or 1
        y = -tma_gain if s.get("y_staging", 0) == 2 else 0.0
        return floor * (1.0 + 0.01 * abs(w - best_w) + 0.02 * abs(z - best_z) + y + tma_gain)
    return ms


def test_candidates_are_within_the_c_abi_limits():
    for name in ("les256", "ens128", "dns64"):
        cfg = workload(name)
        c = A.candidates(cfg)
        assert set(c) == set(A.KNOBS)
        assert all(v == 0 or 4 <= v <= 8 for v in c["gemm_warps"])
        zmax = max(1, (cfg.nzp + 3) // 4)
        assert all(0 <= v <= zmax for v in c["filter_zchunks"])
        assert 0 in c["gemm_warps"] and 0 in c["filter_zchunks"]
        assert c["y_staging"] == ([0, 1, 2] if cfg.precision == 0 else [0])
        assert c["filter_staging"] == ([0, 1, 2] if A.uses_filter3(cfg) else [0])
    assert A.candidates(workload("ens128"))["filter_zchunks"] == [0]     # sigma: no test filter
    assert A.candidates(workload("les256", nx=8))["filter_staging"] == [0]  # 64-byte rows: no TMA
    assert len(A.candidates(workload("les256"))["filter_zchunks"]) > 4  # dynamic: filtered


def test_search_finds_the_minimum_and_counts_trials():
    cfg = workload("les256")
    calls = []
    m = surface()

    def measure(s):
        calls.append(dict(s))
        return m(s)

    res = A.tune(cfg, measure)
    assert res["schedule"] == {"gemm_warps": 6, "filter_zchunks": 3, "y_staging": 2, "filter_staging": 0}
    assert res["ms_per_step"] == pytest.approx(1.0)
    assert res["model_ms_per_step"] == m({"gemm_warps": 0, "filter_zchunks": 0, "y_staging": 0, "filter_staging": 0})
    c = A.candidates(cfg)
    assert len(calls) == 1 + sum(len(c[k]) - 1 for k in A.KNOBS)
    assert len(res["trials"]) == len(calls)


def test_ties_keep_the_model():
    res = A.tune(workload("les256"), lambda s: 1.0 if s["gemm_warps"] else 1.001)
    assert res["schedule"] == {"gemm_warps": 0, "filter_zchunks": 0, "y_staging": 0, "filter_staging": 0}


def test_store_round_trip_and_keys(tmp_path):
    p = str(tmp_path / "sub" / "schedules.json")
    a, b = workload("les256"), workload("les256", precision=1)
    assert A.schedule_key(a, "B200") != A.schedule_key(b, "B200")
    assert A.schedule_key(a, "B200") != A.schedule_key(a, "H100")
    assert A.lookup(a, p, "B200") is None
    cache = A.load_cache(p)
    cache[A.schedule_key(a, "B200")] = {"schedule": {"gemm_warps": 5, "filter_zchunks": 2},
                                        "ms_per_step": 2.0, "model_ms_per_step": 2.1}
    A.save_cache(p, cache)
    assert A.lookup(a, p, "B200") == {"gemm_warps": 5, "filter_zchunks": 2}
    assert A.lookup(b, p, "B200") is None


def test_command_line_help():
    import subprocess
    import sys
    out = subprocess.run([sys.executable, "-m", "lsbflow_b200.autotune", "--help"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0 and "--workload" in out.stdout and "--out" in out.stdout
