"""The C++/OpenMP restatement of the time step (oracle/cpu_step.cpp, the timed CPU baseline)
against the NumPy oracle: four whole steps from the same seeded field, with the dense z
operator, on the configurations of the benchmark's workloads."""
import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import ic
from lsbflow_b200.config import workload
from oracle import cpu_baseline as CB
from oracle import lsb_oracle as O

TOL = 1e-12


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


CASES = [
    ("les-dynamic-dealias-dipole", dict(nx=32, ny=8, nz=16)),
    ("dns-dealias-dipole", dict(nx=32, ny=8, nz=16, sgsflag=0)),
    ("les-no-dealias", dict(nx=32, ny=8, nz=16, dealiasflag=0)),
    ("les-bctype0", dict(nx=32, ny=8, nz=16, bc_amp=0.0)),
    ("les-ref-ceiling", dict(nx=24, ny=6, nz=12, bc3_top=0)),
]


@pytest.mark.parametrize("name,over", CASES, ids=[c[0] for c in CASES])
def test_cpu_step_matches_oracle(name, over):
    cfg = workload("les256", **over)
    st = hs.make_setup(cfg)
    u, v, w = ic.seeded_noise(st, 3, 2e-2)
    n = 4
    sec, got = CB.run(st, u, v, w, n, 2)
    assert sec > 0.0
    old = O.ZDER
    O.ZDER = "dense"
    try:
        ost = O.State.zeros_like(st, u, v, w, st.dt)
        for _ in range(n):
            O.timestep(st, ost)
    finally:
        O.ZDER = old
    for key, ref in (("uf", ost.uf), ("vf", ost.vf), ("wf", ost.wf)):
        assert rel(got[key], ref) < TOL, (key, rel(got[key], ref))
    # the pressure is a near-cancellation (-(Dw + div) / (k^2 dt bdfv)): 1e-9
    assert rel(got["pf"], ost.pf) < 1e-9, rel(got["pf"], ost.pf)


def test_reference_arm_prints_its_line(capsys):
    import json
    import types

    import bench
    args = types.SimpleNamespace(steps=2, warmup=1, gpus=1, workload="dns64")
    bench.run_reference(args, workload("dns64"))
    line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["steps"] >= 1
    assert line["cpu_baseline"]["kind"] == "port" and "cpu_step" in line["cpu_baseline"]["sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0
