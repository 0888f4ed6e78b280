"""The native driver lsb_run (host C++ over the C ABI): it reads the set-up file the Python
set-up writes, reads and writes the reference's restart layout byte for byte, writes q
files in the reference's layout, and fails loudly when no device is present."""
import os
import subprocess

import numpy as np
import pytest

from lsbflow_b200 import build
from lsbflow_b200 import formats as F
from lsbflow_b200 import hostsetup as hs
from lsbflow_b200 import lib
from lsbflow_b200.config import workload


@pytest.fixture(scope="module")
def driver():
    if not os.path.exists(lib.LIBPATH):
        pytest.skip("library not built")
    return build.build_driver()


def run(driver, *args):
    return subprocess.run([driver, *map(str, args)], capture_output=True, text=True, timeout=120)


def random_restart(cfg, seed, isum=40):
    rng = np.random.default_rng(seed)
    r = F.Restart(isum, 0.2, 0.005, 0.005, 0.005, cfg.nx, cfg.ny, cfg.nzp, cfg.nx)
    for name in F.RESTART_VARS:
        r.fields[name] = rng.standard_normal((cfg.nzp, cfg.ny, cfg.nx))
    return r


def test_setup_file_read_back(driver, tmp_path):
    st = hs.make_setup(workload("les256", nx=32, ny=8, nz=16, precision=1))
    path = tmp_path / "setup.bin"
    lib.write_setup_file(str(path), st)
    out = run(driver, "--check-setup", path)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.splitlines()
    head = lines[0].split()
    assert head[:12] == ["nx", "32", "ny", "8", "nz", "16", "precision", "1", "sgsflag", "1", "sgsmodel", "1"]
    assert float(head[13]) == st.grid.dx and float(head[15]) == st.grid.dy
    for line, (name, a) in zip(lines[1:], lib.setup_arrays(st)):
        n, count, total = line.split()
        a = np.asarray(a, dtype=np.float64).ravel()
        assert n == name and int(count) == a.size
        assert abs(float(total) - a.sum()) <= 1e-12 * max(1.0, np.abs(a).sum())


def test_setup_file_rejects_garbage(driver, tmp_path):
    bad = tmp_path / "bad.bin"
    bad.write_bytes(b"NOTSETUP" + bytes(64))
    out = run(driver, "--check-setup", bad)
    assert out.returncode == 1 and "not a set-up file" in out.stderr


def test_restart_and_q_layouts(driver, tmp_path):
    cfg = workload("dns64", nx=16, ny=6, nz=8)
    r = random_restart(cfg, 3)
    start = tmp_path / "start.dat"
    F.write_restart(str(start), r, ref_bug=False)
    out = run(driver, "--io-selftest", start, tmp_path)
    assert out.returncode == 0, out.stderr
    # the C++ reader and writer reproduce the file byte for byte
    assert (tmp_path / "roundtrip.dat").read_bytes() == start.read_bytes()
    # the q file holds u, v, w and (in p's place) T in the reference's (y, z, x) order
    q = F.read_snapshot(str(tmp_path / "q00040.dat"))
    assert (q.isum, q.nx, q.ny, q.nzp, q.nypl) == (40, cfg.nx, cfg.ny, cfg.nzp, cfg.ny)
    for got, name in ((q.u, "u"), (q.v, "v"), (q.w, "w"), (q.p, "T")):
        assert np.array_equal(got, r.fields[name].astype(np.float32).astype(np.float64)), name
    assert not q.T.any()


def test_run_fails_loudly_without_device(driver, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    cfg = workload("dns64", nx=16, ny=6, nz=8)
    st = hs.make_setup(cfg)
    lib.write_setup_file(str(tmp_path / "setup.bin"), st)
    F.write_restart(str(tmp_path / "start.dat"), random_restart(cfg, 4))
    out = run(driver, tmp_path / "setup.bin", tmp_path / "start.dat", 4, 2, tmp_path)
    assert out.returncode == 1 and "lsb_create failed" in out.stderr
    out = run(driver, tmp_path / "setup.bin", tmp_path / "start.dat", 4)
    assert out.returncode == 2 and "usage" in out.stderr


def test_restart_dimension_mismatch_stops_the_run(driver, tmp_path):
    """As src/mpi_io.f90:233-242, a restart of another grid stops the run before any device work."""
    st = hs.make_setup(workload("dns64", nx=16, ny=6, nz=8))
    lib.write_setup_file(str(tmp_path / "setup.bin"), st)
    F.write_restart(str(tmp_path / "start.dat"), random_restart(workload("dns64", nx=16, ny=8, nz=8), 5))
    out = run(driver, tmp_path / "setup.bin", tmp_path / "start.dat", 4, 2, tmp_path)
    assert out.returncode == 1 and "differ from the run's" in out.stderr
