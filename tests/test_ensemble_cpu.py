"""Ensemble member draws: one grid, Re_delta* ~ U[300, 800], dipole amplitude ~ U[0.1, 0.4],
dipole centre ~ U[60, 100] displacement thicknesses, reproducible from the seed."""
import numpy as np

from lsbflow_b200.config import ensemble_configs, workload


def test_ensemble_draws():
    cfgs = ensemble_configs(64, seed=3000)
    again = ensemble_configs(64, seed=3000)
    assert cfgs == again
    assert len({(c.nx, c.ny, c.nz, c.sgsmodel) for c in cfgs}) == 1
    c0 = workload("ens128")
    assert (cfgs[0].nx, cfgs[0].ny, cfgs[0].nz, cfgs[0].sgsmodel) == (c0.nx, c0.ny, c0.nz, 2)
    re_d = np.array([c.xlen / 200.0 / c.xnu * c.u0 for c in cfgs])   # xlen = 200 delta*
    dstar = re_d * cfgs[0].xnu / cfgs[0].u0
    amp = np.array([c.bc3_amp for c in cfgs])
    xc = np.array([c.bc3_xc for c in cfgs]) / dstar
    assert re_d.min() >= 300 and re_d.max() <= 800 and re_d.std() > 50
    assert amp.min() >= 0.1 and amp.max() <= 0.4
    assert xc.min() >= 60 - 1e-9 and xc.max() <= 100 + 1e-9
    # Re_delta* sets x0 through the Blasius displacement thickness 1.72 sqrt(nu x0 / U)
    for c, r in zip(cfgs[:4], re_d[:4]):
        assert abs(1.72 * np.sqrt(c.xnu * c.x0 / c.u0) * c.u0 / c.xnu - r) < 1e-9 * r


def test_default_workload_unchanged():
    c = workload("ens128")
    assert abs(c.bc3_amp - 0.3) < 1e-15 and abs(c.bc3_xc - 80.0 * 0.5) < 1e-12
