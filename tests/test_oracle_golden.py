"""Pins of the host set-up and the FP64 oracle against the reference's own shipped
run (run/grid.dat, run/paral.dat, run/output.txt, run/prev_q0000{1,2}.dat)."""
import os

import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200.config import parse_namelist
from oracle import lsb_oracle as O

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_run.npz"))


@pytest.fixture(scope="module")
def setup():
    cfg = parse_namelist(str(GOLD["input_dat"]))
    return hs.make_setup(cfg)


def test_namelist_matches_grid_header(setup):
    assert tuple(GOLD["grid_dims"]) == (setup.cfg.nx, setup.cfg.ny, setup.cfg.nzp)
    np.testing.assert_array_equal(GOLD["grid_params"], [setup.grid.x0, setup.grid.xl, setup.grid.xlen,
                                                         setup.grid.ylen, setup.grid.zlen])


@pytest.mark.parametrize("name", ["xpts", "ypts", "zpts", "gf"])
def test_grid_bit_exact(setup, name):
    # G1: setup_grid, mapping 2 (src/init.f90:215-229)
    np.testing.assert_array_equal(getattr(setup.grid, name), GOLD[name])


@pytest.mark.parametrize("name,tol", [("ubar", 1e-13), ("ubarp", 1e-12), ("ubarpp", 1e-11),
                                      ("wbar", 1e-13), ("wbarp", 1e-13), ("wbarpp", 1e-12)])
def test_paral(setup, name, tol):
    # G2: blasfl + dpdz through dct_diff at nzp = 33
    ref = GOLD[name]
    got = getattr(setup, name)
    assert np.max(np.abs(got - ref)) <= tol * max(1.0, np.max(np.abs(ref)))


def test_blasfl_iterations_and_dt(setup):
    assert setup.blasfl_iters == int(GOLD["blasfl_iters"])
    assert abs(setup.dt - float(GOLD["dt0"])) <= 4e-15 * float(GOLD["dt0"])


def test_d2_eigenvalues(setup):
    # G3: 31 eigenvalues printed with 7 significant digits
    ref = np.sort(GOLD["eig_d2"])
    got = np.sort(setup.lam)
    np.testing.assert_allclose(got, ref, rtol=6e-7)


def test_blasius_table(setup):
    # G4: the printed (zpts, ubar, ubarp, ubarpp, wbar) columns, 4 significant digits
    tab = GOLD["blasius_table"]
    cols = [setup.grid.zpts, setup.ubar, setup.ubarp, setup.ubarpp, setup.wbar]
    for c, col in enumerate(cols):
        ref = tab[:, c]
        err = np.abs(col - ref)
        assert np.all(err <= 6e-4 * np.abs(ref) + 1e-12 + 5e-4 * (np.abs(ref) < 1e-3))


def test_dct_matches_dense_d(setup):
    # G7: the DCT-I derivative and the closed-form D agree to round-off
    m1 = hs.dct_diff_matrix(setup.grid, 1)
    assert np.max(np.abs(m1 - setup.d)) <= 1e-11 * np.max(np.abs(setup.d))
    m2 = hs.dct_diff_matrix(setup.grid, 2)
    assert np.max(np.abs(m2 - setup.d2)) <= 1e-10 * np.max(np.abs(setup.d2))


@pytest.mark.slow
def test_zero_perturbation_run_matches_snapshots(setup):
    # G5: 20 steps of the shipped input.dat run (dealiasflag 2, adaptive dt),
    # compared with the float32 snapshots the reference wrote at steps 10 and 20.
    c = setup.cfg
    z = np.zeros((c.nzp, c.ny, c.nx))
    s = O.State.zeros_like(setup, z, z, z, setup.dt)
    for _ in range(20):
        O.timestep(setup, s)
        if s.istep in (10, 20):
            hdr = GOLD[f"q{s.istep}_header"]
            assert int(hdr[0]) == s.istep
            assert abs(np.float32(s.t) - hdr[1]) <= 1e-6 * hdr[1]
            assert np.float32(s.dt) == hdr[2]
            u = O.horfft_inv(s.uf, c.nx, c.ny)[..., : c.nx] + setup.ubar[:, None, None]
            np.testing.assert_allclose(u[:, 0, 0], GOLD[f"q{s.istep}_uprof"], rtol=0, atol=1.2e-7)
            assert np.abs(u - u[:, :1, :1]).max() <= 1e-12
            for f, key in ((s.vf, "vmax"), (s.wf, "wmax"), (s.pf, "pmax")):
                p = O.horfft_inv(f, c.nx, c.ny)
                assert np.abs(p).max() <= 1e-14 and float(GOLD[f"q{s.istep}_{key}"]) <= 1e-14


def test_dealias_ref_layout_bug():
    # the reference's y padding (src/dealiasing.f90:329-330,435) misplaces negative ky.
    # For cos(y)^2 on ny=8 (ny_lg=12) the padded spanwise signal becomes complex,
    # c2r keeps its real part 0.5(cos t + cos 7t); its square truncated to rows 0..7 is
    # {0: 1/4, 2: 1/8, 4: 1/8, 6: 1/4}, and the horfft round trip symmetrises ky/-ky:
    # {0: 1/4, 2: 3/16, 4: 1/8, 6: 3/16}.  The correct 3/2 rule gives 1/2 + cos(2y)/2.
    from lsbflow_b200.config import LsbConfig
    cfg = LsbConfig(nx=8, ny=8, nz=8, xlen=2 * np.pi * 7 / 8 * 8 / 7, ylen=2 * np.pi, zlen=1.0,
                    dealiasflag=1, dealias_layout="ref")
    st = hs.make_setup(cfg)
    y = 2 * np.pi * np.arange(8) / 8
    a = np.zeros((cfg.nzp, 8, 10))
    a[..., :8] = np.cos(y)[None, :, None]
    for layout, expect in (("ref", {0: 0.25, 2: 0.1875, 4: 0.125, 6: 0.1875}), ("correct", {0: 0.5, 2: 0.25, 6: 0.25})):
        p = O.dealias_product(st, a, a, layout)
        f = O.to_complex(O.horfft_fwd(p, 8, 8))[0, :, 0]
        got = {j: round(float(f[j].real), 12) for j in range(8) if abs(f[j]) > 1e-12}
        assert got == expect, (layout, got)
