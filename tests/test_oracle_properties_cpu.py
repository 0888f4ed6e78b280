"""Properties of the oracle that hold whatever the implementation: they check the
restatement where no golden data exists.

* sigma model (src/sgsterm.f90:283-423): its differential operator
  D_sigma = s3 (s1 - s2)(s2 - s3) / s1^2 of the singular values of the velocity gradient
  vanishes for every two-dimensional gradient (s3 = 0: pure shear, solid-body rotation)
  and for isotropic expansion (s1 = s2 = s3), and is positive otherwise; tau is
  -2 nu_t S_ij, symmetric.
* 3-point filter (src/filters.f90:363-613): the (a, b, a) / (2a + b) weights in x and y
  and the interpolating non-uniform weights in z keep a constant field constant.
* horfft (src/horfft.f90:61-150): forward after inverse is the identity on normed spectra.
* solve_helmholtz (src/helmholtz.f90:130-208): the eigenbasis solution satisfies the
  Chebyshev Helmholtz equation at the interior points with q = 0 on both walls.
* dealiasing_2d_fftw (src/dealiasing.f90:262-447), textbook 3/2 layout: products of two
  x modes carry no alias of an unresolved sum wavenumber.
* timestep (src/navierstokes.f90:10-90): the velocity stays divergence-free to round-off.
"""
import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200.config import workload
from oracle import lsb_oracle as O


@pytest.fixture(scope="module")
def st():
    return hs.make_setup(workload("dns64", nx=16, ny=8, nz=16))


def gradient(st, g):
    """duidxj[l][m] = g[l][m] everywhere on the physical grid (nzp, ny, nx + 2)."""
    c = st.cfg
    shape = (c.nzp, c.ny, c.nx + 2)
    return [[np.full(shape, float(g[l][m])) for m in range(3)] for l in range(3)]


def smag_scale(st, g):
    return float(np.max((1.35 * st.grid.dx) ** 2) * np.sum(np.asarray(g, float) ** 2) + 1e-300)


@pytest.mark.parametrize("g", [
    [[0, 0, 2.0], [0, 0, 0], [0, 0, 0]],          # pure shear du/dz
    [[0, -1.5, 0], [1.5, 0, 0], [0, 0, 0]],       # solid-body rotation about z
    [[0.3, 1.0, 0], [-0.4, -0.3, 0], [0, 0, 0]],  # any two-dimensional gradient
    [[0.7, 0, 0], [0, 0.7, 0], [0, 0, 0.7]],      # isotropic expansion
])
def test_sigma_model_vanishes_where_it_should(st, g):
    tau = O.sigma_model(st, gradient(st, g))
    nx = st.cfg.nx
    big = max(float(np.abs(tau[l][m][..., :nx]).max()) for l in range(3) for m in range(3))
    assert big <= 1e-6 * smag_scale(st, g)


def test_sigma_model_generic_gradient(st):
    g = np.array([[0.2, 1.1, -0.3], [0.4, -0.5, 0.8], [-0.6, 0.1, 0.3]])
    tau = O.sigma_model(st, gradient(st, g))
    nx = st.cfg.nx
    S = 0.5 * (g + g.T)
    t = np.array([[tau[l][m][3, 2, 5] for m in range(3)] for l in range(3)])
    assert np.allclose(t, t.T, rtol=0, atol=1e-15 * np.abs(t).max())
    # tau = -2 nu_t S with nu_t > 0: the same ratio in every component, negative
    ratio = t[np.abs(S) > 1e-12] / S[np.abs(S) > 1e-12]
    assert np.all(ratio < 0) and np.ptp(ratio) <= 1e-12 * np.abs(ratio).max()
    assert all(np.all(tau[l][m][..., nx:] == 0) for l in range(3) for m in range(3))


@pytest.mark.parametrize("a,b", [(1.0, 1.0), (1.0, 6.0), (1.0, 2.0)])
def test_three_point_filter_keeps_constants(st, a, b):
    c = st.cfg
    q = np.full((c.nzp, c.ny, c.nx + 2), 1.7)
    out = O.filter_q_3pt(st, q, a, b)
    assert np.allclose(out[..., : c.nx], 1.7, rtol=0, atol=1e-14)
    assert np.all(out[..., c.nx:] == 0)


def random_spectral(st, seed):
    c = st.cfg
    f = np.random.default_rng(seed).standard_normal((c.nzp, c.ny, c.nx))
    O.norm([f], c.ny)  # the reference's symmetrisation: a field horfft maps back to itself
    return f


def test_horfft_round_trip(st):
    """horfft(+1) then horfft(-1) (src/horfft.f90:61-150) returns a normed spectrum."""
    c = st.cfg
    f = random_spectral(st, 3)
    back = O.horfft_fwd(O.horfft_inv(f, c.nx, c.ny), c.nx, c.ny)
    assert np.allclose(back, f, rtol=0, atol=1e-13 * np.abs(f).max())


def test_helmholtz_solve_satisfies_its_equation(st):
    """solve_helmholtz (src/helmholtz.f90:130-208): q = 0 on both walls and
    (D2 - k^2 - sigma) q = rhs at the interior points, column by column."""
    c = st.cfg
    nz = c.nz
    rhs = random_spectral(st, 4)
    sigma = 37.5
    q = O.solve_helmholtz(st, rhs.copy(), sigma)
    assert np.all(q[0] == 0) and np.all(q[nz] == 0)
    lhs = np.einsum("km,mji->kji", st.d2, q) - (O.wav2(st)[None] + sigma) * q
    err = np.abs(lhs[1:nz] - rhs[1:nz]).max()
    assert err <= 1e-9 * np.abs(rhs).max()


@pytest.mark.parametrize("k1,k2", [(5, 4), (7, 6), (3, 2)])
def test_padded_product_has_no_aliases_in_x(k1, k2):
    """The 3/2-rule product (src/dealiasing.f90:262-447, textbook layout) of cos(k1 x) and
    cos(k2 x) is 1/2 cos((k1 - k2) x) plus 1/2 cos((k1 + k2) x) when k1 + k2 is resolved,
    and has nothing at the alias nx - (k1 + k2) when it is not."""
    st = hs.make_setup(workload("dns64", nx=16, ny=8, nz=8, dealiasflag=1))
    c = st.cfg
    x = 2.0 * np.pi * np.arange(c.nx) / c.nx
    a = np.zeros((c.nzp, c.ny, c.nx + 2))
    b = np.zeros_like(a)
    a[..., : c.nx] = np.cos(k1 * x)
    b[..., : c.nx] = np.cos(k2 * x)
    f = O.to_complex(O.horfft_fwd(O.dealias_product(st, a, b, "correct"), c.nx, c.ny))[2, 0, :]
    expect = np.zeros(c.nx // 2)
    expect[k1 - k2] += 0.25
    if k1 + k2 < c.nx // 2:
        expect[k1 + k2] += 0.25
    assert np.allclose(f, expect, rtol=0, atol=1e-14)


@pytest.mark.parametrize("name,over", [("dns64", dict(nx=32, ny=8, nz=32, dealiasflag=1)),
                                       ("les256", dict(nx=32, ny=8, nz=32))])
def test_time_step_keeps_velocity_divergence_free(name, over):
    """navierstokes_update (src/navierstokes.f90:1157-1496): the pressure correction and
    the Poisson solve for w leave div u at round-off, walls included."""
    from lsbflow_b200 import ic
    st = hs.make_setup(workload(name, **over))
    u, v, w = ic.seeded_noise(st, 3, 1e-2)
    s = O.State.zeros_like(st, u, v, w, st.dt)
    for _ in range(4):
        O.timestep(st, s)
        div = O.divuv(st, s.uf, s.vf) + O.dfdz(st, s.wf)
        assert np.abs(div).max() <= 1e-12 * np.abs(O.dfdx(st, s.uf)).max()
