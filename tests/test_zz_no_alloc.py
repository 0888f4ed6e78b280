"""The allocation-free Helmholtz entry point (lsb_solve_helmholtz_noalloc).

It serves callers that may not allocate GPU memory themselves (device memory owned
by a pool or framework, or loops that cannot afford cudaMalloc's synchronisation):
they pass device pointers they already own and the library works in a static device
array.  Checked here through the C ABI against the handle-based lsb_solve_helmholtz on
two calls in a row, at a size where the columns are solved in several chunks.  This
file is collected last so that a run stopping at the first failure has run the rest.
"""
import numpy as np
import pytest

from lsbflow_b200 import hostsetup as hs
from lsbflow_b200.config import workload
from oracle import lsb_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the operator tolerance of the parity tests


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


# nx*ny = 16384 columns at nzp = 129 (three chunks of whole 64-column tiles); 17500 columns
# (two full chunks and a tail of 1628, a partly filled last tile); 288 columns at nzp = 33
# (one chunk, a partly filled last tile)
GRIDS = [dict(), dict(nx=250, ny=70), dict(nx=48, ny=6, nz=32)]


@pytest.mark.parametrize("grid", GRIDS, ids=["256x64x129", "250x70x129", "48x6x33"])
def test_noalloc_matches_handle_entry_point_twice(grid):
    import torch
    from lsbflow_b200 import lib
    cfg = workload("les256", dealiasflag=0, sgsflag=0, **grid)
    st = hs.make_setup(cfg)
    s = lib.Solver(st)
    dev = torch.device("cuda")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(dev)
    lam, E, Ei, wx, wy = t(st.lam), t(st.E), t(st.Ei), t(st.grid.wavx), t(st.grid.wavy)
    rng = np.random.default_rng(42)
    for call, dtnui in enumerate((1.0 / (cfg.xnu * st.dt) / (6.0 / 11.0), 0.0)):
        rhs = rng.standard_normal((cfg.nzp, cfg.ny, cfg.nx))
        O.norm([rhs], cfg.ny)
        ref = s.solve_helmholtz(rhs, dtnui)
        rd = t(rhs)
        out = torch.full_like(rd, float("nan"))
        torch.cuda.synchronize()
        lib.solve_helmholtz_noalloc(cfg.nx, cfg.ny, cfg.nz, rd.data_ptr(), out.data_ptr(), lam.data_ptr(),
                                    E.data_ptr(), Ei.data_ptr(), wx.data_ptr(), wy.data_ptr(), dtnui,
                                    torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), call
        assert rel(got, ref) < TOL, (call, rel(got, ref))
    s.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    from lsbflow_b200 import lib
    with pytest.raises(lib.LsbError, match="no-allocation limit"):
        lib.solve_helmholtz_noalloc(16, 8, 200, 8, 16, 24, 32, 40, 48, 56, 0.0)
