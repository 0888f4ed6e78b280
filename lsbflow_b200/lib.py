"""ctypes binding of the C ABI in include/lsbgpu.h (the reference-facing boundary).

``Solver`` owns one library handle.  Arrays use the reference's Fortran storage order,
i.e. numpy C-order arrays shaped (nzp, ny, nx) for spectral fields and (nzp, ny, nx+2)
for physical ones.  The library is loaded from the package directory; there is no
fallback: if it is missing or no CUDA device is present the calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .config import LsbConfig
from .hostsetup import Setup

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "liblsbgpu.so")

_dp = C.POINTER(C.c_double)

# every symbol the header declares (checked by the CPU tests)
EXPORTS = [
    "lsb_last_error", "lsb_version", "lsb_create", "lsb_destroy", "lsb_set_stream", "lsb_upload_state",
    "lsb_download_state", "lsb_upload_state_device", "lsb_download_velocity_device", "lsb_step", "lsb_diag",
    "lsb_synchronize", "lsb_horfft", "lsb_dealias_product", "lsb_dfdx", "lsb_dfdy", "lsb_dfdz", "lsb_d2fdz2",
    "lsb_lapl", "lsb_divuv", "lsb_solve_helmholtz", "lsb_solve_nhom_helmholtz", "lsb_nlterm", "lsb_tau_sgs",
    "lsb_upload_velocity", "lsb_download_velocity", "lsb_timers", "lsb_timer_report",
    "lsb_solve_helmholtz_noalloc", "lsb_tavg", "lsb_spanwise_stats", "lsb_graphs", "lsb_kernel_launches", "lsb_device_bytes",
    "lsb_batch_create", "lsb_batch_destroy", "lsb_batch_step", "lsb_batch_synchronize", "lsb_batch_graphs",
    "lsb_batch_set_stream", "lsb_set_schedule", "lsb_get_schedule",
    "lsb_snapshot_async",
]


class LsbConfigC(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dealiasflag", C.c_int), ("dealias_layout", C.c_int),
        ("sgsflag", C.c_int), ("sgsmodel", C.c_int), ("forcing", C.c_int), ("bctype", C.c_int),
        ("ifrz", C.c_int), ("nstart", C.c_int), ("mapping", C.c_int),
        ("xnu", C.c_double), ("u0", C.c_double), ("x0", C.c_double), ("xlen", C.c_double),
        ("ylen", C.c_double), ("zlen", C.c_double),
        ("a", C.c_double), ("b", C.c_double), ("cs", C.c_double),
        ("kc", C.c_double), ("filt_order", C.c_double), ("filt_amp", C.c_double),
        ("istartbound", C.c_double), ("samp", C.c_double),
        ("bc3_amp", C.c_double), ("bc3_xc", C.c_double), ("bc3_s", C.c_double),
        ("fsize", C.c_double),
        ("dtadapt", C.c_int), ("iomod", C.c_int), ("ifilt", C.c_int), ("modfilt", C.c_int),
        ("otfavg", C.c_int), ("istartavg", C.c_int), ("precision", C.c_int), ("bc3_top", C.c_int),
    ]


class LsbSetupC(C.Structure):
    _fields_ = [
        ("xpts", _dp), ("ypts", _dp), ("zpts", _dp), ("wavx", _dp), ("wavy", _dp),
        ("dx", C.c_double), ("dy", C.c_double),
        ("dz1", _dp), ("dz2", _dp), ("lam", _dp), ("e", _dp), ("ei", _dp),
        ("ubar", _dp), ("ubarp", _dp), ("ubarpp", _dp),
        ("hbot", _dp), ("htop", _dp), ("d2hbot", _dp), ("d2htop", _dp), ("lamx", _dp),
    ]


class LsbDiagC(C.Structure):
    _fields_ = [
        ("divergence", C.c_double), ("umax", C.c_double), ("umin", C.c_double), ("vmax", C.c_double),
        ("vmin", C.c_double), ("wmax", C.c_double), ("wmin", C.c_double),
        ("cflx", C.c_double), ("cfly", C.c_double), ("cflz", C.c_double),
        ("energy_total", C.c_double), ("energy_pert", C.c_double), ("t", C.c_double), ("dt", C.c_double),
        ("istep", C.c_int), ("nonfinite", C.c_int),
    ]


class LsbScheduleC(C.Structure):
    _fields_ = [("gemm_warps", C.c_int), ("filter_zchunks", C.c_int), ("y_staging", C.c_int),
                ("filter_staging", C.c_int)]


_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"{LIBPATH} is missing: run `python -m lsbflow_b200.build`")
        lib = C.CDLL(LIBPATH)
        lib.lsb_last_error.restype = C.c_char_p
        for name in EXPORTS:
            f = getattr(lib, name)
            if name == "lsb_kernel_launches":
                f.restype = C.c_ulonglong
            elif name != "lsb_last_error":
                f.restype = C.c_int
        _lib = lib
    return _lib


class LsbError(RuntimeError):
    pass


def _ck(rc: int):
    if rc != 0:
        raise LsbError(f"lsbgpu error {rc}: {load().lsb_last_error().decode()}")


def _ptr(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def kernel_launches() -> int:
    """Kernels the library has launched since it was loaded (all handles)."""
    return int(load().lsb_kernel_launches())


def config_struct(cfg: LsbConfig) -> LsbConfigC:
    return LsbConfigC(
        cfg.nx, cfg.ny, cfg.nz, cfg.dealiasflag, 0 if cfg.dealias_layout == "ref" else 1,
        cfg.sgsflag, cfg.sgsmodel, cfg.forcing, cfg.bctype, cfg.ifrz, cfg.nstart, cfg.mapping,
        cfg.xnu, cfg.u0, cfg.x0, cfg.xlen, cfg.ylen, cfg.zlen, cfg.a, cfg.b, cfg.CS,
        cfg.kc, cfg.filt_order, cfg.filt_amp, cfg.istartbound, cfg.samp,
        cfg.bc3_amp, cfg.bc3_xc, cfg.bc3_s, cfg.fsize,
        cfg.dtadapt, cfg.iomod, cfg.ifilt, cfg.modfilt, getattr(cfg, "otfavg", 0), getattr(cfg, "istartavg", 0),
        getattr(cfg, "precision", 0), getattr(cfg, "bc3_top", 1),
    )


def solve_helmholtz_noalloc(nx, ny, nz, rhs_ptr, out_ptr, lam_ptr, e_ptr, ei_ptr, wavx_ptr, wavy_ptr, dtnui,
                            stream_ptr=0):
    """Allocation-free Helmholtz solve on device pointers (raw addresses)."""
    lib = load()
    _ck(lib.lsb_solve_helmholtz_noalloc(C.c_int(nx), C.c_int(ny), C.c_int(nz), C.c_void_p(rhs_ptr),
                                        C.c_void_p(out_ptr), C.c_void_p(lam_ptr), C.c_void_p(e_ptr),
                                        C.c_void_p(ei_ptr), C.c_void_p(wavx_ptr), C.c_void_p(wavy_ptr),
                                        C.c_double(dtnui), C.c_void_p(stream_ptr)))


SETUP_MAGIC = b"LSBSETUP"
SETUP_VERSION = 1


def setup_arrays(st: Setup) -> list:
    """The lsb_setup arrays in the struct's order, as (name, float64 array) pairs."""
    g = st.grid
    return [("xpts", g.xpts), ("ypts", g.ypts), ("zpts", g.zpts), ("wavx", g.wavx), ("wavy", g.wavy),
            ("dz1", st.dz1), ("dz2", st.dz2), ("lam", st.lam), ("e", st.E), ("ei", st.Ei),
            ("ubar", st.ubar), ("ubarp", st.ubarp), ("ubarpp", st.ubarpp), ("hbot", st.hbot),
            ("htop", st.htop), ("d2hbot", st.d2hbot), ("d2htop", st.d2htop), ("lamx", st.lam_x)]


def write_setup_file(path: str, st: Setup) -> None:
    """The inputs of lsb_create in one file for a native driver (lsb_run): the magic
    ``LSBSETUP``, int32 version, int32 sizeof(lsb_config) and the struct's bytes, dx and
    dy, then each set-up array as an int64 count and that many little-endian float64."""
    cs = config_struct(st.cfg)
    with open(path, "wb") as f:
        f.write(SETUP_MAGIC)
        f.write(np.array([SETUP_VERSION, C.sizeof(cs)], dtype="<i4").tobytes())
        f.write(bytes(cs))
        f.write(np.array([st.grid.dx, st.grid.dy], dtype="<f8").tobytes())
        for _, a in setup_arrays(st):
            a = np.ascontiguousarray(np.asarray(a, dtype="<f8")).ravel()
            f.write(np.array([a.size], dtype="<i8").tobytes())
            f.write(a.tobytes())


class Solver:
    """One device-resident LSBFLOW run (a library handle)."""

    def __init__(self, st: Setup):
        lib = load()
        self.st = st
        cfg = st.cfg
        self.cfg = cfg
        g = st.grid
        self.nx, self.ny, self.nzp = cfg.nx, cfg.ny, cfg.nzp
        keep = {}

        def arr(x):
            a = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
            keep[id(a)] = a
            return _ptr(a)

        su = LsbSetupC(
            arr(g.xpts), arr(g.ypts), arr(g.zpts), arr(g.wavx), arr(g.wavy), g.dx, g.dy,
            arr(st.dz1), arr(st.dz2), arr(st.lam), arr(st.E), arr(st.Ei),
            arr(st.ubar), arr(st.ubarp), arr(st.ubarpp),
            arr(st.hbot), arr(st.htop), arr(st.d2hbot), arr(st.d2htop), arr(st.lam_x),
        )
        cs = config_struct(cfg)
        self._h = C.c_void_p()
        _ck(lib.lsb_create(C.byref(cs), C.byref(su), C.byref(self._h)))
        self._lib = lib

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._lib.lsb_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- shapes
    def spec_shape(self):
        return (self.nzp, self.ny, self.nx)

    def phys_shape(self):
        return (self.nzp, self.ny, self.nx + 2)

    # ---- tier 2
    def upload(self, uf, vf, wf, pf=None, pnf=None, unif=None, unmif=None, nlnif=None, nlnmif=None,
               t=0.0, dt=None, dt2=None, dt3=None, istep=0):
        dt = self.st.dt if dt is None else dt
        dt2 = dt if dt2 is None else dt2
        dt3 = dt if dt3 is None else dt3

        def p(a):
            return None if a is None else _ptr(np.ascontiguousarray(a, dtype=np.float64))

        arrs = [np.ascontiguousarray(a, dtype=np.float64) if a is not None else None
                for a in (uf, vf, wf, pf, pnf, unif, unmif, nlnif, nlnmif)]
        ptrs = [_ptr(a) if a is not None else None for a in arrs]
        _ck(self._lib.lsb_upload_state(self._h, *ptrs, C.c_double(t), C.c_double(dt), C.c_double(dt2),
                                       C.c_double(dt3), C.c_int(istep)))

    def download(self):
        sh = self.spec_shape()
        out = {k: np.empty(sh) for k in ("uf", "vf", "wf", "pf", "pnf")}
        for k in ("unif", "unmif", "nlnif", "nlnmif"):
            out[k] = np.empty((3,) + sh)
        t, dt, dt2, dt3 = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        ist = C.c_int()
        _ck(self._lib.lsb_download_state(self._h, *[_ptr(out[k]) for k in ("uf", "vf", "wf", "pf", "pnf",
                                                                            "unif", "unmif", "nlnif", "nlnmif")],
                                         C.byref(t), C.byref(dt), C.byref(dt2), C.byref(dt3), C.byref(ist)))
        out.update(t=t.value, dt=dt.value, dt2=dt2.value, dt3=dt3.value, istep=ist.value)
        return out

    def step(self, n: int = 1):
        _ck(self._lib.lsb_step(self._h, C.c_int(n)))

    def graphs(self, enable: bool):
        """Replay steady steps from CUDA graphs (default) or launch every kernel."""
        _ck(self._lib.lsb_graphs(self._h, C.c_int(1 if enable else 0)))

    def synchronize(self):
        _ck(self._lib.lsb_synchronize(self._h))

    def set_schedule(self, sched: dict | None):
        """Launch schedule ({"gemm_warps": 0|4..8, "filter_zchunks": 0|1.., "y_staging": 0|1|2,
        "filter_staging": 0|1|2}); None or zeros: the built-in choices.  Results do not depend
        on it."""
        sched = sched or {}
        sc = LsbScheduleC(int(sched.get("gemm_warps", 0)), int(sched.get("filter_zchunks", 0)),
                          int(sched.get("y_staging", 0)), int(sched.get("filter_staging", 0)))
        _ck(self._lib.lsb_set_schedule(self._h, C.byref(sc)))

    def schedule(self) -> dict:
        sc = LsbScheduleC()
        _ck(self._lib.lsb_get_schedule(self._h, C.byref(sc)))
        return {f: getattr(sc, f) for f, _ in LsbScheduleC._fields_}

    def device_bytes(self) -> int:
        b = C.c_ulonglong()
        _ck(self._lib.lsb_device_bytes(self._h, C.byref(b)))
        return int(b.value)

    def set_stream(self, stream_handle: int | None):
        _ck(self._lib.lsb_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def upload_device(self, u_ptr: int, v_ptr: int, w_ptr: int):
        _ck(self._lib.lsb_upload_state_device(self._h, C.c_void_p(u_ptr), C.c_void_p(v_ptr), C.c_void_p(w_ptr)))

    def download_device(self, u_ptr: int, v_ptr: int, w_ptr: int):
        _ck(self._lib.lsb_download_velocity_device(self._h, C.c_void_p(u_ptr), C.c_void_p(v_ptr),
                                                   C.c_void_p(w_ptr)))

    def upload_velocity_ptr(self, u_ptr: int, v_ptr: int, w_ptr: int):
        """Host (ideally pinned) buffers given as raw addresses; histories stay resident."""
        _ck(self._lib.lsb_upload_velocity(self._h, C.c_void_p(u_ptr), C.c_void_p(v_ptr), C.c_void_p(w_ptr)))

    def download_velocity_ptr(self, u_ptr: int, v_ptr: int, w_ptr: int):
        _ck(self._lib.lsb_download_velocity(self._h, C.c_void_p(u_ptr), C.c_void_p(v_ptr), C.c_void_p(w_ptr)))

    def tavg(self, reset: bool = False):
        sh = self.spec_shape()
        out = [np.empty(sh) for _ in range(4)]
        _ck(self._lib.lsb_tavg(self._h, *[_ptr(a) for a in out], C.c_int(1 if reset else 0)))
        return out

    def spanwise_stats(self):
        """Spanwise (y) mean and rms of u + ubar, v, w, p: two arrays (4, nzp, nx)."""
        c = self.st.cfg
        mean = np.empty((4, c.nzp, c.nx))
        rms = np.empty((4, c.nzp, c.nx))
        _ck(self._lib.lsb_spanwise_stats(self._h, _ptr(mean), _ptr(rms)))
        return mean, rms

    def snapshot_async(self, q_ptr: int):
        """q-file fields (u + ubar, v, w, p; physical, [4][nzp][ny][nx]) copied to the host
        address q_ptr on the handle's stream without waiting (lsb_snapshot_async)."""
        _ck(self._lib.lsb_snapshot_async(self._h, C.c_void_p(q_ptr)))

    def timers(self, enable: bool):
        _ck(self._lib.lsb_timers(self._h, C.c_int(1 if enable else 0)))

    def timer_report(self) -> dict:
        buf = C.create_string_buffer(1 << 16)
        _ck(self._lib.lsb_timer_report(self._h, buf, C.c_int(1 << 16)))
        out = {}
        for line in buf.value.decode().splitlines():
            name, n, ms = line.split()
            out[name] = (int(n), float(ms))
        return out

    def diag(self) -> dict:
        d = LsbDiagC()
        _ck(self._lib.lsb_diag(self._h, C.byref(d)))
        return {f: getattr(d, f) for f, _ in LsbDiagC._fields_}

    # ---- tier 1 (the reference's subroutine interfaces)
    def horfft(self, ain: np.ndarray | None, ainf: np.ndarray | None, is_: int):
        if is_ == -1:
            a = np.ascontiguousarray(ain, dtype=np.float64)
            out = np.empty(self.spec_shape())
            _ck(self._lib.lsb_horfft(self._h, _ptr(a), _ptr(out), C.c_int(-1)))
            return out
        f = np.ascontiguousarray(ainf, dtype=np.float64)
        out = np.empty(self.phys_shape())
        _ck(self._lib.lsb_horfft(self._h, _ptr(out), _ptr(f), C.c_int(1)))
        return out

    def _unary(self, name, uf):
        a = np.ascontiguousarray(uf, dtype=np.float64)
        out = np.empty(self.spec_shape())
        _ck(getattr(self._lib, name)(self._h, _ptr(a), _ptr(out)))
        return out

    def dfdx(self, uf):
        return self._unary("lsb_dfdx", uf)

    def dfdy(self, uf):
        return self._unary("lsb_dfdy", uf)

    def dfdz(self, uf):
        return self._unary("lsb_dfdz", uf)

    def d2fdz2(self, uf):
        return self._unary("lsb_d2fdz2", uf)

    def lapl(self, uf):
        return self._unary("lsb_lapl", uf)

    def divuv(self, uf, vf):
        a = np.ascontiguousarray(uf, dtype=np.float64)
        b = np.ascontiguousarray(vf, dtype=np.float64)
        out = np.empty(self.spec_shape())
        _ck(self._lib.lsb_divuv(self._h, _ptr(a), _ptr(b), _ptr(out)))
        return out

    def solve_helmholtz(self, rhs, dtnui):
        r = np.array(rhs, dtype=np.float64, order="C", copy=True)
        _ck(self._lib.lsb_solve_helmholtz(self._h, _ptr(r), C.c_double(dtnui)))
        return r

    def solve_nhom_helmholtz(self, rhs, bc, dtnui):
        r = np.array(rhs, dtype=np.float64, order="C", copy=True)
        b = np.ascontiguousarray(bc, dtype=np.float64)
        _ck(self._lib.lsb_solve_nhom_helmholtz(self._h, _ptr(r), _ptr(b), C.c_double(dtnui)))
        return r

    def dealias_product(self, a, b):
        x = np.ascontiguousarray(a, dtype=np.float64)
        y = np.ascontiguousarray(b, dtype=np.float64)
        out = np.empty(self.phys_shape())
        _ck(self._lib.lsb_dealias_product(self._h, _ptr(x), _ptr(y), _ptr(out)))
        return out

    def nlterm(self, uif):
        u = np.ascontiguousarray(np.asarray(uif), dtype=np.float64)
        out = np.empty((3,) + self.spec_shape())
        _ck(self._lib.lsb_nlterm(self._h, _ptr(u), _ptr(out)))
        return out

    def tau_sgs(self, ui, uiuj, duidxj):
        """ui: (3, nzp, ny, nx+2); uiuj, duidxj: (3, 3, ...) indexed [m][l] as the Fortran (..., l, m)
        storage; returns tau in the same [m][l] storage."""
        a = np.ascontiguousarray(ui, dtype=np.float64)
        b = np.ascontiguousarray(uiuj, dtype=np.float64)
        g = np.ascontiguousarray(duidxj, dtype=np.float64)
        out = np.empty((3, 3) + self.phys_shape())
        _ck(self._lib.lsb_tau_sgs(self._h, _ptr(a), _ptr(b), _ptr(g), _ptr(out)))
        return out


class Batch:
    """Ensemble members stepped together (``lsb_batch_*``).

    ``members`` are open ``Solver`` objects; the batch does not own them and must be closed
    before any of them.  ``step(n)`` advances every member by n time steps, each member's
    result being the one it reaches when stepped alone.
    """

    def __init__(self, members):
        lib = load()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m._h.value for m in self.members])
        self._b = C.c_void_p()
        _ck(lib.lsb_batch_create(arr, C.c_int(len(self.members)), C.byref(self._b)))
        self._lib = lib

    def close(self):
        if getattr(self, "_b", None) and self._b.value:
            self._lib.lsb_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, n: int = 1):
        _ck(self._lib.lsb_batch_step(self._b, C.c_int(n)))

    def synchronize(self):
        _ck(self._lib.lsb_batch_synchronize(self._b))

    def set_stream(self, stream_handle: int | None):
        """Ensemble graphs go to this CUDA stream (raw handle); None restores the batch's own."""
        _ck(self._lib.lsb_batch_set_stream(self._b, C.c_void_p(stream_handle or 0)))

    def graphs(self, enable: bool):
        """One graph launch per ensemble step when steady (default), or member by member."""
        _ck(self._lib.lsb_batch_graphs(self._b, C.c_int(1 if enable else 0)))
