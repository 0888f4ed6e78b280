"""The C-ABI library builds, loads on a machine without a GPU, exports every symbol the
header declares, and fails loudly (no silent CPU path) when no device is present."""
import os
import re

import pytest

from lsbflow_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "lsbgpu.h")).read()
    return sorted(set(re.findall(r"\b(lsb_[a-z0-9_]+)\s*\(", txt)))


def test_header_and_binding_agree():
    assert header_symbols() == sorted(lib.EXPORTS)


def test_library_exports_every_symbol():
    if not os.path.exists(lib.LIBPATH):
        pytest.skip("library not built")
    l = lib.load()
    for name in header_symbols():
        assert hasattr(l, name), name
    assert l.lsb_version() == 1


def test_create_fails_loudly_without_device():
    import torch
    if torch.cuda.is_available() or not os.path.exists(lib.LIBPATH):
        pytest.skip("a device is present or the library is not built")
    from lsbflow_b200 import hostsetup as hs
    from lsbflow_b200.config import workload
    with pytest.raises(lib.LsbError):
        lib.Solver(hs.make_setup(workload("dns64", nx=16, ny=8, nz=16)))


def test_new_entry_points_reject_null_arguments_before_any_device_work():
    """Argument checks of the ensemble, schedule and snapshot calls need no device."""
    import ctypes as C
    if not os.path.exists(lib.LIBPATH):
        pytest.skip("library not built")
    l = lib.load()
    b = C.c_void_p()
    assert l.lsb_batch_create(None, C.c_int(2), C.byref(b)) == -1
    arr = (C.c_void_p * 2)(None, None)
    assert l.lsb_batch_create(arr, C.c_int(2), C.byref(b)) == -1
    assert b"null member" in l.lsb_last_error()
    assert l.lsb_batch_create(arr, C.c_int(0), C.byref(b)) == -1
    assert l.lsb_batch_step(None, C.c_int(1)) == -1
    assert l.lsb_batch_synchronize(None) == -1
    assert l.lsb_batch_graphs(None, C.c_int(0)) == -1
    assert l.lsb_batch_set_stream(None, None) == -1
    assert l.lsb_batch_destroy(None) == 0          # like free(NULL)
    sc = lib.LsbScheduleC(4, 0)
    assert l.lsb_set_schedule(None, C.byref(sc)) == -1
    assert l.lsb_get_schedule(None, C.byref(sc)) == -1
    assert l.lsb_snapshot_async(None, None) == -1
    assert l.lsb_step(None, C.c_int(1)) == -1
