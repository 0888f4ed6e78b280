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
