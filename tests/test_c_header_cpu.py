"""include/lsbgpu.h is a plain C99 header: a C program that includes it compiles without
warnings under -pedantic, links against the built library and runs its argument checks
(no device needed) -- the path a C or Fortran (iso_c_binding) driver takes."""
import os
import shutil
import subprocess

import pytest

from lsbflow_b200 import lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r"""
#include <stdio.h>
#include "lsbgpu.h"
int main(void) {
    lsb_batch* b = 0;
    lsb_handle* h = 0;
    lsb_schedule s = {4, 0, 0, 0};
    lsb_config cfg = {0};
    lsb_setup su = {0};
    int bad = 0;
    if (lsb_version() != 1) bad |= 1;
    if (lsb_step(0, 1) != LSB_ERR_ARG) bad |= 2;
    if (lsb_batch_create(0, 1, &b) != LSB_ERR_ARG) bad |= 4;
    if (lsb_set_schedule(0, &s) != LSB_ERR_ARG) bad |= 8;
    if (lsb_snapshot_async(0, 0) != LSB_ERR_ARG) bad |= 16;
    if (lsb_horfft(0, 0, 0, 1) != LSB_ERR_ARG) bad |= 32;
    (void)cfg; (void)su; (void)h;
    printf("%d\n", bad);
    return bad;
}
"""


def test_header_compiles_as_c99_and_links(tmp_path):
    if shutil.which("gcc") is None or not os.path.exists(lib.LIBPATH):
        pytest.skip("gcc or the built library missing")
    src = tmp_path / "t.c"
    src.write_text(PROGRAM)
    exe = tmp_path / "t"
    libdir = os.path.dirname(lib.LIBPATH)
    cc = subprocess.run(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror",
                         "-I", os.path.join(ROOT, "include"), str(src), "-L", libdir, "-llsbgpu",
                         f"-Wl,-rpath,{libdir}", "-o", str(exe)], capture_output=True, text=True)
    assert cc.returncode == 0, cc.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert run.returncode == 0 and run.stdout.strip() == "0", (run.stdout, run.stderr)
