"""The drop-in boundary from plain C, without a GPU: include/conductor_rigid.h compiles as
C99 under -pedantic, and a C program links against libconductor_rigid.so and calls its
host-only entry points (what a cgo or C caller of the plugin would do first)."""
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent

C_SOURCE = r"""
#include <stdio.h>
#include "conductor_rigid.h"
int main(void) {
    cr_batch *b = 0;
    cr_derived d;
    cr_params p = {0};
    const double L[3] = {16.0, 16.0, 16.0};
    if (cr_abi_version() != CR_ABI_VERSION) return 1;
    if (cr_batch_create(0, 0, &b) != CR_BAD_PARAM || b) return 2;
    if (cr_destroy(0) != CR_BAD_PARAM) return 3;
    p.xi = 0.8;
    p.errortol = 1e-5;
    if (cr_derive_params(&p, L, &d) != CR_OK) return 4;
    printf("%d %d %d %d\n", d.grid[0], d.grid[1], d.grid[2], d.support);
    return 0;
}
"""


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_header_is_c99_and_links(product_lib, tmp_path):
    src = tmp_path / "caller.c"
    src.write_text(C_SOURCE)
    exe = tmp_path / "caller"
    lib_dir = product_lib.LIB_PATH.parent
    cmd = ["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I", str(ROOT / "include"), str(src),
           "-L", str(lib_dir), "-lconductor_rigid", f"-Wl,-rpath,{lib_dir}", "-o", str(exe)]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    run = subprocess.run([str(exe)], capture_output=True, text=True)
    assert run.returncode == 0, (run.returncode, run.stderr)
    # the derived mesh and support of the C caller equal those of the Python binding
    p = product_lib.make_params(xi=0.8, errortol=1e-5)
    d = product_lib.derive_params(p, (16.0, 16.0, 16.0))
    assert run.stdout.split() == [str(v) for v in (*d.grid, d.support)]
