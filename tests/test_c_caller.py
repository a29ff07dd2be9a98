"""A C program compiled against include/FLAME.h and linked with
libflame_b200.so (tests/c_caller/flame_caller.c): the drop-in boundary seen
from C rather than through ctypes.  On CPU the program must compile and
link; on the GPU it runs FLA_Chol, FLA_LU_piv, FLA_LU_piv_solve,
FLA_QR_UT_create_T, FLA_QR_UT, FLA_Apply_Q_UT_create_workspace and
FLA_Apply_Q_UT on host-attached objects and checks every result itself."""
import os
import shutil
import subprocess

import pytest

from conftest import ROOT

SRC = os.path.join(ROOT, "tests", "c_caller", "flame_caller.c")
LIBDIR = os.path.join(ROOT, "libflame_b200")


def _build(tmp_path):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    if not os.path.exists(os.path.join(LIBDIR, "libflame_b200.so")):
        pytest.skip("libflame_b200.so is not built")
    exe = str(tmp_path / "flame_caller")
    cmd = [cc, "-std=c99", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L", LIBDIR, "-l:libflame_b200.so", "-Wl,-rpath," + LIBDIR, "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    _build(tmp_path)


@pytest.mark.gpu
def test_c_caller_runs_and_checks(tmp_path):
    exe = _build(tmp_path)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
