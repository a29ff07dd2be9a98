"""The C-ABI library loads and exports every function declared in
include/*.h; host-side argument checks behave like the reference's
(LAPACK xerbla convention).  CPU only: no compute call reaches the GPU."""
import ctypes as C
import glob
import os
import re

import pytest

from conftest import ROOT

DECL = re.compile(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(([^;{]*)\)\s*;", re.M)


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        src = re.sub(r"//.*", "", src)
        src = re.sub(r"#.*", "", src)
        for m in DECL.finditer(src):
            name = m.group(1)
            if name in ("if", "while", "for", "return", "sizeof"):
                continue
            names.add(name)
    return sorted(names)


def test_headers_declare_the_path():
    names = declared_functions()
    for must in ["FLA_Init", "FLA_Chol", "FLA_LU_piv", "FLA_QR_UT", "FLA_Apply_Q_UT",
                 "FLA_Chol_solve", "FLA_LU_piv_solve", "FLA_Apply_pivots", "FLA_Shift_pivots_to",
                 "dpotrf_", "dgetrf_", "dgeqrf_", "dposv_", "dgesv_"]:
        assert must in names


def test_library_exports_every_declared_symbol(flame):
    L = flame.lib()
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, "declared in include/*.h but not exported: %s" % missing


def _ip(v):
    return C.byref(C.c_int(v))


def test_lapack_argument_checks_follow_xerbla(flame, capfd):
    L = flame.lib()
    info = C.c_int(0)
    a = (C.c_double * 4)()
    # dpotrf_: bad uplo -> info = -1; bad lda -> info = -4 (dpotrf_check)
    r = L.dpotrf_(C.c_char_p(b"X"), _ip(2), a, _ip(2), C.byref(info))
    assert info.value == -1 and r == -2
    r = L.dpotrf_(C.c_char_p(b"L"), _ip(2), a, _ip(1), C.byref(info))
    assert info.value == -4
    out = capfd.readouterr().out
    assert "On entry to DPOTRF" in out and "parameter number  4" in out
    # n == 0: quick return with info = 0 and no device work
    r = L.dpotrf_(C.c_char_p(b"L"), _ip(0), a, _ip(1), C.byref(info))
    assert info.value == 0 and r == 0
    ipiv = (C.c_int * 2)()
    L.dgetrf_(_ip(-1), _ip(2), a, _ip(2), ipiv, C.byref(info))
    assert info.value == -1
    L.dgetrf_(_ip(3), _ip(2), a, _ip(2), ipiv, C.byref(info))
    assert info.value == -4
    L.dgesv_(_ip(2), _ip(-1), a, _ip(2), ipiv, a, _ip(2), C.byref(info))
    assert info.value == -2
    L.dposv_(C.c_char_p(b"U"), _ip(2), _ip(1), a, _ip(2), a, _ip(1), C.byref(info))
    assert info.value == -7


def test_error_level_roundtrip(flame):
    L = flame.lib()
    old = L.FLA_Check_error_level_set(flame.FLA_MIN_ERROR_CHECKING)
    assert L.FLA_Check_error_level() == flame.FLA_MIN_ERROR_CHECKING
    L.FLA_Check_error_level_set(old)
    assert L.FLA_Check_error_level() == old
