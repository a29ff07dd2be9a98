"""ctypes binding to the CPU restatement oracle (oracle/flame_oracle.c).

Test infrastructure only: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py as the checker; the product never imports
it.  All arrays are float64, Fortran-ordered copies; inputs are not
modified.
"""
import ctypes as C
import os
import subprocess
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libflame_oracle.so")
SUCCESS = -1
_L = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "libflame_oracle.so"], check=True)


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(
                os.path.join(HERE, "flame_oracle.c")):
            build()
        _L = C.CDLL(LIB_PATH)
        for f in ["orc_chol_l", "orc_lu_piv"]:
            getattr(_L, f).restype = C.c_int
    return _L


def _f(a):
    return np.array(a, dtype=np.float64, order="F", copy=True)


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def chol(A, nb=128, nb_inner=32):
    """FLA_Chol(FLA_LOWER_TRIANGULAR, A) restated; returns (A', rval)."""
    a = _f(A)
    n = a.shape[0]
    r = lib().orc_chol_l(n, _p(a), max(n, 1), nb, nb_inner)
    return a, r


def lu_piv(A, nb=128, nb_inner=16):
    """FLA_LU_piv restated; returns (LU, relative zero-based pivots, rval)."""
    a = _f(A)
    m, n = a.shape
    p = np.zeros(min(m, n), dtype=np.int32)
    r = lib().orc_lu_piv(m, n, _p(a), max(m, 1), _p(p), nb, nb_inner)
    return a, p, r


def qr_ut(A, b_alg=None):
    """FLA_QR_UT restated; returns (A', T) with T b_alg x n."""
    a = _f(A)
    m, n = a.shape
    if b_alg is None:
        b_alg = min(32, min(m, n))
    t = np.zeros((b_alg, n), order="F")
    lib().orc_qr_ut(m, n, _p(a), max(m, 1), _p(t), max(b_alg, 1), b_alg)
    return a, t


def apply_qt(A, T, B):
    """FLA_Apply_Q_UT(LEFT, CONJ_TRANSPOSE, FORWARD, COLUMNWISE) restated: Q^T B."""
    a = _f(A)
    t = _f(T)
    b = _f(B)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    m, k = a.shape
    lib().orc_apply_qt(m, k, _p(a), max(m, 1), _p(t), max(t.shape[0], 1), t.shape[0],
                       b.shape[1], _p(b), max(m, 1))
    return b


def chol_solve(Lfac, B):
    a = _f(Lfac)
    b = _f(B)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    n = a.shape[0]
    lib().orc_chol_solve_l(n, b.shape[1], _p(a), max(n, 1), _p(b), max(n, 1))
    return b


def lu_piv_solve(LU, p, B):
    a = _f(LU)
    b = _f(B)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    pp = np.ascontiguousarray(p, dtype=np.int32)
    n = a.shape[0]
    lib().orc_lu_piv_solve(n, b.shape[1], _p(a), max(n, 1), _p(pp), _p(b), max(n, 1))
    return b


def _trsm_lut(U, B):
    """B := inv(U^T) B, U upper non-unit: netlib dtrsm Left/Upper/Transpose,
    rows in ascending order (each row's dot product vectorized)."""
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    for i in range(b.shape[0]):
        b[i] = (b[i] - U[:i, i] @ b[:i]) / U[i, i]
    return b


def _trsm_lltu(L, B):
    """B := inv(L^T) B, L unit lower: netlib dtrsm Left/Lower/Transpose/Unit,
    rows in descending order."""
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    for i in range(b.shape[0] - 1, -1, -1):
        b[i] = b[i] - L[i + 1:, i] @ b[i + 1:]
    return b


def _trsm_lun(U, B):
    """B := inv(U) B, U upper non-unit: dtrsm Left/Upper/No transpose, rows
    descending."""
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    for i in range(b.shape[0] - 1, -1, -1):
        b[i] = (b[i] - U[i, i + 1:] @ b[i + 1:]) / U[i, i]
    return b


def lu_piv_solve_t(LU, p, B):
    """A^T X = B from FLA_LU_piv's factor (relative pivots p): the TRANS = 'T'
    branch of dgetrs (src/map/common/lapacksrc/f2c/dgetrs.c:201-205): X :=
    inv(U^T) B, X := inv(L^T) X (unit), then the interchanges in reverse
    order (dlaswp with incx = -1).  NumPy restatement for small cases."""
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    lu = np.asarray(LU, dtype=np.float64)
    b = _trsm_lltu(lu, _trsm_lut(lu, b))
    return apply_pivots(p, b, transpose=True)


def chol_solve_u(Ufac, B):
    """X := inv(A) B with A = U^T U (upper factor), FLA_Chol_solve's upper
    branch (src/lapack/dec/chol/front/flamec/FLA_Chol_solve.c:29-34): X :=
    inv(U^T) B, then X := inv(U) X.  NumPy restatement for small cases."""
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    u = np.asarray(Ufac, dtype=np.float64)
    return _trsm_lun(u, _trsm_lut(u, b))


def apply_pivots(p, A, transpose=False):
    a = _f(A)
    if a.ndim == 1:
        a = a.reshape(-1, 1, order="F")
    pp = np.ascontiguousarray(p, dtype=np.int32)
    f = lib().orc_apply_pivots_lt if transpose else lib().orc_apply_pivots_ln
    f(a.shape[1], _p(a), max(a.shape[0], 1), 0, len(pp) - 1, _p(pp))
    return a


def trsm_lln(L, B, unit=False):
    a = _f(L)
    b = _f(B)
    lib().orc_trsm_lln(b.shape[0], b.shape[1], int(unit), _p(a), max(a.shape[0], 1), _p(b), max(b.shape[0], 1))
    return b


def trsm_llt(L, B):
    a = _f(L)
    b = _f(B)
    lib().orc_trsm_llt(b.shape[0], b.shape[1], _p(a), max(a.shape[0], 1), _p(b), max(b.shape[0], 1))
    return b


def shift_pivots(p, to_lapack=True):
    pp = np.array(p, dtype=np.int32, copy=True)
    lib().orc_shift_pivots(len(pp), _p(pp), int(to_lapack))
    return pp


# ---- backward-error metrics used by every parity test ---------------------

def chol_backward_error(A, Lfac):
    """||A - L L^T||_F / (n * eps * ||A||_F), lower triangle of Lfac."""
    L = np.tril(Lfac)
    n = A.shape[0]
    return np.linalg.norm(A - L @ L.T) / (n * np.finfo(float).eps * np.linalg.norm(A))


def lu_backward_error(A, LU, p):
    """||P A - L U||_F / (n * eps * ||A||_F) with P from relative pivots p."""
    m, n = LU.shape
    k = min(m, n)
    L = np.tril(LU[:, :k], -1) + np.eye(m, k)
    U = np.triu(LU[:k, :])
    PA = apply_pivots(p, A)
    return np.linalg.norm(PA - L @ U) / (max(m, n) * np.finfo(float).eps * np.linalg.norm(A))


def form_q(A, T, m_cols=None):
    """Explicit Q (m x m_cols) from the UT representation, via Q = Q^T^T:
    Q^T applied to I gives Q^T; its transpose is Q."""
    m = A.shape[0]
    Qt = apply_qt(A, T, np.eye(m))
    Q = Qt.T
    return Q if m_cols is None else Q[:, :m_cols]


def qr_backward_error(A, QR, T):
    """||A - Q R||_F / (max(m,n) * eps * ||A||_F)."""
    m, n = A.shape
    k = min(m, n)
    R = np.triu(QR[:k, :])
    Q = form_q(QR, T, k)
    return np.linalg.norm(A - Q @ R) / (max(m, n) * np.finfo(float).eps * np.linalg.norm(A))
