"""FLA_Chol_solve / FLA_LU_piv_solve and the dposv_/dgesv_/dpotrs_/dgetrs_
LAPACK entry points on the GPU against the oracle and the reference's
fixtures.  Solutions agree within 1e-12 normwise relative (the systems are
well conditioned); pivots are identical."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_fro, seeded, spd, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.mark.parametrize("n,nrhs", [(1, 1), (100, 3), (257, 5), (600, 32)])
def test_chol_solve(cuda, flame, oracle, n, nrhs):
    rng = seeded(n + nrhs)
    A = spd(rng, n)
    B = rng.standard_normal((n, nrhs))
    Lo, _ = oracle.chol(A)
    Xo = oracle.chol_solve(Lo, B)
    Ld, Bd = to_dev(cuda, Lo), to_dev(cuda, B)
    Xd = to_dev(cuda, np.zeros_like(B))
    assert flame.chol_solve(Ld, Bd, Xd) == flame.FLA_SUCCESS
    assert rel_fro(to_host(Xd), Xo) < TOL
    # upper: A = U^T U with U = L^T
    Ud = to_dev(cuda, np.triu(Lo.T))
    assert flame.chol_solve(Ud, Bd, Xd, flame.FLA_UPPER_TRIANGULAR) == flame.FLA_SUCCESS
    assert rel_fro(to_host(Xd), Xo) < TOL


@pytest.mark.parametrize("n,nrhs", [(1, 1), (100, 3), (257, 5), (600, 32)])
def test_lu_piv_solve(cuda, flame, oracle, n, nrhs):
    rng = seeded(10 * n + nrhs)
    A = rng.uniform(-1, 1, (n, n))
    B = rng.standard_normal((n, nrhs))
    LUo, po, _ = oracle.lu_piv(A)
    Xo = oracle.lu_piv_solve(LUo, po, B)
    Ad, Bd = to_dev(cuda, LUo), to_dev(cuda, B)
    pd = cuda.from_numpy(po.copy()).cuda()
    Xd = to_dev(cuda, np.zeros_like(B))
    assert flame.lu_piv_solve(Ad, pd, Bd, Xd) == flame.FLA_SUCCESS
    assert rel_fro(to_host(Xd), Xo) < TOL


def test_solve_golden(cuda, flame, golden, oracle):
    L, _ = oracle.chol(golden["chol_solve_A"])
    Xd = to_dev(cuda, np.zeros_like(golden["chol_solve_B"]))
    assert flame.chol_solve(to_dev(cuda, L), to_dev(cuda, golden["chol_solve_B"]), Xd) == flame.FLA_SUCCESS
    assert rel_fro(to_host(Xd), golden["chol_solve_X"]) < TOL


def _ip(v):
    return C.byref(C.c_int(v))


def test_dposv_dgesv_host_pointers(cuda, flame, golden):
    L = flame.lib()
    A, B = golden["dposv_A"], golden["dposv_B"]
    a, b = np.asfortranarray(A.copy()), np.asfortranarray(B.copy())
    n, nrhs = A.shape[0], B.shape[1]
    info = C.c_int(9)
    L.dposv_(C.c_char_p(b"L"), _ip(n), _ip(nrhs), a.ctypes.data_as(C.c_void_p), _ip(n),
             b.ctypes.data_as(C.c_void_p), _ip(n), C.byref(info))
    assert info.value == 0
    assert rel_fro(b, golden["dposv_X"]) < TOL
    A, B = golden["dgesv_A"], golden["dposv_B"]
    a, b = np.asfortranarray(A.copy()), np.asfortranarray(B.copy())
    ipiv = np.zeros(n, dtype=np.int32)
    L.dgesv_(_ip(n), _ip(nrhs), a.ctypes.data_as(C.c_void_p), _ip(n), ipiv.ctypes.data_as(C.c_void_p),
             b.ctypes.data_as(C.c_void_p), _ip(n), C.byref(info))
    assert info.value == 0
    assert np.array_equal(ipiv, golden["dgesv_ipiv"])
    assert rel_fro(b, golden["dgesv_X"]) < TOL


def test_dgetrs_transpose_and_device_pointers(cuda, flame, oracle):
    torch = cuda
    L = flame.lib()
    rng = seeded(31)
    n, nrhs = 300, 4
    A = rng.uniform(-1, 1, (n, n))
    B = rng.standard_normal((n, nrhs))
    Ad = to_dev(cuda, A)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = C.c_int(9)
    L.dgetrf_(_ip(n), _ip(n), C.c_void_p(Ad.data_ptr()), _ip(n), C.c_void_p(ipiv.data_ptr()), C.byref(info))
    assert info.value == 0
    Bd = to_dev(cuda, B)
    L.dgetrs_(C.c_char_p(b"T"), _ip(n), _ip(nrhs), C.c_void_p(Ad.data_ptr()), _ip(n),
              C.c_void_p(ipiv.data_ptr()), C.c_void_p(Bd.data_ptr()), _ip(n), C.byref(info))
    assert info.value == 0
    X = to_host(Bd)
    assert rel_fro(A.T @ X, B) < 1e-11
    Bd = to_dev(cuda, B)
    L.dgetrs_(C.c_char_p(b"N"), _ip(n), _ip(nrhs), C.c_void_p(Ad.data_ptr()), _ip(n),
              C.c_void_p(ipiv.data_ptr()), C.c_void_p(Bd.data_ptr()), _ip(n), C.byref(info))
    assert rel_fro(A @ to_host(Bd), B) < 1e-11


def test_dgetrs_transpose_matches_oracle(cuda, flame, oracle):
    """dgetrs_ 'T' against the oracle's restatement of dgetrs' transposed
    branch on the oracle's own factor (identical pivots)."""
    torch = cuda
    L = flame.lib()
    rng = seeded(37)
    n, nrhs = 260, 6
    A = rng.uniform(-1, 1, (n, n))
    B = rng.standard_normal((n, nrhs))
    Ad = to_dev(cuda, A)
    ipiv = torch.zeros(n, dtype=torch.int32, device="cuda")
    info = C.c_int(9)
    L.dgetrf_(_ip(n), _ip(n), C.c_void_p(Ad.data_ptr()), _ip(n), C.c_void_p(ipiv.data_ptr()), C.byref(info))
    assert info.value == 0
    LUo, po, ro = oracle.lu_piv(A)
    assert np.array_equal(ipiv.cpu().numpy() - 1 - np.arange(n), po)
    Bd = to_dev(cuda, B)
    L.dgetrs_(C.c_char_p(b"T"), _ip(n), _ip(nrhs), C.c_void_p(Ad.data_ptr()), _ip(n),
              C.c_void_p(ipiv.data_ptr()), C.c_void_p(Bd.data_ptr()), _ip(n), C.byref(info))
    assert info.value == 0
    Xo = oracle.lu_piv_solve_t(LUo, po, B)
    assert rel_fro(to_host(Bd), Xo) < TOL
    assert rel_fro(A.T @ Xo, B) < 1e-11  # the restatement itself solves A^T X = B


def test_dposv_upper_matches_oracle(cuda, flame, oracle):
    """dposv_ 'U' on host buffers: the upper factor against the transpose of
    the oracle's lower factor (U = L^T for the same A), and X against the
    oracle's upper Cholesky solve."""
    L = flame.lib()
    rng = seeded(41)
    n, nrhs = 230, 4
    A = spd(rng, n)
    B = rng.standard_normal((n, nrhs))
    a = np.asfortranarray(A.copy())
    b = np.asfortranarray(B.copy())
    info = C.c_int(9)
    L.dposv_(C.c_char_p(b"U"), _ip(n), _ip(nrhs), a.ctypes.data_as(C.c_void_p), _ip(n),
             b.ctypes.data_as(C.c_void_p), _ip(n), C.byref(info))
    assert info.value == 0
    Lo, ro = oracle.chol(A)
    Uo = np.triu(Lo.T)
    assert rel_fro(np.triu(a), Uo) < TOL
    assert np.array_equal(np.tril(a, -1), np.tril(A, -1))  # the strictly lower part is not referenced
    Xo = oracle.chol_solve_u(Uo, B)
    assert rel_fro(b, Xo) < TOL
    assert rel_fro(A @ Xo, B) < 1e-11
