"""FLA_LU_piv on the GPU against the CPU oracle.

Bar (FP64 plain form): the pivot vector is identical to the oracle's (the
reference's, bit for bit); the factors agree within 1e-12 normwise
(relative Frobenius); the backward error ||PA - LU||_F/(n eps ||A||_F) is at
most the oracle's own plus 1.0; the first null pivot index is identical."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_fro, seeded, to_dev, to_host

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-12


def run_lu(cuda, flame, A):
    torch = cuda
    Ad = to_dev(cuda, A)
    p = torch.zeros(min(A.shape), dtype=torch.int32, device="cuda")
    r = flame.lu_piv(Ad, p)
    return to_host(Ad), p.cpu().numpy(), r


@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (7, 5), (5, 7), (64, 64), (129, 129), (200, 150),
                                 (150, 200), (300, 300), (513, 257), (1024, 1024),
                                 # tall panels: 16-CTA clusters with 1024 and more rows per CTA
                                 (16384, 48), (20000, 64), (40000, 24)])
def test_lu_matches_oracle(cuda, flame, oracle, m, n):
    rng = seeded(m * 7 + n)
    A = rng.uniform(-1, 1, (m, n))
    LU, p, r = run_lu(cuda, flame, A)
    LUo, po, ro = oracle.lu_piv(A)
    assert r == ro == flame.FLA_SUCCESS, flame.last_error()
    assert np.array_equal(p, po)
    assert rel_fro(LU, LUo) < FACTOR_TOL
    be, be_o = oracle.lu_backward_error(A, LU, p), oracle.lu_backward_error(A, LUo, po)
    assert be <= be_o + 1.0, (be, be_o)


def test_lu_golden_fixtures(cuda, flame, golden):
    for key in ["1x1", "33x17", "17x33", "130x130", "160x120", "ties", "null"]:
        A = golden["lu_%s_A" % key]
        LU, p, r = run_lu(cuda, flame, A)
        assert np.array_equal(p, golden["lu_%s_p" % key]), key
        assert r == int(golden["lu_%s_r" % key]), key
        assert rel_fro(LU, golden["lu_%s_LU" % key]) < FACTOR_TOL, key


@pytest.mark.parametrize("zero_col", [0, 3, 128, 200])
def test_lu_null_pivot(cuda, flame, oracle, zero_col):
    rng = seeded(500 + zero_col)
    A = rng.uniform(-1, 1, (260, 260))
    A[:, zero_col] = 0.0
    LU, p, r = run_lu(cuda, flame, A)
    LUo, po, ro = oracle.lu_piv(A)
    assert r == ro == zero_col
    assert np.array_equal(p, po)
    assert rel_fro(LU, LUo) < FACTOR_TOL


def test_lu_ties_first_max_wins(cuda, flame, oracle):
    rng = seeded(9)
    A = rng.integers(-3, 4, (300, 300)).astype(np.float64)
    LU, p, r = run_lu(cuda, flame, A)
    LUo, po, ro = oracle.lu_piv(A)
    assert np.array_equal(p, po)
    assert r == ro


def test_lu_host_buffers(cuda, flame, oracle):
    rng = seeded(10)
    A = rng.uniform(-1, 1, (301, 299))
    H = np.asfortranarray(A.copy())
    p = np.zeros(299, dtype=np.int32)
    assert flame.lu_piv(H, p) == flame.FLA_SUCCESS
    LUo, po, _ = oracle.lu_piv(A)
    assert np.array_equal(p, po)
    assert rel_fro(H, LUo) < FACTOR_TOL


def test_apply_pivots_and_shift(cuda, flame, oracle):
    rng = seeded(11)
    A = rng.uniform(-1, 1, (200, 200))
    _, po, _ = oracle.lu_piv(A)
    B = rng.standard_normal((200, 9))
    Bd = to_dev(cuda, B)
    pd = cuda.from_numpy(po.copy()).cuda()
    assert flame.apply_pivots(pd, Bd) == flame.FLA_SUCCESS
    assert np.array_equal(to_host(Bd), oracle.apply_pivots(po, B))
    assert flame.apply_pivots(pd, Bd, flame.FLA_TRANSPOSE) == flame.FLA_SUCCESS
    assert np.array_equal(to_host(Bd), B)
    assert flame.shift_pivots_to(flame.FLA_LAPACK_PIVOTS, pd) == flame.FLA_SUCCESS
    assert np.array_equal(pd.cpu().numpy(), oracle.shift_pivots(po, True))
    assert flame.shift_pivots_to(flame.FLA_NATIVE_PIVOTS, pd) == flame.FLA_SUCCESS
    assert np.array_equal(pd.cpu().numpy(), po)


def test_dgetrf_lapack_abi(cuda, flame, golden):
    A = golden["dgetrf_A"]
    a = np.asfortranarray(A.copy())
    n = C.c_int(a.shape[0])
    ipiv = np.zeros(a.shape[0], dtype=np.int32)
    info = C.c_int(99)
    flame.lib().dgetrf_(C.byref(n), C.byref(n), a.ctypes.data_as(C.c_void_p), C.byref(n),
                        ipiv.ctypes.data_as(C.c_void_p), C.byref(info))
    assert info.value == 0
    assert np.array_equal(ipiv, golden["dgetrf_ipiv"])
    assert rel_fro(a, golden["dgetrf_LU"]) < FACTOR_TOL


def test_lu_bitwise_repeatable(cuda, flame):
    """Five factorizations of one matrix (n = 4096, panels on the second
    stream beside the trailing updates) give bitwise identical factors and
    pivots."""
    torch = cuda
    n = 4096
    g = torch.Generator(device="cuda").manual_seed(4)
    A = torch.rand((n, n), dtype=torch.float64, device="cuda", generator=g) * 2 - 1
    W = torch.empty_like(A).t()
    p = torch.empty(n, dtype=torch.int32, device="cuda")
    ref = refp = None
    for _ in range(5):
        W.copy_(A.t())
        torch.cuda.synchronize()
        assert flame.lu_piv(W, p) == flame.FLA_SUCCESS
        if ref is None:
            ref, refp = W.clone(), p.clone()
        else:
            assert torch.equal(W, ref) and torch.equal(p, refp)
