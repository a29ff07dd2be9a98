"""FLA_QR_UT / FLA_Apply_Q_UT / FLA_QR_UT_recover_tau / dgeqrf_ on the GPU
against the CPU oracle and the reference's fixtures.

Bar: R and the Householder vectors (the factored A) agree with the oracle
within 1e-12 normwise; the defined entries of T (upper triangle of each
b x b block) within 1e-12 normwise; ||A - QR||_F/(max(m,n) eps ||A||_F) at
most the oracle's own + 1.0; Q^T B within 1e-12 normwise."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_fro, seeded, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL = 1e-12


def t_mask(T, k):
    b = T.shape[0]
    mask = np.zeros(T.shape, dtype=bool)
    for j in range(k):
        mask[: (j % b) + 1, j] = True
    return mask


def run_qr(cuda, flame, A):
    m, n = A.shape
    b = min(32, m, n)
    Ad = to_dev(cuda, A)
    Td = to_dev(cuda, np.zeros((b, n)))
    r = flame.qr_ut(Ad, Td)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    return to_host(Ad), to_host(Td)


@pytest.mark.parametrize("m,n", [(1, 1), (5, 3), (3, 5), (40, 40), (64, 64), (65, 64), (130, 100),
                                 (100, 130), (300, 200), (513, 257), (1000, 640)])
def test_qr_ut_matches_oracle(cuda, flame, oracle, m, n):
    rng = seeded(m * 13 + n)
    A = rng.standard_normal((m, n))
    QR, T = run_qr(cuda, flame, A)
    QRo, To = oracle.qr_ut(A)
    assert rel_fro(QR, QRo) < TOL
    mask = t_mask(To, min(m, n))
    assert rel_fro(T[mask], To[mask]) < TOL
    be, be_o = oracle.qr_backward_error(A, QR, T), oracle.qr_backward_error(A, QRo, To)
    assert be <= be_o + 1.0, (be, be_o)


# Tall panels and other T block sizes: 16-CTA cluster leaves of width 32
# (8000 rows), 16 (9000, 20000 rows) and 8, pieces beyond any cluster
# (40000 rows: the cooperative panel kernel), the recursive panel's T
# assembly, panels of 96 (b = 48) and 200 (b = 200) columns.
@pytest.mark.parametrize("m,n,b", [(8000, 96, 32), (9000, 64, 32), (20000, 40, 32), (40000, 24, 8),
                                   (3000, 200, 48), (600, 300, 200), (700, 520, 16)])
def test_qr_ut_tall_and_block_sizes(cuda, flame, oracle, m, n, b):
    rng = seeded(m * 17 + n + b)
    A = rng.standard_normal((m, n))
    Ad = to_dev(cuda, A)
    Td = to_dev(cuda, np.zeros((b, n)))
    assert flame.qr_ut(Ad, Td) == flame.FLA_SUCCESS, flame.last_error()
    QR, T = to_host(Ad), to_host(Td)
    QRo, To = oracle.qr_ut(A, b)
    assert rel_fro(QR, QRo) < TOL
    mask = t_mask(To, min(m, n))
    assert rel_fro(T[mask], To[mask]) < TOL
    be, be_o = _be_tall(oracle, A, QR, T), _be_tall(oracle, A, QRo, To)
    assert be <= be_o + 1.0, (be, be_o)


def _be_tall(oracle, A, QR, T):
    """||Q^T A - [R; 0]||_F / (max(m,n) eps ||A||_F), equal to ||A - QR|| for
    an orthogonal Q, without forming the m x m Q."""
    m, n = A.shape
    k = min(m, n)
    R = np.zeros((m, n))
    R[:k] = np.triu(QR[:k, :])
    return np.linalg.norm(oracle.apply_qt(QR, T, A) - R) / (max(m, n) * np.finfo(float).eps * np.linalg.norm(A))


def test_qr_golden(cuda, flame, golden):
    for key in ["40x40", "130x64", "160x80"]:
        A = golden["qr_%s_A" % key]
        QR, T = run_qr(cuda, flame, A)
        assert rel_fro(QR, golden["qr_%s_QR" % key]) < TOL
        Tg = golden["qr_%s_T" % key]
        mask = t_mask(Tg, min(A.shape))
        assert rel_fro(T[mask], Tg[mask]) < TOL
        Bd = to_dev(cuda, golden["qr_%s_B" % key])
        assert flame.apply_q_ut(to_dev(cuda, golden["qr_%s_QR" % key]), to_dev(cuda, Tg), Bd) == flame.FLA_SUCCESS
        assert rel_fro(to_host(Bd), golden["qr_%s_QtB" % key]) < TOL


@pytest.mark.parametrize("m,n,nrhs", [(200, 120, 7), (600, 600, 64), (1030, 500, 3)])
def test_apply_q_ut(cuda, flame, oracle, m, n, nrhs):
    rng = seeded(m + n + nrhs)
    A = rng.standard_normal((m, n))
    QRo, To = oracle.qr_ut(A)
    B = rng.standard_normal((m, nrhs))
    ref = oracle.apply_qt(QRo, To, B)
    Ad, Td, Bd = to_dev(cuda, QRo), to_dev(cuda, To), to_dev(cuda, B)
    assert flame.apply_q_ut(Ad, Td, Bd) == flame.FLA_SUCCESS
    assert rel_fro(to_host(Bd), ref) < TOL
    # Q (Q^T B) = B
    assert flame.apply_q_ut(Ad, Td, Bd, flame.FLA_NO_TRANSPOSE) == flame.FLA_SUCCESS
    assert rel_fro(to_host(Bd), B) < 1e-13


def test_recover_tau_and_dgeqrf(cuda, flame, golden, oracle):
    A = golden["dgeqrf_A"]
    m, n = A.shape
    QRo, To = oracle.qr_ut(A)
    Td = to_dev(cuda, To)
    t = cuda.zeros(min(m, n), dtype=cuda.float64, device="cuda")
    assert flame.qr_ut_recover_tau(Td, t) == flame.FLA_SUCCESS
    exp = np.array([To[j % To.shape[0], j] for j in range(min(m, n))])
    assert np.array_equal(t.cpu().numpy(), exp)
    a = np.asfortranarray(A.copy())
    tau = np.zeros(min(m, n))
    work = np.zeros(n * 32)
    info = C.c_int(9)
    mm, nn, lw = C.c_int(m), C.c_int(n), C.c_int(n * 32)
    flame.lib().dgeqrf_(C.byref(mm), C.byref(nn), a.ctypes.data_as(C.c_void_p), C.byref(mm),
                        tau.ctypes.data_as(C.c_void_p), work.ctypes.data_as(C.c_void_p), C.byref(lw), C.byref(info))
    assert info.value == 0
    assert rel_fro(a, golden["dgeqrf_QR"]) < TOL
    assert rel_fro(tau, golden["dgeqrf_tau"]) < TOL


def test_create_t_and_workspace_objects(cuda, flame, oracle):
    """FLA_QR_UT_create_T and FLA_Apply_Q_UT_create_workspace through the
    C-ABI: the objects they allocate (in HBM) have the reference's shapes
    (T: min(32, min_dim) x width(A); W: length(T) x max_dim(B), as
    FLA_Apply_Q_UT_create_workspace.c:19-22) and drive
    FLA_QR_UT and FLA_Apply_Q_UT to the oracle's results; FLA_Obj_free
    releases them."""
    L = flame.lib()
    rng = seeded(53)
    m, n, nrhs = 300, 180, 5
    A = rng.standard_normal((m, n))
    B = rng.standard_normal((m, nrhs))
    Ad, Bd = to_dev(cuda, A), to_dev(cuda, B)
    va, vb = flame.View(Ad), flame.View(Bd)
    T, W = flame.FLA_Obj(), flame.FLA_Obj()
    assert L.FLA_QR_UT_create_T(va.obj, C.byref(T)) == flame.FLA_SUCCESS
    assert (L.FLA_Obj_length(T), L.FLA_Obj_width(T)) == (32, n)
    assert L.FLA_QR_UT(va.obj, T) == flame.FLA_SUCCESS, flame.last_error()
    assert L.FLA_Apply_Q_UT_create_workspace(T, vb.obj, C.byref(W)) == flame.FLA_SUCCESS
    assert (L.FLA_Obj_length(W), L.FLA_Obj_width(W)) == (32, max(m, nrhs))
    assert L.FLA_Apply_Q_UT(flame.FLA_LEFT, flame.FLA_CONJ_TRANSPOSE, flame.FLA_FORWARD, flame.FLA_COLUMNWISE,
                            va.obj, T, W, vb.obj) == flame.FLA_SUCCESS, flame.last_error()
    QRo, To = oracle.qr_ut(A)
    assert rel_fro(to_host(Ad), QRo) < TOL
    assert rel_fro(to_host(Bd), oracle.apply_qt(QRo, To, B)) < TOL
    assert L.FLA_Obj_free(C.byref(T)) == flame.FLA_SUCCESS
    assert L.FLA_Obj_free(C.byref(W)) == flame.FLA_SUCCESS
