"""FLASH front-ends on hierarchical (storage-by-blocks) objects, driven the
way the reference's own tests drive them (test/src/test_lu_piv.c:173-226,
test_qrut.c:188-240): hierarchical copies of flat objects
(FLASH_Obj_create_hier_copy_of_flat, FLASH_QR_UT_create_hier_matrices),
the FLASH front-end, FLASH_Obj_flatten back into the flat object.  Results
against the oracle (factors within 1e-12, pivots identical, solutions
within 1e-11), the block layout through FLASH_Copy_hier_to_flat windows,
and the reference's argument rules (depth 1 for LU/QR, b_alg == b_flash)."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_fro, seeded, spd

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _flat(flame, a):
    """An FLA_Obj view over a Fortran-ordered host array (kept alive by the caller)."""
    return flame.View(a)


def _hier(flame, view, b):
    H = flame.FLA_Obj()
    bb = C.c_ulong(b)
    assert flame.lib().FLASH_Obj_create_hier_copy_of_flat(view.obj, 1, C.byref(bb), C.byref(H)) == flame.FLA_SUCCESS
    return H


@pytest.mark.parametrize("n,b", [(1, 1), (100, 32), (257, 64), (384, 128)])
def test_flash_chol_and_solve(cuda, flame, oracle, n, b):
    L = flame.lib()
    rng = seeded(n + b)
    A = np.asfortranarray(spd(rng, n))
    B = np.asfortranarray(rng.standard_normal((n, 3)))
    X = np.asfortranarray(np.zeros((n, 3)))
    vA, vB, vX = _flat(flame, A.copy(order="F")), _flat(flame, B), _flat(flame, X)
    H, HB, HX = _hier(flame, vA, b), _hier(flame, vB, b), _hier(flame, vX, b)
    assert L.FLASH_Obj_depth(H) == 1
    assert (L.FLASH_Obj_scalar_length(H), L.FLASH_Obj_scalar_width(H)) == (n, n)
    bm, bn = C.c_ulong(), C.c_ulong()
    assert L.FLASH_Obj_blocksizes(H, C.byref(bm), C.byref(bn)) == 1 and bm.value == min(b, n)
    assert L.FLASH_Chol(flame.FLA_LOWER_TRIANGULAR, H) == flame.FLA_SUCCESS, flame.last_error()
    assert L.FLASH_Chol_solve(flame.FLA_LOWER_TRIANGULAR, H, HB, HX) == flame.FLA_SUCCESS, flame.last_error()
    assert L.FLASH_Obj_flatten(H, vA.obj) == flame.FLA_SUCCESS
    assert L.FLASH_Obj_flatten(HX, vX.obj) == flame.FLA_SUCCESS
    Lo, ro = oracle.chol(A)
    assert ro == -1
    assert rel_fro(np.tril(vA.buf), np.tril(Lo)) < TOL
    assert np.array_equal(np.triu(vA.buf, 1), np.triu(A, 1))
    assert rel_fro(vX.buf, oracle.chol_solve(Lo, B)) < 1e-11
    for h in (H, HB, HX):
        L.FLASH_Obj_free(C.byref(h))


@pytest.mark.parametrize("m,n,b", [(200, 200, 64), (300, 190, 32), (129, 260, 128)])
def test_flash_lu_piv(cuda, flame, oracle, m, n, b):
    L = flame.lib()
    rng = seeded(m * 3 + n + b)
    A = np.asfortranarray(rng.uniform(-1, 1, (m, n)))
    p = np.zeros(min(m, n), dtype=np.int32)
    vA, vp = _flat(flame, A.copy(order="F")), _flat(flame, p)
    H, Hp = _hier(flame, vA, b), _hier(flame, vp, b)
    assert L.FLASH_LU_piv(H, Hp) == flame.FLA_SUCCESS, flame.last_error()
    assert L.FLASH_Obj_flatten(H, vA.obj) == flame.FLA_SUCCESS
    assert L.FLASH_Obj_flatten(Hp, vp.obj) == flame.FLA_SUCCESS
    LUo, po, ro = oracle.lu_piv(A)
    assert np.array_equal(vp.buf, po)
    assert rel_fro(vA.buf, LUo) < TOL
    if m == n:
        B = np.asfortranarray(rng.standard_normal((n, 2)))
        X = np.asfortranarray(np.zeros((n, 2)))
        vB, vX = _flat(flame, B), _flat(flame, X)
        HB, HX = _hier(flame, vB, b), _hier(flame, vX, b)
        assert L.FLASH_LU_piv_solve(H, Hp, HB, HX) == flame.FLA_SUCCESS, flame.last_error()
        assert L.FLASH_Obj_flatten(HX, vX.obj) == flame.FLA_SUCCESS
        assert rel_fro(vX.buf, oracle.lu_piv_solve(LUo, po, B)) < 1e-11
        for h in (HB, HX):
            L.FLASH_Obj_free(C.byref(h))
    for h in (H, Hp):
        L.FLASH_Obj_free(C.byref(h))


@pytest.mark.parametrize("m,n,b", [(256, 128, 32), (300, 192, 64), (128, 256, 32)])
def test_flash_qr_ut_apply_and_solve(cuda, flame, oracle, m, n, b):
    L = flame.lib()
    rng = seeded(m + 7 * n + b)
    A = np.asfortranarray(rng.standard_normal((m, n)))
    vA = _flat(flame, A.copy(order="F"))
    H, TW = flame.FLA_Obj(), flame.FLA_Obj()
    bb = C.c_ulong(b)
    assert L.FLASH_QR_UT_create_hier_matrices(vA.obj, 1, C.byref(bb), C.byref(H), C.byref(TW)) == flame.FLA_SUCCESS
    k = min(m, n)
    assert (L.FLASH_Obj_scalar_length(TW), L.FLASH_Obj_scalar_width(TW)) == (k, k)
    assert L.FLASH_QR_UT(H, TW) == flame.FLA_SUCCESS, flame.last_error()
    assert L.FLASH_Obj_flatten(H, vA.obj) == flame.FLA_SUCCESS
    QRo, To = oracle.qr_ut(A, b)
    assert rel_fro(vA.buf, QRo) < TOL
    # T block q sits in TW's diagonal block (q, q)
    Tq = np.asfortranarray(np.zeros((b, b)))
    vT = _flat(flame, Tq)
    for q in range(k // b):
        assert L.FLASH_Copy_hier_to_flat(q * b, q * b, TW, vT.obj) == flame.FLA_SUCCESS
        assert rel_fro(np.triu(vT.buf), np.triu(To[:, q * b:(q + 1) * b])) < TOL
    # Q^T B through FLASH_Apply_Q_UT
    Bm = np.asfortranarray(rng.standard_normal((m, 4)))
    vB = _flat(flame, Bm.copy(order="F"))
    HB = _hier(flame, vB, b)
    W = flame.FLA_Obj()
    assert L.FLASH_Apply_Q_UT_create_workspace(TW, HB, C.byref(W)) == flame.FLA_SUCCESS
    assert L.FLASH_Apply_Q_UT(flame.FLA_LEFT, flame.FLA_CONJ_TRANSPOSE, flame.FLA_FORWARD, flame.FLA_COLUMNWISE,
                              H, TW, W, HB) == flame.FLA_SUCCESS, flame.last_error()
    assert L.FLASH_Obj_flatten(HB, vB.obj) == flame.FLA_SUCCESS
    assert rel_fro(vB.buf, oracle.apply_qt(QRo, To, Bm)) < TOL
    if m >= n:
        X = np.asfortranarray(np.zeros((n, 4)))
        vX = _flat(flame, X)
        HB2, HX = _hier(flame, _flat(flame, Bm), b), _hier(flame, vX, b)
        assert L.FLASH_QR_UT_solve(H, TW, HB2, HX) == flame.FLA_SUCCESS, flame.last_error()
        assert L.FLASH_Obj_flatten(HX, vX.obj) == flame.FLA_SUCCESS
        Xref = np.linalg.lstsq(A, Bm, rcond=None)[0]
        assert rel_fro(vX.buf, Xref) < 1e-10
        for h in (HB2, HX):
            L.FLASH_Obj_free(C.byref(h))
    for h in (H, TW, HB, W):
        L.FLASH_Obj_free(C.byref(h))


def test_flash_block_layout_and_windows(cuda, flame):
    """FLASH_Copy_flat_to_hier / hier_to_flat move windows at any scalar
    offset, across block boundaries, and round trip."""
    L = flame.lib()
    rng = seeded(5)
    m, n, b = 70, 45, 16
    A = np.asfortranarray(rng.standard_normal((m, n)))
    vA = _flat(flame, A)
    H = _hier(flame, vA, b)
    win = np.asfortranarray(np.zeros((20, 13)))
    vw = _flat(flame, win)
    assert L.FLASH_Copy_hier_to_flat(11, 7, H, vw.obj) == flame.FLA_SUCCESS
    assert np.array_equal(vw.buf, A[11:31, 7:20])
    new = np.asfortranarray(rng.standard_normal((20, 13)))
    vn = _flat(flame, new)
    assert L.FLASH_Copy_flat_to_hier(vn.obj, 30, 30, H) == flame.FLA_SUCCESS
    out = np.asfortranarray(np.zeros((m, n)))
    vo = _flat(flame, out)
    assert L.FLASH_Obj_flatten(H, vo.obj) == flame.FLA_SUCCESS
    ref = A.copy()
    ref[30:50, 30:43] = new
    assert np.array_equal(vo.buf, ref)
    F = flame.FLA_Obj()
    assert L.FLASH_Obj_create_flat_copy_of_hier(H, C.byref(F)) == flame.FLA_SUCCESS
    assert (F.m, F.n) == (m, n)
    L.FLA_Obj_free(C.byref(F))
    L.FLASH_Obj_free(C.byref(H))
