"""The CPU restatement oracle (oracle/flame_oracle.c) against the reference
libflame: bit for bit against the committed fixtures that the reference
produced (tests/golden/reference_small.npz), and against the live reference
library when oracle/_ref is built here.  CPU only."""
import numpy as np
import pytest

from conftest import ref_available, seeded, spd


def _t_mask(T, n_cols):
    """Entries of T the reference defines: the upper triangle (with the
    diagonal) of each b x b block; the rest of T is workspace."""
    b = T.shape[0]
    mask = np.zeros(T.shape, dtype=bool)
    for j in range(n_cols):
        mask[: (j % b) + 1, j] = True
    return mask


@pytest.mark.parametrize("n", [1, 17, 64, 130])
def test_chol_lower_matches_reference_bitwise(golden, oracle, n):
    A = golden["chol_l_%d_A" % n]
    L, r = oracle.chol(A)
    assert r == int(golden["chol_l_%d_r" % n]) == -1
    assert np.array_equal(np.tril(L), np.tril(golden["chol_l_%d_L" % n]))
    # strictly upper triangle is left untouched, as in the reference
    assert np.array_equal(np.triu(L, 1), np.triu(A, 1))


def test_chol_failure_index(golden, oracle):
    L, r = oracle.chol(golden["chol_fail_A"])
    assert r == int(golden["chol_fail_r"]) == 37


@pytest.mark.parametrize("shape", ["1x1", "33x17", "17x33", "130x130", "160x120", "ties", "null"])
def test_lu_piv_matches_reference_bitwise(golden, oracle, shape):
    A = golden["lu_%s_A" % shape]
    LU, p, r = oracle.lu_piv(A)
    assert r == int(golden["lu_%s_r" % shape])
    assert np.array_equal(p, golden["lu_%s_p" % shape])
    assert np.array_equal(LU, golden["lu_%s_LU" % shape])


def test_lu_null_pivot_index(golden, oracle):
    assert int(golden["lu_null_r"]) == 11


@pytest.mark.parametrize("shape", ["40x40", "130x64", "160x80"])
def test_qr_ut_and_apply_q_match_reference_bitwise(golden, oracle, shape):
    A = golden["qr_%s_A" % shape]
    QR, T = oracle.qr_ut(A)
    assert np.array_equal(QR, golden["qr_%s_QR" % shape])
    Tg = golden["qr_%s_T" % shape]
    mask = _t_mask(Tg, min(A.shape))
    assert np.array_equal(T[mask], Tg[mask])
    QtB = oracle.apply_qt(golden["qr_%s_QR" % shape], Tg, golden["qr_%s_B" % shape])
    assert np.array_equal(QtB, golden["qr_%s_QtB" % shape])


def test_solves_match_reference_bitwise(golden, oracle):
    L, _ = oracle.chol(golden["chol_solve_A"])
    X = oracle.chol_solve(L, golden["chol_solve_B"])
    assert np.array_equal(X, golden["chol_solve_X"])
    LU, p, _ = oracle.lu_piv(golden["lu_solve_A"])
    X = oracle.lu_piv_solve(LU, p, golden["lu_solve_B"])
    assert np.array_equal(X, golden["lu_solve_X"])


def test_lapack_pivot_shift(golden, oracle):
    A = golden["dgetrf_A"]
    LU, p, _ = oracle.lu_piv(A)
    assert np.array_equal(oracle.shift_pivots(p, True), golden["dgetrf_ipiv"])
    assert np.array_equal(LU, golden["dgetrf_LU"])
    assert np.array_equal(oracle.shift_pivots(golden["dgetrf_ipiv"], False), p)


def test_backward_errors_are_small(golden, oracle):
    A = golden["chol_l_130_A"]
    L, _ = oracle.chol(A)
    assert oracle.chol_backward_error(A, L) < 1.0
    A = golden["lu_130x130_A"]
    LU, p, _ = oracle.lu_piv(A)
    assert oracle.lu_backward_error(A, LU, p) < 1.0
    A = golden["qr_130x64_A"]
    QR, T = oracle.qr_ut(A)
    assert oracle.qr_backward_error(A, QR, T) < 1.0


@pytest.mark.skipif(not ref_available(), reason="reference library not built here")
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_against_live_reference(oracle, seed):
    import refbind as R
    rng = seeded(seed)
    n = int(rng.integers(150, 400))
    A = spd(rng, n)
    assert np.array_equal(np.tril(oracle.chol(A)[0]), np.tril(R.chol(A)[0]))
    m = int(rng.integers(150, 400))
    A = rng.uniform(-1, 1, (m, n))
    l1, p1, r1 = oracle.lu_piv(A)
    l2, p2, r2 = R.lu_piv(A)
    assert np.array_equal(p1, p2) and np.array_equal(l1, l2) and r1 == r2
    A = rng.standard_normal((max(m, n), n))
    q1, t1 = oracle.qr_ut(A)
    q2, t2, _ = R.qr_ut(A)
    assert np.array_equal(q1, q2)


def test_transposed_and_upper_solves_solve_their_systems(oracle):
    """The oracle's dgetrs 'T' and upper FLA_Chol_solve restatements (used as
    the GPU checkers) solve A^T X = B and A X = B on small systems."""
    rng = np.random.default_rng(7)
    n = 40
    A = rng.uniform(-1, 1, (n, n))
    B = rng.standard_normal((n, 3))
    LU, p, r = oracle.lu_piv(A)
    X = oracle.lu_piv_solve_t(LU, p, B)
    assert np.linalg.norm(A.T @ X - B) / np.linalg.norm(B) < 1e-12
    S = A @ A.T + n * np.eye(n)
    Lf, r = oracle.chol(S)
    X = oracle.chol_solve_u(np.triu(Lf.T), B)
    assert np.linalg.norm(S @ X - B) / np.linalg.norm(B) < 1e-12
