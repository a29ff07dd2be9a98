"""Generate the golden fixtures in tests/golden/ by running the reference
libflame itself (oracle/_ref/libflame_ref.so, built from the reference
sources by oracle/build_ref.py) on seeded inputs.

    python tests/golden/make_golden.py

The reference has no golden vectors or known-answer files of its own (its
test driver checks residual thresholds on rand() inputs), so these fixtures,
produced by the reference on this machine, pin the CPU restatement oracle
(tests/test_oracle.py checks it bit for bit) and through it the GPU results.
Inputs are stored alongside the outputs so the fixtures are self-contained.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refbind as R  # noqa: E402


def spd(rng, n):
    G = rng.standard_normal((n, n))
    return G @ G.T / n + np.eye(n)


def main():
    out = {}
    rng = np.random.default_rng(20261203)
    # FLA_Chol (lower, and upper)
    for n in [1, 17, 64, 130]:
        A = spd(rng, n)
        L, r = R.chol(A)
        out["chol_l_%d_A" % n] = A
        out["chol_l_%d_L" % n] = L
        out["chol_l_%d_r" % n] = np.array(r)
    for n in [33, 150]:
        A = spd(rng, n)
        U, r = R.chol(A, R.FLA_UPPER_TRIANGULAR)
        out["chol_u_%d_A" % n] = A
        out["chol_u_%d_U" % n] = U
        out["chol_u_%d_r" % n] = np.array(r)
    # non-SPD: the failing column is reported
    A = spd(rng, 60)
    A[37, 37] = -1.0
    L, r = R.chol(A)
    out["chol_fail_A"] = A
    out["chol_fail_r"] = np.array(r)
    # FLA_LU_piv
    for (m, n) in [(1, 1), (33, 17), (17, 33), (130, 130), (160, 120)]:
        A = rng.uniform(-1, 1, (m, n))
        LU, p, r = R.lu_piv(A)
        key = "lu_%dx%d" % (m, n)
        out[key + "_A"] = A
        out[key + "_LU"] = LU
        out[key + "_p"] = p
        out[key + "_r"] = np.array(r)
    # exact ties: small integers, first maximum wins
    A = rng.integers(-2, 3, (50, 50)).astype(np.float64)
    LU, p, r = R.lu_piv(A)
    out["lu_ties_A"], out["lu_ties_LU"], out["lu_ties_p"], out["lu_ties_r"] = A, LU, p, np.array(r)
    # zero column: first null pivot index reported, factorization completes
    A = rng.uniform(-1, 1, (40, 40))
    A[:, 11] = 0.0
    LU, p, r = R.lu_piv(A)
    out["lu_null_A"], out["lu_null_LU"], out["lu_null_p"], out["lu_null_r"] = A, LU, p, np.array(r)
    # FLA_QR_UT + FLA_Apply_Q_UT
    for (m, n) in [(40, 40), (130, 64), (160, 80)]:
        A = rng.standard_normal((m, n))
        QR, T, r = R.qr_ut(A)
        B = rng.standard_normal((m, 3))
        QtB, _ = R.apply_q_ut(QR, T, B)
        key = "qr_%dx%d" % (m, n)
        out[key + "_A"], out[key + "_QR"], out[key + "_T"] = A, QR, T
        out[key + "_B"], out[key + "_QtB"] = B, QtB
    # solves
    n = 100
    A = spd(rng, n)
    B = rng.standard_normal((n, 3))
    L, _ = R.chol(A)
    X, _ = R.chol_solve(L, B)
    out["chol_solve_A"], out["chol_solve_B"], out["chol_solve_X"] = A, B, X
    A = rng.uniform(-1, 1, (n, n))
    LU, p, _ = R.lu_piv(A)
    X, _ = R.lu_piv_solve(LU, p, B)
    out["lu_solve_A"], out["lu_solve_B"], out["lu_solve_X"] = A, B, X
    # LAPACK ABI through lapack2flame
    A = spd(rng, 70)
    a, info = R.dpotrf(A, "U")
    out["dpotrf_A"], out["dpotrf_U"], out["dpotrf_info"] = A, a, np.array(info)
    A = rng.uniform(-1, 1, (70, 70))
    a, ipiv, info = R.dgetrf(A)
    out["dgetrf_A"], out["dgetrf_LU"], out["dgetrf_ipiv"], out["dgetrf_info"] = A, a, ipiv, np.array(info)
    A = rng.standard_normal((80, 60))
    a, tau, info = R.dgeqrf(A)
    out["dgeqrf_A"], out["dgeqrf_QR"], out["dgeqrf_tau"], out["dgeqrf_info"] = A, a, tau, np.array(info)
    A = spd(rng, 60)
    B = rng.standard_normal((60, 2))
    a, x, info = R.dposv(A, B)
    out["dposv_A"], out["dposv_B"], out["dposv_X"], out["dposv_info"] = A, B, x, np.array(info)
    A = rng.uniform(-1, 1, (60, 60))
    a, ipiv, x, info = R.dgesv(A, B)
    out["dgesv_A"], out["dgesv_B"], out["dgesv_X"], out["dgesv_ipiv"] = A, B, x, ipiv
    # the reference's own mixed-precision IR drivers
    A = spd(rng, 100)
    B = rng.standard_normal((100, 2))
    x, it, info = R.dsposv(A, B)
    out["dsposv_A"], out["dsposv_B"], out["dsposv_X"], out["dsposv_iter"] = A, B, x, np.array(it)
    A = rng.uniform(-1, 1, (100, 100))
    x, it, info = R.dsgesv(A, B)
    out["dsgesv_A"], out["dsgesv_B"], out["dsgesv_X"], out["dsgesv_iter"] = A, B, x, np.array(it)
    # the steps after QR: least squares, explicit Q, LAPACK ormqr / orgqr
    for (m, n) in [(90, 40), (170, 130)]:
        A = rng.standard_normal((m, n))
        QR, T, _ = R.qr_ut(A)
        B = rng.standard_normal((m, 3))
        X, _ = R.qr_ut_solve(QR, T, B)
        Q, _ = R.qr_ut_form_q(QR, T, n)
        key = "qrx_%dx%d" % (m, n)
        out[key + "_A"], out[key + "_B"], out[key + "_X"], out[key + "_Q"] = A, B, X, Q
        a, tau, _ = R.dgeqrf(A)
        CL = rng.standard_normal((m, 5))
        CR = rng.standard_normal((4, m))
        out[key + "_CL"], out[key + "_CR"] = CL, CR
        for side, trans, Cm in [("L", "T", CL), ("L", "N", CL), ("R", "N", CR), ("R", "T", CR)]:
            c, info = R.dormqr(side, trans, a, tau, Cm)
            out[key + "_ormqr_%s%s" % (side, trans)] = c
        q, info = R.dorgqr(a, tau, n)
        out[key + "_orgqr"] = q
        Tt, _ = R.accum_t_ut(a, 1.0 / tau, min(32, n))
        out[key + "_accumT"] = Tt
    # inversion: FLA_SPDinv, FLA_Trinv, FLA_Ttmm, dpotri_
    for n in [50, 140]:
        A = spd(rng, n)
        out["spdinv_%d_A" % n] = A
        out["spdinv_%d_L" % n], _ = R.spdinv(A, R.FLA_LOWER_TRIANGULAR)
        out["spdinv_%d_U" % n], _ = R.spdinv(A, R.FLA_UPPER_TRIANGULAR)
        Lf, _ = R.chol(A)
        out["dpotri_%d_L" % n], _ = R.dpotri(Lf, "L")
        M = rng.uniform(-1, 1, (n, n)) + 4 * np.eye(n)
        out["trinv_%d_M" % n] = M
        for uplo, ul in [(R.FLA_LOWER_TRIANGULAR, "l"), (R.FLA_UPPER_TRIANGULAR, "u")]:
            for diag, dg in [(R.FLA_NONUNIT_DIAG, "n"), (R.FLA_UNIT_DIAG, "u")]:
                out["trinv_%d_%s%s" % (n, ul, dg)], _ = R.trinv(M, uplo, diag)
            out["ttmm_%d_%s" % (n, ul)], _ = R.ttmm(M, uplo)
    path = os.path.join(HERE, "reference_small.npz")
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes,", len(out), "arrays")


if __name__ == "__main__":
    main()
