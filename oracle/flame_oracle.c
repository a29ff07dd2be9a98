/*
 * flame_oracle.c -- CPU restatement of the reference libflame algorithms on
 * the dense-factorization path (FP64, column-major).
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: tests/,
 * __graft_entry__.smoke() and the CPU-baseline leg of bench.py load it as
 * the checker.  The product library (libflame_b200) never links, loads or
 * calls it.
 *
 * Each routine restates the reference algorithm with the same blocking, the
 * same unblocked leaf and the same loop order as the reference's built-in
 * netlib BLAS (src/flablas/f2c), so that on the same inputs it reproduces
 * the reference library's results; tests/test_oracle.py checks that against
 * the reference itself (oracle/_ref, built by oracle/build_ref.py) and
 * against the committed fixtures in tests/golden/.
 *
 * Conventions (all as in the reference):
 *   - matrices are column-major with leading dimension ld (rs=1, cs=ld);
 *   - LU pivots are relative and zero-based: row i was swapped with row
 *     i + p[i] (docs/libflame/40-user-api.tex:9021-9069);
 *   - return values are FLA_SUCCESS (-1) or a zero-based column index.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_SUCCESS (-1)
#define A_(i, j) a[(size_t)(i) + (size_t)(j) * (size_t)lda]
#define B_(i, j) b[(size_t)(i) + (size_t)(j) * (size_t)ldb]
#define C_(i, j) c[(size_t)(i) + (size_t)(j) * (size_t)ldc]

static int imin(int x, int y) { return x < y ? x : y; }

/* ---------------------------------------------------------------------------
 * netlib BLAS restated (src/flablas/f2c/*.c).  Only the cases the path uses.
 * ------------------------------------------------------------------------- */

/* ddot: src/flablas/f2c/ddot.c.  The unit-stride branch unrolls by 5 but
 * adds left to right, which equals the sequential sum. */
static double o_ddot(int n, const double *x, int incx, const double *y, int incy)
{
    double t = 0.0;
    for (int i = 0; i < n; ++i) t = t + x[(size_t)i * incx] * y[(size_t)i * incy];
    return t;
}

/* dgemv 'N', beta = 1: src/flablas/f2c/dgemv.c (y := alpha*A*x + y). */
static void o_dgemv_n(int m, int n, double alpha, const double *a, int lda,
                      const double *x, int incx, double *y, int incy)
{
    if (m == 0 || n == 0 || alpha == 0.0) return;
    for (int j = 0; j < n; ++j) {
        double xj = x[(size_t)j * incx];
        if (xj != 0.0) {
            double temp = alpha * xj;
            for (int i = 0; i < m; ++i) y[(size_t)i * incy] += temp * A_(i, j);
        }
    }
}

/* dgemv 'T', beta = 1: y := alpha*A^T*x + y. */
static void o_dgemv_t(int m, int n, double alpha, const double *a, int lda,
                      const double *x, int incx, double *y, int incy)
{
    if (m == 0 || n == 0 || alpha == 0.0) return;
    for (int j = 0; j < n; ++j) {
        double temp = 0.0;
        for (int i = 0; i < m; ++i) temp += A_(i, j) * x[(size_t)i * incx];
        y[(size_t)j * incy] += alpha * temp;
    }
}

/* dger: src/flablas/f2c/dger.c (A := alpha*x*y^T + A). */
static void o_dger(int m, int n, double alpha, const double *x, int incx,
                   const double *y, int incy, double *a, int lda)
{
    if (m == 0 || n == 0 || alpha == 0.0) return;
    for (int j = 0; j < n; ++j) {
        double yj = y[(size_t)j * incy];
        if (yj != 0.0) {
            double temp = alpha * yj;
            for (int i = 0; i < m; ++i) A_(i, j) += x[(size_t)i * incx] * temp;
        }
    }
}

static void o_dscal(int n, double alpha, double *x, int incx)
{
    for (int i = 0; i < n; ++i) x[(size_t)i * incx] = alpha * x[(size_t)i * incx];
}

/* bl1_dinvscalv: src/base/flamec/blis/1/bl1_invscalv.c:26-37 -- multiply by
 * the reciprocal, and skip when alpha == 1. */
static void o_invscal(int n, double alpha, double *x, int incx)
{
    if (alpha == 1.0) return;
    o_dscal(n, 1.0 / alpha, x, incx);
}

/* dnrm2: src/flablas/f2c/dnrm2.c (scaled sum of squares, 1993 version). */
static double o_dnrm2(int n, const double *x, int incx)
{
    if (n < 1 || incx < 1) return 0.0;
    if (n == 1) return fabs(x[0]);
    double scale = 0.0, ssq = 1.0;
    for (int i = 0; i < n; ++i) {
        double xi = x[(size_t)i * incx];
        if (xi != 0.0) {
            double absxi = fabs(xi);
            if (scale < absxi) {
                double r = scale / absxi;
                ssq = ssq * (r * r) + 1.0;
                scale = absxi;
            } else {
                double r = absxi / scale;
                ssq += r * r;
            }
        }
    }
    return scale * sqrt(ssq);
}

/* idamax - 1 (bl1_damax, src/base/flamec/blis/1/bl1_amax.c:24-33;
 * src/flablas/f2c/idamax.c:41,60: strict '>' so the first maximum wins). */
static int o_iamax(int n, const double *x, int incx)
{
    if (n < 1) return 0;
    int best = 0;
    double dmax = fabs(x[0]);
    for (int i = 1; i < n; ++i) {
        double v = fabs(x[(size_t)i * incx]);
        if (v > dmax) { best = i; dmax = v; }
    }
    return best;
}

/* dgemm 'N','N', beta = 1: src/flablas/f2c/dgemm.c (C := alpha*A*B + C). */
static void o_dgemm_nn(int m, int n, int k, double alpha, const double *a, int lda,
                       const double *b, int ldb, double *c, int ldc)
{
    if (m == 0 || n == 0 || k == 0 || alpha == 0.0) return;
    for (int j = 0; j < n; ++j)
        for (int l = 0; l < k; ++l)
            if (B_(l, j) != 0.0) {
                double temp = alpha * B_(l, j);
                for (int i = 0; i < m; ++i) C_(i, j) += temp * A_(i, l);
            }
}

/* dgemm 'T','N', beta = 1 (C := alpha*A^T*B + C). */
static void o_dgemm_tn(int m, int n, int k, double alpha, const double *a, int lda,
                       const double *b, int ldb, double *c, int ldc)
{
    if (m == 0 || n == 0 || k == 0 || alpha == 0.0) return;
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double temp = 0.0;
            for (int l = 0; l < k; ++l) temp += A_(l, i) * B_(l, j);
            C_(i, j) = alpha * temp + C_(i, j);
        }
}

/* dsyrk 'L','N', beta = 1: src/flablas/f2c/dsyrk.c (lower C := alpha*A*A^T + C). */
static void o_dsyrk_ln(int n, int k, double alpha, const double *a, int lda,
                       double *c, int ldc)
{
    if (n == 0 || k == 0 || alpha == 0.0) return;
    for (int j = 0; j < n; ++j)
        for (int l = 0; l < k; ++l)
            if (A_(j, l) != 0.0) {
                double temp = alpha * A_(j, l);
                for (int i = j; i < n; ++i) C_(i, j) += temp * A_(i, l);
            }
}

/* dtrsm 'R','L','T','N', alpha = 1 (B := B*inv(A^T)), src/flablas/f2c/dtrsm.c. */
static void o_dtrsm_rltn(int m, int n, const double *a, int lda, double *b, int ldb)
{
    for (int k = 0; k < n; ++k) {
        double temp = 1.0 / A_(k, k);
        for (int i = 0; i < m; ++i) B_(i, k) = temp * B_(i, k);
        for (int j = k + 1; j < n; ++j)
            if (A_(j, k) != 0.0) {
                temp = A_(j, k);
                for (int i = 0; i < m; ++i) B_(i, j) -= temp * B_(i, k);
            }
    }
}

/* dtrsm 'L','L','N', diag (B := inv(A)*B). */
static void o_dtrsm_lln(int m, int n, int unit, const double *a, int lda, double *b, int ldb)
{
    for (int j = 0; j < n; ++j)
        for (int k = 0; k < m; ++k)
            if (B_(k, j) != 0.0) {
                if (!unit) B_(k, j) /= A_(k, k);
                for (int i = k + 1; i < m; ++i) B_(i, j) -= B_(k, j) * A_(i, k);
            }
}

/* dtrsm 'L','L','T', non-unit (B := inv(A^T)*B). */
static void o_dtrsm_llt(int m, int n, const double *a, int lda, double *b, int ldb)
{
    for (int j = 0; j < n; ++j)
        for (int i = m - 1; i >= 0; --i) {
            double temp = B_(i, j);
            for (int k = i + 1; k < m; ++k) temp -= A_(k, i) * B_(k, j);
            temp /= A_(i, i);
            B_(i, j) = temp;
        }
}

/* dtrsm 'L','U','N', non-unit (B := inv(A)*B). */
static void o_dtrsm_lun(int m, int n, const double *a, int lda, double *b, int ldb)
{
    for (int j = 0; j < n; ++j)
        for (int k = m - 1; k >= 0; --k)
            if (B_(k, j) != 0.0) {
                B_(k, j) /= A_(k, k);
                for (int i = 0; i < k; ++i) B_(i, j) -= B_(k, j) * A_(i, k);
            }
}

/* dtrsm 'L','U','T', non-unit (B := inv(A^T)*B). */
static void o_dtrsm_lut(int m, int n, const double *a, int lda, double *b, int ldb)
{
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double temp = B_(i, j);
            for (int k = 0; k < i; ++k) temp -= A_(k, i) * B_(k, j);
            temp /= A_(i, i);
            B_(i, j) = temp;
        }
}

/* dtrmm 'L','L','T','U', alpha = 1 (B := A^T*B, A unit lower). */
static void o_dtrmm_lltu(int m, int n, const double *a, int lda, double *b, int ldb)
{
    for (int j = 0; j < n; ++j)
        for (int i = 0; i < m; ++i) {
            double temp = B_(i, j);
            for (int k = i + 1; k < m; ++k) temp += A_(k, i) * B_(k, j);
            B_(i, j) = temp;
        }
}

/* dtrmm 'L','L','N','U' (B := alpha*A*B, A unit lower). */
static void o_dtrmm_llnu(int m, int n, double alpha, const double *a, int lda, double *b, int ldb)
{
    for (int j = 0; j < n; ++j)
        for (int k = m - 1; k >= 0; --k)
            if (B_(k, j) != 0.0) {
                double temp = alpha * B_(k, j);
                B_(k, j) = temp;
                for (int i = k + 1; i < m; ++i) B_(i, j) += temp * A_(i, k);
            }
}

/* dtrmm 'L','L','T','U' with alpha applied (used by the Q (no-transpose)
 * application). */

/* ---------------------------------------------------------------------------
 * Row pivoting: FLA_Apply_pivots_ln_opd_var1
 * (src/lapack/util/app/piv/ln/flamec/FLA_Apply_pivots_ln_opt_var1.c:274-340),
 * column-major branch: for each column, for i = k1..k2 swap rows i, i+p[i].
 * ------------------------------------------------------------------------- */
void orc_apply_pivots_ln(int ncols, double *a, int lda, int k1, int k2, const int *p)
{
    for (int j = 0; j < ncols; ++j)
        for (int i = k1; i <= k2; ++i) {
            int pi = p[i] + i;
            double t = A_(pi, j);
            A_(pi, j) = A_(i, j);
            A_(i, j) = t;
        }
}

/* Transposed pivots (P^T applied): the same swaps in reverse order
 * (FLA_Apply_pivots with FLA_TRANSPOSE walks i = k2..k1). */
void orc_apply_pivots_lt(int ncols, double *a, int lda, int k1, int k2, const int *p)
{
    for (int j = 0; j < ncols; ++j)
        for (int i = k2; i >= k1; --i) {
            int pi = p[i] + i;
            double t = A_(pi, j);
            A_(pi, j) = A_(i, j);
            A_(i, j) = t;
        }
}

/* ---------------------------------------------------------------------------
 * Cholesky, lower.
 * ------------------------------------------------------------------------- */

/* FLA_Chol_l_opd_var2 (src/lapack/dec/chol/l/flamec/FLA_Chol_l_opt_var2.c:136-193):
 *   alpha11 -= a10t a10t^T;  a21 -= A20 a10t^T;  alpha11 = sqrt(alpha11)
 *   (fails when alpha11 <= 0 or NaN: bl1_dsqrte, blis_macro_defs.h:134-136);
 *   a21 *= 1/alpha11. */
static int chol_l_unb(int n, double *a, int lda)
{
    for (int i = 0; i < n; ++i) {
        double *a10t = &A_(i, 0), *A20 = &A_(i + 1, 0), *alpha11 = &A_(i, i), *a21 = &A_(i + 1, i);
        int ahead = n - i - 1;
        double dot = o_ddot(i, a10t, lda, a10t, lda);
        *alpha11 = 1.0 * *alpha11 + (-1.0) * dot;
        o_dgemv_n(ahead, i, -1.0, A20, lda, a10t, lda, a21, 1);
        if (!(*alpha11 > 0.0)) return i;   /* also catches NaN */
        *alpha11 = sqrt(*alpha11);
        o_invscal(ahead, *alpha11, a21, 1);
    }
    return ORC_SUCCESS;
}

/* FLA_Chol_l_blk_var3 (src/lapack/dec/chol/l/flamec/FLA_Chol_l_blk_var3.c:13-66):
 * chol(A11); A21 := A21 inv(A11^T); A22 -= A21 A21^T.  The control tree is
 * outer b=128 -> inner b=32 -> unblocked var2
 * (src/base/flamec/control/init/lapack/fla/FLA_Chol_cntl_init.c:23-61). */
static int chol_l_blk(int n, double *a, int lda, int nb, int inner)
{
    for (int k = 0; k < n; k += nb) {
        int b = imin(nb, n - k);
        int r = inner > 0 ? chol_l_blk(b, &A_(k, k), lda, inner, 0)
                          : chol_l_unb(b, &A_(k, k), lda);
        if (r != ORC_SUCCESS) return k + r;
        int m2 = n - k - b;
        o_dtrsm_rltn(m2, b, &A_(k, k), lda, &A_(k + b, k), lda);
        o_dsyrk_ln(m2, b, -1.0, &A_(k + b, k), lda, &A_(k + b, k + b), lda);
    }
    return ORC_SUCCESS;
}

int orc_chol_l(int n, double *a, int lda, int nb, int nb_inner)
{
    return chol_l_blk(n, a, lda, nb, nb_inner);
}

/* ---------------------------------------------------------------------------
 * LU with partial pivoting.
 * ------------------------------------------------------------------------- */

/* FLA_LU_piv_opd_var4 (src/lapack/dec/lu/piv/vars/flamec/FLA_LU_piv_opt_var4.c:218-331),
 * Crout form on an m x n panel. */
static int lu_piv_unb(int m, int n, double *a, int lda, int *p)
{
    int r_val = ORC_SUCCESS;
    int mn = imin(m, n);
    for (int i = 0; i < mn; ++i) {
        double *a10t = &A_(i, 0), *A20 = &A_(i + 1, 0), *a01 = &A_(0, i);
        double *alpha11 = &A_(i, i), *a21 = &A_(i + 1, i);
        double *A02 = &A_(0, i + 1), *a12t = &A_(i, i + 1);
        int m_ahead = m - i - 1, n_ahead = n - i - 1;
        double dot = o_ddot(i, a10t, lda, a01, 1);
        *alpha11 = 1.0 * *alpha11 + (-1.0) * dot;
        o_dgemv_n(m_ahead, i, -1.0, A20, lda, a01, 1, a21, 1);
        p[i] = o_iamax(m_ahead + 1, alpha11, 1);
        int null_piv = (alpha11[p[i]] == 0.0);
        if (null_piv) {
            if (r_val == ORC_SUCCESS) r_val = i;
        } else {
            /* swap rows i and i+p[i] in every column of the panel */
            orc_apply_pivots_ln(1, alpha11, lda, 0, 0, &p[i]);
            orc_apply_pivots_ln(i, a10t, lda, 0, 0, &p[i]);
            orc_apply_pivots_ln(n_ahead, a12t, lda, 0, 0, &p[i]);
        }
        o_dgemv_t(i, n_ahead, -1.0, A02, lda, a10t, lda, a12t, lda);
        if (!null_piv) o_invscal(m_ahead, *alpha11, a21, 1);
    }
    return r_val;
}

/* FLA_LU_piv_blk_var5 (src/lapack/dec/lu/piv/vars/flamec/FLA_LU_piv_blk_var5.c:13-114):
 * LU_piv([A11;A21]); pivot [A10;A20] and [A12;A22]; A12 := inv(L11) A12;
 * A22 -= A21 A12.  Control tree: outer b=128 -> inner b=16 -> Crout var4
 * (src/base/flamec/control/init/lapack/fla/FLA_LU_piv_cntl_init.c:24-74). */
static int lu_piv_blk(int m, int n, double *a, int lda, int *p, int nb, int inner)
{
    int r_val = ORC_SUCCESS;
    int mn = imin(m, n);
    for (int k = 0; k < mn; k += nb) {
        int b = imin(nb, mn - k);
        int r = inner > 0 ? lu_piv_blk(m - k, b, &A_(k, k), lda, p + k, inner, 0)
                          : lu_piv_unb(m - k, b, &A_(k, k), lda, p + k);
        if (r_val == ORC_SUCCESS && r >= 0) r_val = k + r;
        orc_apply_pivots_ln(k, &A_(k, 0), lda, 0, b - 1, p + k);
        orc_apply_pivots_ln(n - k - b, &A_(k, k + b), lda, 0, b - 1, p + k);
        o_dtrsm_lln(b, n - k - b, 1, &A_(k, k), lda, &A_(k, k + b), lda);
        o_dgemm_nn(m - k - b, n - k - b, b, -1.0, &A_(k + b, k), lda,
                   &A_(k, k + b), lda, &A_(k + b, k + b), lda);
    }
    return r_val;
}

int orc_lu_piv(int m, int n, double *a, int lda, int *p, int nb, int nb_inner)
{
    return lu_piv_blk(m, n, a, lda, p, nb, nb_inner);
}

/* ---------------------------------------------------------------------------
 * QR via the UT transform.
 * ------------------------------------------------------------------------- */

/* FLA_Househ2_UT_l_opd (src/base/flamec/util/lapack/FLA_Househ2_UT.c:274-386). */
static void househ2_ut_l(int m_x2, double *chi_1, double *x2, int inc, double *tau)
{
    double norm_x_2 = o_dnrm2(m_x2, x2, inc);
    if (norm_x_2 == 0.0) {
        *chi_1 = -(*chi_1);
        *tau = 0.5;
        return;
    }
    double abs_chi_1 = o_dnrm2(1, chi_1, 1);
    double y[2] = {abs_chi_1, norm_x_2};
    double norm_x = o_dnrm2(2, y, 1);
    double sgn = (*chi_1 < 0.0) ? -1.0 : 1.0;
    double alpha = -sgn * norm_x;
    double chi_1_minus_alpha = *chi_1 - alpha;
    o_invscal(m_x2, chi_1_minus_alpha, x2, inc);
    double abs_cma = fabs(chi_1_minus_alpha);
    double q = norm_x_2 / abs_cma;
    *tau = 0.5 + 0.5 * (q * q);
    *chi_1 = alpha;
}

/* FLA_Apply_H2_UT_l_opd_var1 (src/lapack/util/app/h2ut/l/flamec/FLA_Apply_H2_UT_l_opt_var1.c):
 * w1t = (a1t + u2^T A2)/tau; a1t -= w1t; A2 -= u2 w1t. */
static void apply_h2_ut_l(int m, int n, double tau, const double *u2, double *a1t, int inc_a1t,
                          double *A2, int lda)
{
    if (n == 0 && tau == 0.0) return;
    double *w = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    for (int j = 0; j < n; ++j) w[j] = a1t[(size_t)j * inc_a1t];
    o_dgemv_t(m, n, 1.0, A2, lda, u2, 1, w, 1);
    o_invscal(n, tau, w, 1);
    for (int j = 0; j < n; ++j) a1t[(size_t)j * inc_a1t] += -1.0 * w[j];
    o_dger(m, n, -1.0, u2, 1, w, 1, A2, lda);
    free(w);
}

/* FLA_QR_UT_opd_var2 (src/lapack/dec/q/qrut/vars/flamec/FLA_QR_UT_opt_var2.c:161-226):
 * per column Householder, apply to the rest of the panel, then
 * t01 = a10t^T + A20^T u21 and tau11 on T's diagonal. */
static void qr_ut_unb(int m, int n, double *a, int lda, double *t, int ldt)
{
    int mn = imin(m, n);
    for (int i = 0; i < mn; ++i) {
        double *alpha11 = &a[i + (size_t)i * lda], *a21 = alpha11 + 1;
        double *a12t = &a[i + (size_t)(i + 1) * lda], *A22 = &a[i + 1 + (size_t)(i + 1) * lda];
        double *a10t = &a[i], *A20 = &a[i + 1];
        double *tau11 = &t[i + (size_t)i * ldt], *t01 = &t[(size_t)i * ldt];
        int m_ahead = m - i - 1, n_ahead = n - i - 1;
        househ2_ut_l(m_ahead, alpha11, a21, 1, tau11);
        apply_h2_ut_l(m_ahead, n_ahead, *tau11, a21, a12t, lda, A22, lda);
        for (int j = 0; j < i; ++j) t01[j] = a10t[(size_t)j * lda];
        o_dgemv_t(m_ahead, i, 1.0, A20, lda, a21, 1, t01, 1);
    }
}

/* One step of FLA_Apply_Q_UT_lhfc_blk_var1
 * (src/lapack/util/app/qut/lhfc/flamec/FLA_Apply_Q_UT_lhfc_blk_var1.c:148-182)
 * for a block of b reflectors stored in the m x b panel U (unit lower part)
 * with triangular factor T1 (b x b, upper), applied from the left as Q^T to
 * the m x nb block B.  W is b x nb scratch. */
static void apply_qt_block(int m, int b, const double *u, int ldu, const double *t1, int ldt,
                           int nb, double *bm, int ldb, double *w)
{
    int ldw = b;
    /* W = B1 */
    for (int j = 0; j < nb; ++j)
        for (int i = 0; i < b; ++i) w[i + (size_t)j * ldw] = bm[i + (size_t)j * ldb];
    /* W = U11^T W (unit lower) */
    o_dtrmm_lltu(b, nb, u, ldu, w, ldw);
    /* W += U21^T B2 */
    o_dgemm_tn(b, nb, m - b, 1.0, u + b, ldu, bm + b, ldb, w, ldw);
    /* W = inv(T1^T) W (T1 upper, non-unit) */
    o_dtrsm_lut(b, nb, t1, ldt, w, ldw);
    /* B2 -= U21 W */
    o_dgemm_nn(m - b, nb, b, -1.0, u + b, ldu, w, ldw, bm + b, ldb);
    /* W = -U11 W (unit lower) */
    o_dtrmm_llnu(b, nb, -1.0, u, ldu, w, ldw);
    /* B1 += W */
    for (int j = 0; j < nb; ++j)
        for (int i = 0; i < b; ++i) bm[i + (size_t)j * ldb] += 1.0 * w[i + (size_t)j * ldw];
}

/* FLA_QR_UT_blk_var1 (src/lapack/dec/q/qrut/vars/flamec/FLA_QR_UT_blk_var1.c:13-102):
 * blocks of b_alg = length(T) columns; panel QR into T1; apply Q1^T to the
 * trailing columns.  T is b_alg x n with ld ldt. */
void orc_qr_ut(int m, int n, double *a, int lda, double *t, int ldt, int b_alg)
{
    int mn = imin(m, n);
    double *w = (double *)malloc(sizeof(double) * (size_t)b_alg * (n > 0 ? n : 1));
    for (int k = 0; k < mn; k += b_alg) {
        int b = imin(b_alg, mn - k);
        double *t1 = &t[(size_t)k * ldt];
        qr_ut_unb(m - k, b, &A_(k, k), lda, t1, ldt);
        int n2 = n - k - b;
        if (n2 > 0) {
            /* apply_qt_block keeps W with leading dimension b */
            apply_qt_block(m - k, b, &A_(k, k), lda, t1, ldt, n2, &A_(k, k + b), lda, w);
        }
    }
    free(w);
}

/* FLA_Apply_Q_UT(LEFT, CONJ_TRANSPOSE, FORWARD, COLUMNWISE) via lhfc var1:
 * B := Q^T B with Q = H(0) H(1) ... from the m x k matrix U (from QR_UT)
 * and T (b_alg x k). */
void orc_apply_qt(int m, int k, const double *a, int lda, const double *t, int ldt, int b_alg,
                  int nrhs, double *b, int ldb)
{
    int kk = imin(m, k);
    double *w = (double *)malloc(sizeof(double) * (size_t)b_alg * (nrhs > 0 ? nrhs : 1));
    for (int j = 0; j < kk; j += b_alg) {
        int bs = imin(b_alg, kk - j);
        apply_qt_block(m - j, bs, &A_(j, j), lda, &t[(size_t)j * ldt], ldt, nrhs, &B_(j, 0), ldb, w);
    }
    free(w);
}

/* ---------------------------------------------------------------------------
 * Solves.
 * ------------------------------------------------------------------------- */

/* FLA_Chol_solve, lower (src/lapack/dec/chol/front/flamec/FLA_Chol_solve.c:13-35):
 * X := inv(L) B; X := inv(L^T) X.  B is overwritten with X. */
void orc_chol_solve_l(int n, int nrhs, const double *a, int lda, double *b, int ldb)
{
    o_dtrsm_lln(n, nrhs, 0, a, lda, b, ldb);
    o_dtrsm_llt(n, nrhs, a, lda, b, ldb);
}

/* FLA_LU_piv_solve (src/lapack/dec/lu/piv/front/flamec/FLA_LU_piv_solve.c:13-29):
 * X := P B; X := inv(L) X (unit); X := inv(U) X. */
void orc_lu_piv_solve(int n, int nrhs, const double *a, int lda, const int *p, double *b, int ldb)
{
    orc_apply_pivots_ln(nrhs, b, ldb, 0, n - 1, p);
    o_dtrsm_lln(n, nrhs, 1, a, lda, b, ldb);
    o_dtrsm_lun(n, nrhs, a, lda, b, ldb);
}

/* Plain triangular solves exposed for the adjoint/gradient references. */
void orc_trsm_lln(int m, int n, int unit, const double *a, int lda, double *b, int ldb)
{
    o_dtrsm_lln(m, n, unit, a, lda, b, ldb);
}

void orc_trsm_llt(int m, int n, const double *a, int lda, double *b, int ldb)
{
    o_dtrsm_llt(m, n, a, lda, b, ldb);
}

/* FLA_Shift_pivots_to (src/base/flamec/util/lapack/FLA_Shift_pivots_to.c:13-42):
 * to LAPACK: p[i] += i + 1; to native: p[i] -= i + 1. */
void orc_shift_pivots(int n, int *p, int to_lapack)
{
    for (int i = 0; i < n; ++i) p[i] += to_lapack ? (i + 1) : -(i + 1);
}
