/*
 * A plain C caller of libflame_b200 written against include/FLAME.h only,
 * the way a program written for the reference libflame calls it: FLA_Obj
 * views over host arrays (the library stages them through HBM), T and W
 * objects from FLA_QR_UT_create_T / FLA_Apply_Q_UT_create_workspace.  Each
 * result is checked here on the CPU:
 *   FLA_Chol (lower):    ||A - L L^T||_F / ||A||_F
 *   FLA_LU_piv:          ||P A - L U||_F / ||A||_F, pivots in range
 *   FLA_LU_piv_solve:    ||A X - B||_F / (||A||_F ||X||_F)
 *   FLA_QR_UT + FLA_Apply_Q_UT: Q^T A against the computed R (zero below)
 * Prints one line per check and exits 0 when every check passes.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "FLAME.h"

static unsigned long long rng_state = 88172645463325252ull;
static double urand(void) { /* xorshift64, uniform in [-1, 1) */
  rng_state ^= rng_state << 13;
  rng_state ^= rng_state >> 7;
  rng_state ^= rng_state << 17;
  return (double)(rng_state >> 11) / 9007199254740992.0 * 2.0 - 1.0;
}

static double fro(const double* a, long n) {
  double s = 0.0;
  for (long i = 0; i < n; ++i) s += a[i] * a[i];
  return sqrt(s);
}

static int view(double* buf, dim_t m, dim_t n, FLA_Obj* obj) {
  if (FLA_Obj_create_without_buffer(FLA_DOUBLE, m, n, obj) != FLA_SUCCESS) return 1;
  return FLA_Obj_attach_buffer(buf, 1, m, obj) != FLA_SUCCESS;
}

static int report(const char* what, double v, double tol) {
  const int ok = v < tol;
  printf("%-28s %.3e (< %.0e) %s\n", what, v, tol, ok ? "ok" : "FAILED");
  return ok ? 0 : 1;
}

int main(void) {
  const long n = 256, m = 384, nq = 200, nrhs = 3;
  int fails = 0;
  FLA_Init();

  /* ---- FLA_Chol on an SPD matrix A = G G^T + n I */
  {
    double* G = malloc(sizeof(double) * n * n);
    double* A = malloc(sizeof(double) * n * n);
    double* L = malloc(sizeof(double) * n * n);
    for (long i = 0; i < n * n; ++i) G[i] = urand();
    for (long j = 0; j < n; ++j)
      for (long i = 0; i < n; ++i) {
        double s = (i == j) ? (double)n : 0.0;
        for (long k = 0; k < n; ++k) s += G[i + k * n] * G[j + k * n];
        A[i + j * n] = s;
      }
    memcpy(L, A, sizeof(double) * n * n);
    FLA_Obj Lo;
    fails += view(L, n, n, &Lo);
    const FLA_Error r = FLA_Chol(FLA_LOWER_TRIANGULAR, Lo);
    if (r != FLA_SUCCESS) { printf("FLA_Chol returned %d\n", r); ++fails; }
    double* R = malloc(sizeof(double) * n * n);
    for (long j = 0; j < n; ++j)
      for (long i = 0; i < n; ++i) {
        double s = 0.0;
        for (long k = 0; k <= (i < j ? i : j); ++k) s += L[i + k * n] * L[j + k * n];
        R[i + j * n] = A[i + j * n] - s;
      }
    fails += report("FLA_Chol residual", fro(R, n * n) / fro(A, n * n), 1e-14);
    FLA_Obj_free_without_buffer(&Lo);
    free(G); free(A); free(L); free(R);
  }

  /* ---- FLA_LU_piv and FLA_LU_piv_solve */
  {
    double* A = malloc(sizeof(double) * n * n);
    double* F = malloc(sizeof(double) * n * n);
    double* B = malloc(sizeof(double) * n * nrhs);
    double* X = malloc(sizeof(double) * n * nrhs);
    int* p = malloc(sizeof(int) * n);
    for (long i = 0; i < n * n; ++i) A[i] = urand();
    for (long i = 0; i < n * nrhs; ++i) B[i] = urand();
    memcpy(F, A, sizeof(double) * n * n);
    FLA_Obj Fo, po, Bo, Xo;
    fails += view(F, n, n, &Fo);
    fails += FLA_Obj_create_without_buffer(FLA_INT, n, 1, &po) != FLA_SUCCESS;
    fails += FLA_Obj_attach_buffer(p, 1, n, &po) != FLA_SUCCESS;
    fails += view(B, n, nrhs, &Bo);
    fails += view(X, n, nrhs, &Xo);
    const FLA_Error r = FLA_LU_piv(Fo, po);
    if (r != FLA_SUCCESS) { printf("FLA_LU_piv returned %d\n", r); ++fails; }
    int bad = 0;
    for (long i = 0; i < n; ++i) bad += (p[i] < 0 || i + p[i] >= n);
    if (bad) { printf("FLA_LU_piv: %d pivots out of range\n", bad); ++fails; }
    /* P A: apply the relative pivots in order to a copy of A */
    double* PA = malloc(sizeof(double) * n * n);
    memcpy(PA, A, sizeof(double) * n * n);
    for (long i = 0; i < n; ++i) {
      const long k = i + p[i];
      if (k != i)
        for (long j = 0; j < n; ++j) {
          const double t = PA[i + j * n];
          PA[i + j * n] = PA[k + j * n];
          PA[k + j * n] = t;
        }
    }
    for (long j = 0; j < n; ++j)
      for (long i = 0; i < n; ++i) {
        double s = 0.0;
        const long kk = i < j ? i : j;
        for (long k = 0; k <= kk; ++k) s += (k == i ? 1.0 : F[i + k * n]) * F[k + j * n];
        PA[i + j * n] -= s;
      }
    fails += report("FLA_LU_piv residual", fro(PA, n * n) / fro(A, n * n), 1e-13);
    const FLA_Error rs = FLA_LU_piv_solve(Fo, po, Bo, Xo);
    if (rs != FLA_SUCCESS) { printf("FLA_LU_piv_solve returned %d\n", rs); ++fails; }
    double* Rs = malloc(sizeof(double) * n * nrhs);
    for (long c = 0; c < nrhs; ++c)
      for (long i = 0; i < n; ++i) {
        double s = -B[i + c * n];
        for (long k = 0; k < n; ++k) s += A[i + k * n] * X[k + c * n];
        Rs[i + c * n] = s;
      }
    fails += report("FLA_LU_piv_solve residual", fro(Rs, n * nrhs) / (fro(A, n * n) * fro(X, n * nrhs)), 1e-14);
    FLA_Obj_free_without_buffer(&Fo);
    FLA_Obj_free_without_buffer(&po);
    FLA_Obj_free_without_buffer(&Bo);
    FLA_Obj_free_without_buffer(&Xo);
    free(A); free(F); free(B); free(X); free(p); free(PA); free(Rs);
  }

  /* ---- FLA_QR_UT with T from FLA_QR_UT_create_T, then Q^T A through
   * FLA_Apply_Q_UT with W from FLA_Apply_Q_UT_create_workspace */
  {
    double* A = malloc(sizeof(double) * m * nq);
    double* F = malloc(sizeof(double) * m * nq);
    double* Q = malloc(sizeof(double) * m * nq);
    for (long i = 0; i < m * nq; ++i) A[i] = urand();
    memcpy(F, A, sizeof(double) * m * nq);
    memcpy(Q, A, sizeof(double) * m * nq);
    FLA_Obj Fo, Qo, T, W;
    fails += view(F, m, nq, &Fo);
    fails += view(Q, m, nq, &Qo);
    fails += FLA_QR_UT_create_T(Fo, &T) != FLA_SUCCESS;
    printf("FLA_QR_UT_create_T: %lu x %lu\n", (unsigned long)FLA_Obj_length(T), (unsigned long)FLA_Obj_width(T));
    if (FLA_Obj_width(T) != (dim_t)nq || FLA_Obj_length(T) < 1) ++fails;
    const FLA_Error r = FLA_QR_UT(Fo, T);
    if (r != FLA_SUCCESS) { printf("FLA_QR_UT returned %d\n", r); ++fails; }
    fails += FLA_Apply_Q_UT_create_workspace(T, Qo, &W) != FLA_SUCCESS;
    const FLA_Error ra = FLA_Apply_Q_UT(FLA_LEFT, FLA_CONJ_TRANSPOSE, FLA_FORWARD, FLA_COLUMNWISE, Fo, T, W, Qo);
    if (ra != FLA_SUCCESS) { printf("FLA_Apply_Q_UT returned %d\n", ra); ++fails; }
    /* Q^T A must equal R (upper triangle of the factor) and zero below */
    for (long j = 0; j < nq; ++j)
      for (long i = 0; i < m; ++i) Q[i + j * m] -= (i <= j) ? F[i + j * m] : 0.0;
    fails += report("FLA_QR_UT / Apply_Q_UT", fro(Q, m * nq) / fro(A, m * nq), 1e-13);
    FLA_Obj_free(&T);
    FLA_Obj_free(&W);
    FLA_Obj_free_without_buffer(&Fo);
    FLA_Obj_free_without_buffer(&Qo);
    free(A); free(F); free(Q);
  }

  FLA_Finalize();
  printf("%s\n", fails ? "FAILED" : "all checks passed");
  return fails ? 1 : 0;
}
