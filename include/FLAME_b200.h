/*
 * FLAME_b200.h -- entry points of libflame_b200 that have no counterpart in
 * the reference libflame: runtime introspection of the GPU library.  The
 * new forms (mixed precision, batched, adjoint) are declared in their own
 * sections below as they are added.  Included by FLAME.h.
 */
#ifndef LIBFLAME_B200_FLAME_B200_H
#define LIBFLAME_B200_FLAME_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Number of CUDA kernels this library has launched since FLA_Init (one
 * replay of a captured graph counts each kernel node it runs). */
unsigned long long FLA_B200_kernel_launches( void );

/* Message of the last CUDA or kernel-timeout error seen by the library
 * ("" if none).  Operations that hit such an error return FLA_FAILURE. */
const char*   FLA_B200_last_error( void );

/* Number of SMs of the device bound at FLA_Init. */
int           FLA_B200_num_sms( void );

/* Device time (CUDA events on the library's stream) of the device work of
 * the last factorization/solve call, in milliseconds. */
double        FLA_B200_last_op_ms( void );

/* Per-kernel-class device timing.  FLA_B200_profile(1) resets the counters
 * and brackets every later launch of the classes below with CUDA events;
 * FLA_B200_profile_read returns the summed duration, the summed
 * algorithmic flops (2mnk for a GEMM, n(n+1)k for the lower update) and
 * the number of launches.  Classes: 0 GEMM engine, 1 panel factorization,
 * 2 triangular solves, 3 row interchanges, 4 diagonal blocks, 5 other. */
void          FLA_B200_profile( int on );
int           FLA_B200_profile_read( int kernel_class, double* ms, double* flops,
                                     unsigned long long* launches );

/* The FP64 GEMM engine on device buffers (column-major):
 * C := alpha op(A) op(B) + beta C; lower_only writes C(i,j), i >= j only. */
int           FLA_B200_dgemm( int transa, int transb, long m, long n, long k, double alpha,
                              const double* A, long lda, const double* B, long ldb,
                              double beta, double* C, long ldc, int lower_only );

/* No counterpart in the reference libflame.  Concurrency self-test of the
 * FP64 GEMM engine: `iters` times, C := C - A B (m x n x k, beta = 1, the
 * factorizations' trailing-update shape) on the library's main stream while
 * its second stream runs Cholesky-panel work (diagonal-block factorization,
 * triangle inverse, panel GEMMs, transpose), as the lookahead of FLA_Chol
 * and FLA_LU_piv does; every result is compared bitwise with the update
 * computed alone and *mismatches receives the number of differing elements
 * summed over all iterations (0 on a correct GPU).  Allocates its operands
 * (about 3 m n doubles) and frees them before returning. */
int           FLA_B200_gemm_concurrency_check( long m, long n, long k, int iters,
                                               unsigned long long* mismatches );

/* No counterpart in the reference libflame.  LU factorization with partial
 * pivoting of one m x n panel (n <= 128, m >= n) held in device memory (A,
 * column-major, lda >= m; piv receives n relative zero-based pivots, as
 * FLA_LU_piv), for callers that cannot let a library allocate device
 * memory: the call makes no cudaMalloc/cudaFree, and keeps its scratch in a
 * fixed ~334 KB array in device memory that the library carries.  Runs on
 * `stream` (a cudaStream_t, or NULL for the default stream) and returns
 * when the panel is done: FLA_SUCCESS, the zero-based index of the first
 * zero pivot, or FLA_FAILURE with the reason in FLA_B200_last_error()
 * (sizes beyond the limits are rejected).  The first call on a device
 * looks up the array's device address, so make it before any stream
 * capture.  All calls on a device share the array: calls that overlap on
 * the GPU race and must be serialized by the caller. */
int           FLA_B200_LU_piv_panel_noalloc( int m, int n, double* A, int lda, int* piv,
                                             void* stream );

/* ---- Mixed precision (no counterpart in the reference beyond dsgesv_ /
 * dsposv_, whose conventions they follow) ----
 * X := A^-1 B for a square FLA_DOUBLE A (device or host buffers): the
 * factorization runs in low precision (FP32 storage, 16-bit tensor-core
 * trailing updates with FP32 accumulation, panels in FP64) and FP64
 * iterative refinement restores FP64 accuracy; A is left unchanged.
 * prec: 0 BF16, 1 FP16 with power-of-two equilibration, 2 3xTF32
 * (FP32-accurate), 3 FP16 hi/lo split (FP32-accurate, on the 16-bit
 * tensor cores), -1 the library default (FLA_B200_IR_PREC, else the FP16
 * hi/lo split).
 * solver: 0 classic refinement (dsgesv_'s), 1 GMRES-IR (GMRES in FP64
 * preconditioned by the low-precision factors, for ill-conditioned A),
 * 2 adaptive (classic refinement while each step cuts the backward error
 * at least fourfold, else the next format of the ladder below), -1 the
 * default (FLA_B200_IR_SOLVER = ir | gmres | auto, else adaptive).
 * A 16-bit format whose refinement stalls escalates to the FP16 hi/lo
 * split; classic and GMRES-IR also to 3xTF32; then the FP64 factorization.
 * iter (optional) receives the
 * number of refinement steps, or -3 (low-precision factorization failed)
 * / -31 (no convergence in 30 steps) when the FP64 factorization of a copy
 * produced X; inner (optional) the GMRES iterations.  Returns FLA_SUCCESS,
 * the zero-based failing column of the FP64 fallback, or FLA_FAILURE. */
FLA_Error     FLA_B200_LU_piv_solve_mixed( FLA_Obj A, FLA_Obj B, FLA_Obj X, int prec, int solver,
                                           int* iter, int* inner );
FLA_Error     FLA_B200_Chol_solve_mixed( FLA_Uplo uplo, FLA_Obj A, FLA_Obj B, FLA_Obj X, int prec,
                                         int solver, int* iter, int* inner );

/* The tensor-core GEMM of the mixed-precision factorizations on device
 * buffers: C (FP32, column-major) := alpha A B^T + beta C, A m x k and B
 * n x k FP32 column-major, rounded to prec (0 BF16, 1 FP16: tcgen05 with an
 * FP32 TMEM accumulator; 2 3xTF32; 3 FP16 hi/lo split, three tcgen05
 * products, FP32-accurate), accumulated in FP32. */
int           FLA_B200_lp_gemm( int prec, long m, long n, long k, float alpha, const float* A, long lda,
                                const float* B, long ldb, float beta, float* C, long ldc );

/* ---- Batched factorizations (no counterpart in the reference) ----
 * `count` independent matrices A[i] (device pointers, column-major, order
 * n[i] <= 512 -- <= 1024 for the FP64 Cholesky, whose updates run on the
 * FP64 tensor cores --, leading dimension lda[i]; the arrays n, A, lda, piv, B, ldb
 * and info are host arrays) in one persistent launch, largest first.  Each
 * matrix gets the single-matrix semantics: info[i] = FLA_SUCCESS, or the
 * zero-based failing column (Cholesky) / first zero-pivot column (LU).
 * nrhs in 0..8: with nrhs > 0 every B[i] (n[i] x nrhs, ldb[i], device) is
 * overwritten in the same launch by the solution of A[i] X = B[i] (skipped
 * for matrices that failed).  LU pivots go to piv[i] (device, n[i] ints,
 * relative as FLA_LU_piv).  Only the lower Cholesky is provided. */
FLA_Error     FLA_Chol_batched( FLA_Uplo uplo, int count, const int* n, double** A, const int* lda,
                                int nrhs, double** B, const int* ldb, int* info );
FLA_Error     FLA_LU_piv_batched( int count, const int* n, double** A, const int* lda, int** piv,
                                  int nrhs, double** B, const int* ldb, int* info );
FLA_Error     FLA_B200_Chol_batched_f32( int count, const int* n, float** A, const int* lda, int nrhs,
                                         float** B, const int* ldb, int* info );
FLA_Error     FLA_B200_LU_piv_batched_f32( int count, const int* n, float** A, const int* lda, int** piv,
                                           int nrhs, float** B, const int* ldb, int* info );
/* FLA_Chol_batched (lower, FP64; orders up to 1024) that also returns
 * logdet[i] = sum_j log L_i(j, j) (host array of count doubles, NaN where
 * the factorization failed): the forward pass of a batch of Gaussian-process
 * likelihoods (with nrhs = 1, B[i] := K_i^-1 y_i). */
FLA_Error     FLA_B200_Chol_batched_logdet( int count, const int* n, double** A, const int* lda, int nrhs,
                                            double** B, const int* ldb, double* logdet, int* info );
/* Autotuner of the batched kernels: per size bin (orders 1-32, 33-64,
 * 65-128, 129-256, 257-512) times the panel widths 8, 16, 24, 32 on
 * `samples` scratch matrices and keeps the fastest for later calls on this
 * device (lu: 0 Cholesky, 1 LU; f64: 0 FP32, 1 FP64).  times (optional, 20
 * doubles) receives the bin x width timings in ms. */
int           FLA_B200_batched_tune( int lu, int f64, int samples, double* times );
/* Panel width the batched kernels use for order n. */
int           FLA_B200_batched_nb( int lu, int f64, int n );

/* ---- Differentiation (no counterpart in the reference) ----
 * Adjoint of the lower Cholesky factorization A = L L^T (blocked reverse
 * mode, in place): L holds the factor from FLA_Chol, Lbar the adjoint of L
 * in its lower triangle; on return the lower triangle of Lbar holds Abar,
 * the adjoint of the lower entries of A (the gradient with respect to a
 * symmetric A is (Abar + Abar^T)/2).  Only FLA_LOWER_TRIANGULAR. */
FLA_Error     FLA_Chol_adjoint( FLA_Uplo uplo, FLA_Obj L, FLA_Obj Lbar );
/* FLA_Chol_adjoint over a batch (device pointers, host arrays n, ld, L,
 * Lbar; L[i] and Lbar[i] share the leading dimension ld[i]): Lbar[i](j,j)
 * += logdet_scale / L[i](j,j) first (0 skips it), then Lbar[i] := Abar[i]
 * in its lower triangle.  The backward pass of a batch of GP likelihoods. */
FLA_Error     FLA_Chol_adjoint_batched( int count, const int* n, double** L, const int* ld, double** Lbar,
                                        double logdet_scale );
/* Lbar += scale * diag(1/L(i,i)): the adjoint of scale * sum_i log L(i,i)
 * (log det A = 2 sum_i log L(i,i)); logdet (optional) receives the sum. */
FLA_Error     FLA_B200_Chol_logdet_adjoint( FLA_Obj L, FLA_Obj Lbar, double scale, double* logdet );
/* Adjoint of X = inv(L) B (left, lower, no transpose, non-unit): on entry X
 * and Xbar; on return Xbar := Bbar = inv(L)^T Xbar and Lbar -= tril(Bbar X^T). */
FLA_Error     FLA_B200_Trsm_llnn_adjoint( FLA_Obj L, FLA_Obj X, FLA_Obj Xbar, FLA_Obj Lbar );

#ifdef __cplusplus
}
#endif

#endif
