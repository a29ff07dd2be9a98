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

#ifdef __cplusplus
}
#endif

#endif
