// Low-precision kernels of the mixed-precision solvers (lp_gemm.cu).
#pragma once
#include <cstdint>

#include "common.h"

namespace fb {

enum LowPrec : int { LP_BF16 = 0, LP_FP16 = 1 };

// C (FP32, column-major) := alpha * A * B^T + beta * C; A m x k and B n x k
// packed 16-bit, k contiguous (row r at A + r * lda; lda, ldb multiples of 8,
// 16-byte aligned bases).  GEMM_LOWER: only i - j >= diag_off is written.
int lp_gemm(cudaStream_t st, LowPrec prec, long m, long n, long k, float alpha, const uint16_t* A, long lda,
            const uint16_t* B, long ldb, float beta, float* C, long ldc, GemmMode mode = GEMM_FULL,
            long diag_off = 0, const int* guard = nullptr, int guard_limit = 0x7fffffff);
// dst[r * ldd + kk] := 16-bit(scale * src(r, kk)), src(r, kk) at
// src[r * rs + kk * cs]; columns kdim .. round8(kdim) of dst are zeroed.
template <typename TS>
int pack16(cudaStream_t st, LowPrec prec, const TS* src, long rs, long cs, uint16_t* dst, long ldd, long rows,
           long kdim, float scale);
// dst (m x n, ld ldd) := src (m x n, ld lds), converted.
template <typename TD, typename TS>
int convert2d(cudaStream_t st, const TS* src, long lds, TD* dst, long ldd, long m, long n);
// FP32 C := alpha op(A) op(B) + beta C (SIMT).
int sgemm(cudaStream_t st, bool ta, bool tb, long m, long n, long k, float alpha, const float* A, long lda,
          const float* B, long ldb, float beta, float* C, long ldc);

}  // namespace fb
