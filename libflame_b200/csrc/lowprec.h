// Low-precision kernels of the mixed-precision solvers (lp_gemm.cu).
#pragma once
#include <cstdint>

#include "common.h"

namespace fb {

// LP_FP16X3: FP32-accurate products on the 16-bit tensor cores, each operand
// split into FP16 planes hi = fp16(x), lo = fp16((x - hi) * 2^11).
enum LowPrec : int { LP_BF16 = 0, LP_FP16 = 1, LP_TF32X3 = 2, LP_FP16X3 = 3 };

// Packed operands: 16-bit formats hold rows * ld uint16 values; LP_TF32X3
// holds two FP32 planes (hi, then lo), the lo plane a caller-chosen number
// of floats (the "plane") after the hi plane; ld is counted in the
// operand's own element type (a multiple of 8).
inline size_t lp_packed_bytes(LowPrec p, long rows, long ld) {
  const size_t e = (size_t)(rows > 0 ? rows : 1) * (size_t)ld;
  return (p == LP_TF32X3 ? 2 * e * sizeof(float) : (p == LP_FP16X3 ? 2 : 1) * e * sizeof(uint16_t)) + 256;
}

// C (FP32, column-major) := alpha * A * B^T + beta * C; A m x k and B n x k
// packed 16-bit, k contiguous (row r at A + r * lda; lda, ldb multiples of 8,
// 16-byte aligned bases).  GEMM_LOWER: only i - j >= diag_off is written.
// LP_TF32X3: A, B are the hi planes (float, ld in floats) and the lo planes
// follow at aplane / bplane floats; LP_FP16X3 likewise with FP16 planes
// (aplane / bplane in 16-bit elements).
int lp_gemm(cudaStream_t st, LowPrec prec, long m, long n, long k, float alpha, const uint16_t* A, long lda,
            const uint16_t* B, long ldb, float beta, float* C, long ldc, GemmMode mode = GEMM_FULL,
            long diag_off = 0, const int* guard = nullptr, int guard_limit = 0x7fffffff, long aplane = 0,
            long bplane = 0);
// The 16-bit case on the tcgen05 tensor cores (tc_gemm.cu): TMA-fed
// K-major operands, FP32 accumulator in TMEM.
int tc_gemm16(cudaStream_t st, bool bf16, bool split, long m, long n, long k, float alpha, const uint16_t* A,
              long lda, const uint16_t* B, long ldb, float beta, float* C, long ldc, GemmMode mode, long diag_off,
              const int* guard, int guard_limit, long aplane, long bplane);
// Element offset into a packed operand buffer (16-bit elements, or floats
// for LP_TF32X3).
inline uint16_t* lp_off(uint16_t* base, LowPrec p, size_t elems) {
  return base + elems * (p == LP_TF32X3 ? 2 : 1);
}
// dst[r * ldd + kk] := 16-bit(scale * src(r, kk)), src(r, kk) at
// src[r * rs + kk * cs]; columns kdim .. round8(kdim) of dst are zeroed.
template <typename TS>
int pack16(cudaStream_t st, LowPrec prec, const TS* src, long rs, long cs, uint16_t* dst, long ldd, long rows,
           long kdim, float scale, long plane = 0);
// dst (m x n, ld ldd) := src (m x n, ld lds), converted.
template <typename TD, typename TS>
int convert2d(cudaStream_t st, const TS* src, long lds, TD* dst, long ldd, long m, long n);
// FP32 C := alpha op(A) op(B) + beta C (SIMT).
int sgemm(cudaStream_t st, bool ta, bool tb, long m, long n, long k, float alpha, const float* A, long lda,
          const float* B, long ldb, float beta, float* C, long ldc);

}  // namespace fb
