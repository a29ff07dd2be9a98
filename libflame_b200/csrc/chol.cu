// FP64 Cholesky factorization (FLA_Chol) on the GPU.
//
// Right-looking blocked algorithm with the reference's structure
// (src/lapack/dec/chol/l/flamec/FLA_Chol_l_blk_var3.c:13-66):
//   for each 128-column block:  A11 := chol(A11)        [potrf_diag_kernel]
//                               A21 := A21 inv(A11)^T   [DMMA GEMM with inv(L11)]
//                               A22 -= A21 A21^T (lower) [DMMA GEMM engine]
// with the next block column factored on a second stream while the rest of
// the trailing update runs (chol_lower_enqueue).
// The diagonal block is factored in shared memory in 32-column steps (the
// reference's inner blocksize, FLA_Chol_cntl_init.c:23-61): a warp factors
// each 32x32 block (the unblocked var2/var3 leaf), the rows below are solved
// against it and the trailing part of the block is updated, all in SMEM.
// A failing pivot (<= 0 or NaN, bl1_dsqrte in
// src/base/flamec/blis/include/blis_macro_defs.h:134-136) records the
// zero-based global column in the status block; every later kernel of the
// factorization sees it and returns without touching memory.
#include <climits>

#include "common.h"
#include "dev_util.cuh"

namespace fb {

namespace {

constexpr int NB = 128;        // outer block
constexpr int IB = 32;         // inner block
constexpr int LDS = NB + 1;    // SMEM leading dimension (odd: spreads banks)
constexpr int POTRF_THREADS = 256;
constexpr int POTRF_SMEM = NB * LDS * 8;

__device__ __forceinline__ bool guard_failed(const int* info) {
  return *((volatile const int*)info) != INT_MAX;
}

// Factor the b x b (b <= 128) lower-triangular diagonal block at A (ld) in
// place.  gcol = global index of its first column (for the info word).
__global__ void __launch_bounds__(POTRF_THREADS) potrf_diag_kernel(double* A, long ld, int b, int gcol,
                                                                   int* info) {
  extern __shared__ double S[];  // S[r + c*LDS]
  __shared__ int s_fail;
  if (guard_failed(info)) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // load lower triangle (and diagonal); upper part of S is never read
  for (int c = warp; c < b; c += POTRF_THREADS / 32)
    for (int r = c + lane; r < b; r += 32) S[r + c * LDS] = A[r + (long)c * ld];
  if (tid == 0) s_fail = -1;
  __syncthreads();

  for (int jb = 0; jb < b; jb += IB) {
    const int w = min(IB, b - jb);
    // (a) warp 0: unblocked Cholesky of the w x w diagonal block
    if (warp == 0) {
      for (int j = 0; j < w; ++j) {
        double d = 0.0;
        int bad = 0;
        if (lane == j) {
          d = S[(jb + j) + (jb + j) * LDS];
          if (!(d > 0.0)) bad = 1;  // <= 0 or NaN
          else d = sqrt(d);
        }
        d = __shfl_sync(0xffffffffu, d, j);
        bad = __shfl_sync(0xffffffffu, bad, j);
        if (bad) {
          if (lane == 0) s_fail = jb + j;
          break;
        }
        if (lane == j) S[(jb + j) + (jb + j) * LDS] = d;
        const double rinv = 1.0 / d;
        if (lane > j && lane < w) S[(jb + lane) + (jb + j) * LDS] *= rinv;
        __syncwarp();
        if (lane > j && lane < w) {
          const double lij = S[(jb + lane) + (jb + j) * LDS];
          for (int c = j + 1; c <= lane; ++c)
            S[(jb + lane) + (jb + c) * LDS] -= lij * S[(jb + c) + (jb + j) * LDS];
        }
        __syncwarp();
      }
    }
    __syncthreads();
    if (s_fail >= 0) break;
    const int r0 = jb + w;  // first row below the diagonal block
    // (b) rows below: X := X inv(D)^T, one thread per row (right-looking,
    //     multiply by the reciprocal of the pivot like dtrsm R,L,T,N)
    for (int r = r0 + tid; r < b; r += POTRF_THREADS) {
      for (int j = 0; j < w; ++j) {
        const double x = S[r + (jb + j) * LDS] * (1.0 / S[(jb + j) + (jb + j) * LDS]);
        S[r + (jb + j) * LDS] = x;
        for (int c = j + 1; c < w; ++c) S[r + (jb + c) * LDS] -= x * S[(jb + c) + (jb + j) * LDS];
      }
    }
    __syncthreads();
    // (c) trailing lower triangle of the block: S22 -= X X^T
    const int m2 = b - r0;
    const int nel = m2 * (m2 + 1) / 2;
    for (int e = tid; e < nel; e += POTRF_THREADS) {
      // map e -> (i, c) with c <= i, column-major over the lower triangle
      int c = (int)((2.0 * m2 + 1.0 - sqrt((2.0 * m2 + 1.0) * (2.0 * m2 + 1.0) - 8.0 * e)) * 0.5);
      int start = c * m2 - c * (c - 1) / 2;
      while (start > e) { --c; start = c * m2 - c * (c - 1) / 2; }
      while (start + (m2 - c) <= e) { start += m2 - c; ++c; }
      const int i = c + (e - start);
      double s = 0.0;
      for (int j = 0; j < w; ++j) s += S[(r0 + i) + (jb + j) * LDS] * S[(r0 + c) + (jb + j) * LDS];
      S[(r0 + i) + (r0 + c) * LDS] -= s;
    }
    __syncthreads();
  }
  // write back the lower triangle (the strictly upper part of A is untouched)
  for (int c = warp; c < b; c += POTRF_THREADS / 32)
    for (int r = c + lane; r < b; r += 32) A[r + (long)c * ld] = S[r + c * LDS];
  if (tid == 0 && s_fail >= 0) atomicMin(info, gcol + s_fail);
}

bool g_attr_done = false;
void set_attrs() {
  if (g_attr_done) return;
  cudaFuncSetAttribute(potrf_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, POTRF_SMEM);
  g_attr_done = true;
}

}  // namespace

// Enqueue the blocked factorization of the lower triangle of A on `st`, with
// a lookahead of one panel when `st` is the library's main stream:
//   panel k (side stream):  A11 := chol(A11); inv(L11) formed next to it;
//                           A21 := A21 inv(L11)^T as a DMMA GEMM
//   main stream, step k:    A22(:, next panel) -= A21 A21(next rows)^T,
//                           then the next panel goes to the side stream,
//                           A22(rest) -= A21 A21^T (lower) concurrently.
// Failure semantics follow FLA_Chol_l_blk_var3: the updates of step k run
// unless a column before k + b has failed (the guard limit of each launch),
// so a failure in the next panel does not cut short step k's update.
int chol_lower_enqueue(DMat A, cudaStream_t st) {
  set_attrs();
  Context& cx = ctx();
  const long n = A.m, ld = A.ld;
  if (n <= 0) return FLA_SUCCESS;
  int* info = cx.d_status + ST_INFO;
  const bool lookahead = (st == cx.stream);
  cudaStream_t sd = lookahead ? cx.side : st;
  double* Linv = (double*)ws_get(WS_MISC, sizeof(double) * NB * NB);
  double* W = (double*)ws_get(WS_MISC2, sizeof(double) * NB * (size_t)(std::max<long>(0, n - NB) + 2));
  if (!Linv || !W) return FLA_FAILURE;
  cudaEvent_t ev_look = cx.ev[2], ev_panel = cx.ev[3];
  auto at = [&](long i, long j) { return A.p + i + j * ld; };

  // Panel k: diagonal block, its inverse, and the block column below it.
  auto panel = [&](long k, cudaStream_t s) -> int {
    const int b = (int)std::min<long>(NB, n - k);
    int ps = prof_begin(s);
    potrf_diag_kernel<<<1, POTRF_THREADS, POTRF_SMEM, s>>>(at(k, k), ld, b, (int)k, info);
    prof_end(ps, s, PROF_DIAG, (double)b * b * b / 3.0);
    count_launch();
    FB_CK(cudaGetLastError());
    const long m2 = n - k - b;
    if (m2 <= 0) return FLA_SUCCESS;
    const long ldl = (b + 1) & ~1L;  // TMA: 16-byte leading dimensions
    if (tri_inverse_lower(at(k, k), ld, b, false, Linv, ldl, s) != FLA_SUCCESS) return FLA_FAILURE;
    const long ldw = (m2 + 1) & ~1L;
    FB_CK(cudaMemcpy2DAsync(W, sizeof(double) * ldw, at(k + b, k), sizeof(double) * ld, sizeof(double) * m2, b,
                            cudaMemcpyDeviceToDevice, s));
    return gemm_f64(s, false, true, m2, b, b, 1.0, W, ldw, Linv, ldl, 0.0, at(k + b, k), ld, GEMM_FULL, 0, info,
                    (int)(k + b));
  };

  if (panel(0, st) != FLA_SUCCESS) return FLA_FAILURE;
  for (long k = 0; k < n; k += NB) {
    const int b = (int)std::min<long>(NB, n - k);
    const long m2 = n - k - b;
    if (m2 <= 0) break;
    const int lim = (int)(k + b);
    const int nb2 = (int)std::min<long>(NB, m2);
    // the next panel's columns first
    if (gemm_f64(st, false, true, m2, nb2, b, -1.0, at(k + b, k), ld, at(k + b, k), ld, 1.0, at(k + b, k + b), ld,
                 GEMM_LOWER, 0, info, lim) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_look, st));
    FB_CK(cudaStreamWaitEvent(sd, ev_look, 0));
    if (panel(k + b, sd) != FLA_SUCCESS) return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_panel, sd));
    if (m2 > nb2 &&
        gemm_f64(st, false, true, m2 - nb2, m2 - nb2, b, -1.0, at(k + b + nb2, k), ld, at(k + b + nb2, k), ld, 1.0,
                 at(k + b + nb2, k + b + nb2), ld, GEMM_LOWER, 0, info, lim) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaStreamWaitEvent(st, ev_panel, 0));
  }
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// Factor one b x b (b <= 128) lower diagonal block in place (FP64); gcol is
// the global index of its first column for the info word.
int potrf_diag_dev(double* A, long ld, int b, int gcol, cudaStream_t st) {
  set_attrs();
  int ps = prof_begin(st);
  potrf_diag_kernel<<<1, POTRF_THREADS, POTRF_SMEM, st>>>(A, ld, b, gcol, ctx().d_status + ST_INFO);
  prof_end(ps, st, PROF_DIAG, (double)b * b * b / 3.0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

int chol_lower_dev(DMat A, int* info) {
  if (A.m == 0) {
    *info = -1;
    return FLA_SUCCESS;
  }
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;
  if (chol_lower_enqueue(A, ctx().stream) != FLA_SUCCESS) return FLA_FAILURE;
  return status_read(info);
}

}  // namespace fb
