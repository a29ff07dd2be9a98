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
#include <algorithm>
#include <climits>
#include <cstdlib>

#include "common.h"
#include "dev_util.cuh"

namespace fb {

namespace {

constexpr int NB = 128;        // outer block
constexpr int IB = 32;         // inner block
constexpr int LDS = NB + 1;    // SMEM leading dimension (odd: spreads banks)
constexpr int POTRF_THREADS = 256;
constexpr int POTRF_SMEM = NB * LDS * 8;
// Block columns of at most this many rows below the diagonal block are
// solved by substitution; taller ones through inv(L11) and a DMMA GEMM.
// FLA_B200_CHOL_SUBST_ROWS overrides it for tuning.
long chol_subst_rows() {
  static long v = -1;
  if (v < 0) {
    v = 4096;
    if (const char* e = std::getenv("FLA_B200_CHOL_SUBST_ROWS")) v = std::max(0L, std::atol(e));
  }
  return v;
}

__device__ __forceinline__ bool guard_failed(const int* info) {
  return *((volatile const int*)info) != INT_MAX;
}

// Factor the b x b (b <= 128) lower-triangular diagonal block at A (ld) in
// place.  gcol = global index of its first column (for the info word).
// Per 32-column chunk: (a) warp 0 factors the 32 x 32 diagonal block with
// one row per lane in registers, (b) one thread per row below solves
// X := X inv(L11)^T with its row in registers, (c) the trailing lower
// triangle of the block is updated, each thread a register tile of
// interleaved rows and columns (the shared-memory loads of one warp are
// broadcasts or consecutive words).  The update of the next chunk's 32
// columns comes first; warp 0 then factors the next diagonal block while
// the other seven warps update the columns beyond it.
// The pivot chain of (a) carries register values only: the next pivot is
// formed by its own lane from its own multiplier (fma(-l, l, a), the value
// the shared-memory column broadcast gives) and shuffled; each pivot's
// reciprocal square root is one rsqrt, its square root d * rsqrt(d).
__device__ __forceinline__ void cp_async8(double* dst, const double* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}

// S[r + c*LDS] -= sum_k S[r + (jb+k)*LDS] S[c + (jb+k)*LDS] (k < w) for the
// rows r in [r_lo, b) and columns c in [c_lo, c_hi), c <= r: thread (tx, ty)
// of a TX x TY grid owns rows r_lo + ty + TY a (a < RA) and columns c_lo +
// tx + TX q (q < CQ).
template <int TX, int TY, int RA, int CQ>
__device__ __forceinline__ void syrk_tile(double* S, int jb, int w, int r_lo, int c_lo, int c_hi, int b, int t) {
  const int tx = t % TX, ty = t / TX;
  double acc[RA][CQ];
#pragma unroll
  for (int a = 0; a < RA; ++a)
#pragma unroll
    for (int q = 0; q < CQ; ++q) acc[a][q] = 0.0;
  int ri[RA], ci[CQ];
#pragma unroll
  for (int a = 0; a < RA; ++a) ri[a] = min(r_lo + ty + TY * a, b - 1);
#pragma unroll
  for (int q = 0; q < CQ; ++q) ci[q] = min(c_lo + tx + TX * q, b - 1);
  for (int k = 0; k < w; ++k) {
    const double* col = S + (jb + k) * LDS;
    double xr[RA], xc[CQ];
#pragma unroll
    for (int a = 0; a < RA; ++a) xr[a] = col[ri[a]];
#pragma unroll
    for (int q = 0; q < CQ; ++q) xc[q] = col[ci[q]];
#pragma unroll
    for (int a = 0; a < RA; ++a)
#pragma unroll
      for (int q = 0; q < CQ; ++q) acc[a][q] += xr[a] * xc[q];
  }
#pragma unroll
  for (int a = 0; a < RA; ++a)
#pragma unroll
    for (int q = 0; q < CQ; ++q) {
      const int r = r_lo + ty + TY * a, c = c_lo + tx + TX * q;
      if (r < b && c < c_hi && c <= r) S[r + c * LDS] -= acc[a][q];
    }
}

// (a): warp 0 factors the w x w diagonal block at (jb, jb).  Every update is
// unconditional (no divergent branches in the chain): a lane only ever reads
// a[c] of its own row for c <= lane, and entries above the diagonal or past
// w never reach those.  After a failing pivot the rest of the block is not
// meaningful; the failing column is what is reported.
__device__ __forceinline__ void potrf_diag32(double* S, int jb, int w, int lane, double* s_rinv, double* s_col,
                                             int* s_fail) {
  double a[IB];
#pragma unroll
  for (int c = 0; c < IB; ++c)  // rows past w: unit pivots
    a[c] = (c <= lane && lane < w) ? S[(jb + lane) + (jb + c) * LDS] : (c == lane ? 1.0 : 0.0);
  int fail = -1;
  double d = __shfl_sync(0xffffffffu, a[0], 0);
#pragma unroll
  for (int j = 0; j < IB; ++j) {
    if (!(d > 0.0) && fail < 0 && j < w) fail = j;  // <= 0 or NaN
    const double rinv = rsqrt(d), sd = d * rinv;
    a[j] = lane == j ? sd : (lane > j ? a[j] * rinv : a[j]);
    if (lane == 0) s_rinv[j] = rinv;
    const double lj = a[j];
    if (j + 1 < IB) {
      // lane j + 1's next pivot from its own multiplier, then the broadcast
      const double dn = fma(-lj, lj, a[j + 1]);
      d = __shfl_sync(0xffffffffu, dn, j + 1);
      double* col = s_col + (j & 1) * IB;  // double-buffered column
      col[lane] = lj;
      __syncwarp();
#pragma unroll
      for (int c = j + 1; c < IB; ++c) a[c] = fma(-lj, col[c], a[c]);
    }
  }
#pragma unroll
  for (int c = 0; c < IB; ++c)
    if (c <= lane && lane < w) S[(jb + lane) + (jb + c) * LDS] = a[c];
  if (lane == 0 && fail >= 0) *s_fail = jb + fail;
}

__global__ void __launch_bounds__(POTRF_THREADS, 1) potrf_diag_kernel(double* A, long ld, int b, int gcol,
                                                                   int* info) {
  extern __shared__ double S[];  // S[r + c*LDS]
  __shared__ int s_fail;
  __shared__ double s_rinv[IB];
  __shared__ double s_col[2 * IB];
  if (guard_failed(info)) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // load the lower triangle (and diagonal) with asynchronous copies, all in
  // flight at once; the upper part of S is never read
  for (int c = warp; c < b; c += POTRF_THREADS / 32)
    for (int r = c + lane; r < b; r += 32) cp_async8(S + r + c * LDS, A + r + (long)c * ld);
  asm volatile("cp.async.wait_all;" ::: "memory");
  if (tid == 0) s_fail = -1;
  __syncthreads();
  if (warp == 0) potrf_diag32(S, 0, min(IB, b), lane, s_rinv, s_col, &s_fail);
  __syncthreads();
  for (int jb = 0;;) {
    if (s_fail >= 0) break;
    const int w = min(IB, b - jb);
    const int r0 = jb + w;  // first row below the diagonal block
    // (b) rows below: X := X inv(L11)^T, one thread per row (right-looking,
    //     multiply by the reciprocal of the pivot like dtrsm R,L,T,N).
    //     Columns past w only collect values that are never stored.
    for (int r = r0 + tid; r < b; r += POTRF_THREADS) {
      double x[IB];
#pragma unroll
      for (int c = 0; c < IB; ++c) x[c] = c < w ? S[r + (jb + c) * LDS] : 0.0;
#pragma unroll
      for (int j = 0; j < IB; ++j) {
        x[j] *= s_rinv[j];
#pragma unroll
        for (int c = j + 1; c < IB; ++c) x[c] -= x[j] * S[(jb + c) + (jb + j) * LDS];
      }
#pragma unroll
      for (int c = 0; c < IB; ++c)
        if (c < w) S[r + (jb + c) * LDS] = x[c];
    }
    __syncthreads();
    if (r0 >= b) break;
    const int w2 = min(IB, b - r0);
    // (c) first the next chunk's columns (all rows below r0) ...
    syrk_tile<32, 8, 12, 1>(S, jb, w, r0, r0, r0 + w2, b, tid);
    __syncthreads();
    // ... then warp 0 factors the next diagonal block while the other warps
    // update the columns beyond it
    if (warp == 0) {
      potrf_diag32(S, r0, w2, lane, s_rinv, s_col, &s_fail);
    } else if (r0 + w2 < b) {
      syrk_tile<16, 14, 5, 4>(S, jb, w, r0 + w2, r0 + w2, b, b, tid - 32);
    }
    __syncthreads();
    jb = r0;
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

// Outer blocksize of FLA_Chol: the depth of the trailing updates.  256 by
// default (the DMMA GEMM runs its K=256 updates about a fifth faster than
// K=128 ones); FLA_B200_CHOL_BLOCKSIZE = 128 or 256 overrides it.
int chol_blocksize() {
  static int nb = 0;
  if (nb == 0) {
    nb = 256;
    if (const char* e = std::getenv("FLA_B200_CHOL_BLOCKSIZE")) {
      const int v = std::atoi(e);
      if (v == 128 || v == 256) nb = v;
    }
  }
  return nb;
}

// Enqueue the blocked factorization of the lower triangle of A on `st`.
// Outer blocks of NBO = 128 or 256 columns; each outer panel is factored as
// 128-column sub-panels:
//   sub-panel j:   A11 := chol(A11); inv(L11) formed next to it;
//                  A21 := A21 inv(L11)^T as a DMMA GEMM;
//                  the panel's later columns -= A21 A21^T
//   then the panel's rows below its diagonal block are copied transposed,
//   and step k updates A22(:, next panel) -= A21 A21(next rows)^T, factors
//   the next panel on the second stream, and meanwhile updates
//   A22(rest) -= A21 A21^T (lower) on the main stream.
// Failure semantics follow FLA_Chol_l_blk_var3: the updates of step k run
// unless a column before k + b has failed (the guard limit of each launch),
// so a failure in the next panel does not cut short step k's update.
int chol_lower_enqueue(DMat A, cudaStream_t st) {
  set_attrs();
  Context& cx = ctx();
  const long n = A.m, ld = A.ld;
  if (n <= 0) return FLA_SUCCESS;
  int* info = cx.d_status + ST_INFO;
  // The next panel is factored on the library's second stream beside the
  // trailing update (as in FLA_LU_piv); FLA_B200_CHOL_LOOKAHEAD=0 keeps the
  // panels in stream order.  Only calls on the library's main stream
  // overlap; a call on another stream runs in that stream's order.
  static const bool look = [] {
    const char* e = std::getenv("FLA_B200_CHOL_LOOKAHEAD");
    return !(e && e[0] == '0');
  }();
  cudaStream_t sd = (look && st == cx.stream) ? cx.side : st;
  const long NBO = chol_blocksize();
  double* Linv = (double*)ws_get(WS_MISC, sizeof(double) * NB * NB);
  double* W = (double*)ws_get(WS_MISC2, sizeof(double) * NB * (size_t)(std::max<long>(0, n - NB) + 2));
  // Transposed copy of each factored outer panel's rows below its diagonal
  // block (NBO x rows, k contiguous), two buffers used in turn: the
  // lookahead and trailing updates take their second operand from it
  // k-contiguous (one 16 x 64 TMA box per stage, the LU's operand shape).
  const long ldpt = NBO;
  double* PT = (double*)ws_get(WS_PANEL_T, sizeof(double) * 2 * (size_t)ldpt * (size_t)std::max<long>(n, 1));
  if (!Linv || !W || !PT) return FLA_FAILURE;
  auto pt_of = [&](long k) { return PT + ((k / NBO) & 1) * (size_t)ldpt * (size_t)n; };
  cudaEvent_t ev_look = cx.ev[2], ev_panel = cx.ev[3];
  auto at = [&](long i, long j) { return A.p + i + j * ld; };

  // 128-column sub-panel at column k: diagonal block, its inverse, and the
  // block column below it.
  auto sub = [&](long k, cudaStream_t s) -> int {
    const int b = (int)std::min<long>(NB, n - k);
    int ps = prof_begin(s);
    potrf_diag_kernel<<<1, POTRF_THREADS, POTRF_SMEM, s>>>(at(k, k), ld, b, (int)k, info);
    prof_end(ps, s, PROF_DIAG, (double)b * b * b / 3.0);
    count_launch();
    FB_CK(cudaGetLastError());
    const long m2 = n - k - b;
    if (m2 <= 0) return FLA_SUCCESS;
    // a short block column: forward substitution in one launch (the latency
    // of the inverse, the copy and the product would dominate it)
    if (m2 <= chol_subst_rows()) return trsm_rlt_subst(at(k, k), at(k + b, k), ld, b, m2, info, (int)(k + b), s);
    const long ldl = (b + 1) & ~1L;  // TMA: 16-byte leading dimensions
    if (tri_inverse_lower(at(k, k), ld, b, false, Linv, ldl, s) != FLA_SUCCESS) return FLA_FAILURE;
    const long ldw = (m2 + 1) & ~1L;
    FB_CK(cudaMemcpy2DAsync(W, sizeof(double) * ldw, at(k + b, k), sizeof(double) * ld, sizeof(double) * m2, b,
                            cudaMemcpyDeviceToDevice, s));
    return gemm_f64(s, false, true, m2, b, b, 1.0, W, ldw, Linv, ldl, 0.0, at(k + b, k), ld, GEMM_FULL, 0, info,
                    (int)(k + b));
  };
  // Outer panel at column k: its sub-panels left to right, each followed by
  // the update of the panel's remaining columns; then the transposed copy of
  // its rows below the diagonal block.
  auto panel = [&](long k, cudaStream_t s) -> int {
    const long kend = std::min<long>(n, k + NBO);
    for (long j = k; j < kend; j += NB) {
      if (sub(j, s) != FLA_SUCCESS) return FLA_FAILURE;
      const long bj = std::min<long>(NB, n - j), j2 = j + bj;
      if (j2 >= kend) break;
      if (gemm_f64(s, false, true, n - j2, kend - j2, bj, -1.0, at(j2, j), ld, at(j2, j), ld, 1.0, at(j2, j2), ld,
                   GEMM_LOWER, 0, info, (int)j2) != FLA_SUCCESS)
        return FLA_FAILURE;
    }
    if (n > kend)
      return transpose_dev(at(kend, k), ld, pt_of(k), ldpt, n - kend, kend - k, false, s);
    return FLA_SUCCESS;
  };

  if (panel(0, st) != FLA_SUCCESS) return FLA_FAILURE;
  for (long k = 0; k < n; k += NBO) {
    const long b = std::min<long>(NBO, n - k);
    const long m2 = n - k - b;
    if (m2 <= 0) break;
    const int lim = (int)(k + b);
    const long nb2 = std::min<long>(NBO, m2);
    // the next panel's columns first; op(B) = panel^T from its transposed copy
    // (column c of the copy is panel row k + b + c)
    const double* pt = pt_of(k);
    if (gemm_f64(st, false, false, m2, nb2, b, -1.0, at(k + b, k), ld, pt, ldpt, 1.0, at(k + b, k + b), ld,
                 GEMM_LOWER, 0, info, lim) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_look, st));
    FB_CK(cudaStreamWaitEvent(sd, ev_look, 0));
    if (panel(k + b, sd) != FLA_SUCCESS) return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_panel, sd));
    if (m2 > nb2 &&
        gemm_f64(st, false, false, m2 - nb2, m2 - nb2, b, -1.0, at(k + b + nb2, k), ld, pt + nb2 * ldpt, ldpt, 1.0,
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
