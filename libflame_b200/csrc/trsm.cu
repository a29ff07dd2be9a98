// Triangular solves with one diagonal block (b <= 128) on the GPU.
//
//   left:  X := inv(op(T)) X   for a b x n block X      (LU: A12 := inv(L11) A12,
//                                                      solves, QR: W := T^-T W)
//   right: X := X inv(L)^T     for an m x b block X      (Chol: A21 := A21 inv(L11)^T)
//
// Replaces the dtrsm_ calls of the reference's blocked algorithms
// (FLA_Trsm_external, src/base/flamec/wrappers/blas/3/external/
// FLA_Trsm_external.c:72).  Substitution order follows dtrsm: forward when
// op(T) is lower, backward when upper; non-unit diagonals are applied as a
// multiplication by the reciprocal of the pivot (as dtrsm's R,L,T,N case,
// src/flablas/f2c/dtrsm.c).
//
// One CTA owns 64 right-hand sides (columns of X for left, rows for right),
// kept in shared memory with the triangle, and sweeps the b steps: scale the
// current unknown (one thread per right-hand side), then update the
// remaining unknowns (all threads).  The step loop is not unrolled, so the
// kernel stays small in the instruction cache.
#include <algorithm>

#include "common.h"
#include "dev_util.cuh"

namespace fb {

namespace {

constexpr int TB = 128;             // max triangle order
constexpr int NV = 64;              // right-hand sides per CTA
constexpr int THREADS = 256;
constexpr int LDT = TB + 1;         // SMEM stride of the triangle
constexpr int LDX = TB + 1;         // SMEM stride of one right-hand side
constexpr size_t SMEM = (size_t)(TB * LDT + NV * LDX + NV + TB) * sizeof(double);

// coef(r, j): entry of op(T) at (r, j), from the stored triangle S
template <bool TRANS>
__device__ __forceinline__ double coef(const double* S, int r, int j) {
  return TRANS ? S[j + r * LDT] : S[r + j * LDT];
}

template <bool LOWER, bool TRANS, bool UNIT, bool RIGHT>
__global__ void __launch_bounds__(THREADS) trsm_tile_kernel(const double* __restrict__ T, long ldt,
                                                            double* __restrict__ X, long ldx, int b,
                                                            int nvec, const int* guard) {
  extern __shared__ double sm[];
  double* ST = sm;                    // b x b triangle (stored part only)
  double* SX = ST + TB * LDT;         // NV right-hand sides, SX[r + v*LDX]
  double* sx = SX + NV * LDX;         // scaled current unknown per rhs
  double* sd = sx + NV;               // reciprocal diagonal
  if (guard && *((volatile const int*)guard) != 0x7fffffff) return;
  constexpr bool FWD = (LOWER != TRANS);
  const int tid = threadIdx.x;
  const int v0 = blockIdx.x * NV;
  const int nv = min(NV, nvec - v0);
  load_block_f64<THREADS, true>(T, ldt, b, ST, LDT, [](int r, int c) { return LOWER ? (r >= c) : (r <= c); });
  // right-hand side v, unknown r: left -> X(r, v0+v); right -> X(v0+v, r)
  if (!RIGHT) {
    for (int v = tid >> 5; v < nv; v += THREADS / 32)
      for (int r = tid & 31; r < b; r += 32) SX[r + v * LDX] = X[r + (long)(v0 + v) * ldx];
  } else {
    for (int r = tid >> 6; r < b; r += THREADS / 64)
      for (int v = tid & 63; v < nv; v += 64) SX[r + v * LDX] = X[(long)(v0 + v) + (long)r * ldx];
  }
  __syncthreads();
  if (!UNIT)
    for (int j = tid; j < b; j += THREADS) sd[j] = 1.0 / ST[j + j * LDT];
  __syncthreads();
  for (int jj = 0; jj < b; ++jj) {
    const int j = FWD ? jj : (b - 1 - jj);
    if (tid < nv) {
      double x = SX[j + tid * LDX];
      if (!UNIT) {
        x *= sd[j];
        SX[j + tid * LDX] = x;
      }
      sx[tid] = x;
    }
    __syncthreads();
    // remaining unknowns: FWD r in (j, b), BWD r in [0, j)
    const int r_lo = FWD ? j + 1 : 0;
    const int cnt = (FWD ? (b - j - 1) : j) * nv;
    if (nv == NV) {
      for (int e = tid; e < cnt; e += THREADS) {
        const int r = r_lo + (e >> 6), v = e & (NV - 1);
        SX[r + v * LDX] -= coef<TRANS>(ST, r, j) * sx[v];
      }
    } else {
      for (int e = tid; e < cnt; e += THREADS) {
        const int r = r_lo + e / nv, v = e % nv;
        SX[r + v * LDX] -= coef<TRANS>(ST, r, j) * sx[v];
      }
    }
    __syncthreads();
  }
  if (!RIGHT) {
    for (int v = tid >> 5; v < nv; v += THREADS / 32)
      for (int r = tid & 31; r < b; r += 32) X[r + (long)(v0 + v) * ldx] = SX[r + v * LDX];
  } else {
    for (int r = tid >> 6; r < b; r += THREADS / 64)
      for (int v = tid & 63; v < nv; v += 64) X[(long)(v0 + v) + (long)r * ldx] = SX[r + v * LDX];
  }
}

// X := inv(T) for a b x b triangular T (b <= 128), one warp per column of X.
// Column c of inv(T) solves T x = e_c: the warp keeps the running right-hand
// side in registers (lane l holds rows l, l+32, l+64, l+96), and at each step
// the owner of the current unknown broadcasts it (multiplied by the
// reciprocal of the pivot unless UNIT) and every lane updates its rows with
// one column of T from shared memory.  No block barriers inside the sweep,
// so the b steps cost only warp-level latency.
constexpr int INV_WARPS = 16;
constexpr size_t INV_SMEM = (size_t)(TB * LDT + TB) * sizeof(double);
// Batched over the diagonal blocks of order bs (<= TB) of an n x n
// triangle: blockIdx.y = block index q, T_q = T + q*bs*(1 + ldt), X_q = X +
// q * xstride; with gridDim.y = 1 and n = b, the single b x b block.
template <bool LOWER, bool UNIT>
__global__ void __launch_bounds__(INV_WARPS * 32) tri_inv_kernel(const double* __restrict__ T, long ldt,
                                                                 double* __restrict__ X, long ldx, int n,
                                                                 long xstride, int bs = TB) {
  extern __shared__ double sm[];
  double* ST = sm;             // stored triangle, ST[r + c*LDT]
  double* sd = ST + TB * LDT;  // reciprocal diagonal
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = blockIdx.y;
  const int b = min(bs, n - q * bs);
  T += (long)q * bs * (1 + ldt);
  X += (long)q * xstride;
  load_block_f64<INV_WARPS * 32, true>(T, ldt, b, ST, LDT, [](int r, int c) { return LOWER ? (r >= c) : (r <= c); });
  __syncthreads();
  if (!UNIT)
    for (int j = tid; j < b; j += INV_WARPS * 32) sd[j] = 1.0 / ST[j + j * LDT];
  __syncthreads();
  const int c = blockIdx.x * INV_WARPS + warp;
  if (c >= b) return;
  double r[4];
#pragma unroll
  for (int m = 0; m < 4; ++m) r[m] = (lane + 32 * m == c) ? 1.0 : 0.0;
  const int j_first = c, j_last = LOWER ? b - 1 : 0;
  const int nsteps = LOWER ? (b - c) : (c + 1);
  for (int s = 0; s < nsteps; ++s) {
    const int j = LOWER ? j_first + s : j_first - s;
    const int slot = j >> 5;
    double v = r[0];
#pragma unroll
    for (int m = 1; m < 4; ++m)
      if (slot == m) v = r[m];
    double xj = __shfl_sync(0xffffffffu, v, j & 31);
    if (!UNIT) xj *= sd[j];
    // branch-free: rows outside the triangle multiply a zero of ST
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      const int i = lane + 32 * m;
      const double t = r[m] - ST[i + j * LDT] * xj;
      r[m] = (i == j) ? xj : ((LOWER ? (i > j) : (i < j)) ? t : r[m]);
    }
  }
  (void)j_last;
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    const int i = lane + 32 * m;
    if (i < b) X[i + (long)c * ldx] = (LOWER ? i >= c : i <= c) ? r[m] : 0.0;
  }
}

template <bool L, bool T, bool U, bool R>
void set_attr_one() {
  cudaFuncSetAttribute(trsm_tile_kernel<L, T, U, R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
}

bool g_attr = false;
void set_attrs() {
  if (g_attr) return;
  set_attr_one<true, false, true, false>();
  set_attr_one<true, false, false, false>();
  set_attr_one<true, true, true, false>();
  set_attr_one<true, true, false, false>();
  set_attr_one<false, false, true, false>();
  set_attr_one<false, false, false, false>();
  set_attr_one<false, true, true, false>();
  set_attr_one<false, true, false, false>();
  set_attr_one<true, false, false, true>();
  set_attr_one<true, false, true, true>();
  set_attr_one<true, true, false, true>();
  set_attr_one<true, true, true, true>();
  set_attr_one<false, false, false, true>();
  set_attr_one<false, false, true, true>();
  set_attr_one<false, true, false, true>();
  set_attr_one<false, true, true, true>();
  cudaFuncSetAttribute(tri_inv_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INV_SMEM);
  cudaFuncSetAttribute(tri_inv_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INV_SMEM);
  cudaFuncSetAttribute(tri_inv_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INV_SMEM);
  cudaFuncSetAttribute(tri_inv_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INV_SMEM);
  g_attr = true;
}

}  // namespace

// B := inv(op(T)) B for a b x n block B, T b x b (b <= 128) triangular.
int trsm_block(const double* T, long ldt, double* B, long ldb, int b, long n, bool lower, bool trans,
               bool unit, cudaStream_t st) {
  set_attrs();
  if (n <= 0 || b <= 0) return FLA_SUCCESS;
  const unsigned grid = (unsigned)((n + NV - 1) / NV);
  const int ps = prof_begin(st);
#define FB_TRSM_LAUNCH(L, T_, U) \
  trsm_tile_kernel<L, T_, U, false><<<grid, THREADS, SMEM, st>>>(T, ldt, B, ldb, b, (int)n, nullptr)
  if (lower) {
    if (!trans) { if (unit) FB_TRSM_LAUNCH(true, false, true); else FB_TRSM_LAUNCH(true, false, false); }
    else        { if (unit) FB_TRSM_LAUNCH(true, true, true);  else FB_TRSM_LAUNCH(true, true, false); }
  } else {
    if (!trans) { if (unit) FB_TRSM_LAUNCH(false, false, true); else FB_TRSM_LAUNCH(false, false, false); }
    else        { if (unit) FB_TRSM_LAUNCH(false, true, true);  else FB_TRSM_LAUNCH(false, true, false); }
  }
#undef FB_TRSM_LAUNCH
  prof_end(ps, st, PROF_TRSM, (double)b * (double)b * (double)n);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// X := X inv(L)^T for an m x b block X, L b x b lower non-unit (b <= 128);
// the kernel returns at once when *guard no longer holds INT_MAX.
int trsm_right_lt_block(const double* L, long ldl, double* X, long ldx, long m, int b, const int* guard,
                        cudaStream_t st) {
  set_attrs();
  if (m <= 0 || b <= 0) return FLA_SUCCESS;
  const unsigned grid = (unsigned)((m + NV - 1) / NV);
  const int ps = prof_begin(st);
  // X L^T = B  <=>  L X^T = B^T: a forward solve with L per row of X
  trsm_tile_kernel<true, false, false, true><<<grid, THREADS, SMEM, st>>>(L, ldl, X, ldx, b, (int)m, guard);
  prof_end(ps, st, PROF_TRSM, (double)m * (double)b * (double)b);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}


__global__ void set_identity_kernel(double* X, long ldx, int n) {
  const long total = (long)n * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long r = e % n, c = e / n;
    X[r + c * ldx] = (r == c) ? 1.0 : 0.0;
  }
}

// X := inv(L) for the b x b lower-triangular L (unit diagonal if `unit`),
// X b x b with leading dimension ldx: X := I, then the blocked left solve
// L X = I (128-row diagonal solves and GEMM updates).  Used to turn the
// factorizations' panel triangular solves into DMMA GEMMs.
int tri_inverse_lower(const double* L, long ldl, int b, bool unit, double* X, long ldx, cudaStream_t st) {
  return tri_inverse(L, ldl, b, true, unit, X, ldx, st);
}


// Every row x of the m x b block X := solution y of op(T) y = x, i.e.
// X := X inv(op(T))^T (T b x b, b <= 128).
int trsm_right_block(const double* T, long ldt, double* X, long ldx, long m, int b, bool lower, bool trans,
                     bool unit, cudaStream_t st) {
  set_attrs();
  if (m <= 0 || b <= 0) return FLA_SUCCESS;
  const unsigned grid = (unsigned)((m + NV - 1) / NV);
  const int ps = prof_begin(st);
#define FB_TRSM_R(L, T_, U) \
  trsm_tile_kernel<L, T_, U, true><<<grid, THREADS, SMEM, st>>>(T, ldt, X, ldx, b, (int)m, nullptr)
  if (lower) {
    if (!trans) { if (unit) FB_TRSM_R(true, false, true); else FB_TRSM_R(true, false, false); }
    else        { if (unit) FB_TRSM_R(true, true, true);  else FB_TRSM_R(true, true, false); }
  } else {
    if (!trans) { if (unit) FB_TRSM_R(false, false, true); else FB_TRSM_R(false, false, false); }
    else        { if (unit) FB_TRSM_R(false, true, true);  else FB_TRSM_R(false, true, false); }
  }
#undef FB_TRSM_R
  prof_end(ps, st, PROF_TRSM, (double)m * (double)b * (double)b);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// X := inv(T) for a b x b triangular T: one warp per column when b <= 128,
// else X := I and the blocked left solve.
int tri_inverse(const double* T, long ldt, int b, bool lower, bool unit, double* X, long ldx, cudaStream_t st) {
  if (b <= 0) return FLA_SUCCESS;
  if (b <= TB) {
    set_attrs();
    const unsigned grid = (unsigned)((b + INV_WARPS - 1) / INV_WARPS);
    const int ps = prof_begin(st);
    if (lower) {
      if (unit) tri_inv_kernel<true, true><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, ldx, b, 0);
      else tri_inv_kernel<true, false><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, ldx, b, 0);
    } else {
      if (unit) tri_inv_kernel<false, true><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, ldx, b, 0);
      else tri_inv_kernel<false, false><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, ldx, b, 0);
    }
    prof_end(ps, st, PROF_TRSM, (double)b * b * b / 3.0);
    count_launch();
    FB_CK(cudaGetLastError());
    return FLA_SUCCESS;
  }
  const int blocks = (int)std::min<long>(1024, ((long)b * b + 255) / 256);
  set_identity_kernel<<<blocks, 256, 0, st>>>(X, ldx, b);
  count_launch();
  FB_CK(cudaGetLastError());
  DMat Tm, B;
  Tm.p = const_cast<double*>(T);
  Tm.ld = ldt;
  Tm.m = Tm.n = b;
  B.p = X;
  B.ld = ldx;
  B.m = B.n = b;
  return trsm_left_dev(Tm, B, lower, false, unit, st);
}


// Inverses of all 128 x 128 diagonal blocks of the n x n triangle T in one
// launch: block q (order min(128, n - 128 q)) into X + q * 128 * 128, ld 128.
int tri_inverse_blocks(const double* T, long ldt, long n, bool lower, bool unit, double* X, cudaStream_t st) {
  if (n <= 0) return FLA_SUCCESS;
  set_attrs();
  const long nblk = (n + TB - 1) / TB;
  dim3 grid((unsigned)((TB + INV_WARPS - 1) / INV_WARPS), (unsigned)nblk);
  const long xs = (long)TB * TB;
  const int ps = prof_begin(st);
  if (lower) {
    if (unit) tri_inv_kernel<true, true><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, TB, (int)n, xs);
    else tri_inv_kernel<true, false><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, TB, (int)n, xs);
  } else {
    if (unit) tri_inv_kernel<false, true><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, TB, (int)n, xs);
    else tri_inv_kernel<false, false><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, TB, (int)n, xs);
  }
  prof_end(ps, st, PROF_TRSM, (double)n * TB * TB / 3.0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// Inverses of the bs x bs diagonal blocks (bs <= 128) of the n x n
// triangle T in one launch: block q (order min(bs, n - bs q)) into
// X + q * bs * bs, ld bs.
int tri_inverse_blocks_bs(const double* T, long ldt, long n, int bs, bool lower, bool unit, double* X,
                          cudaStream_t st) {
  if (n <= 0) return FLA_SUCCESS;
  set_attrs();
  const long nblk = (n + bs - 1) / bs;
  dim3 grid((unsigned)((bs + INV_WARPS - 1) / INV_WARPS), (unsigned)nblk);
  const long xs = (long)bs * bs;
  const int ps = prof_begin(st);
  if (lower) {
    if (unit) tri_inv_kernel<true, true><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, bs, (int)n, xs, bs);
    else tri_inv_kernel<true, false><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, bs, (int)n, xs, bs);
  } else {
    if (unit) tri_inv_kernel<false, true><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, bs, (int)n, xs, bs);
    else tri_inv_kernel<false, false><<<grid, INV_WARPS * 32, INV_SMEM, st>>>(T, ldt, X, bs, (int)n, xs, bs);
  }
  prof_end(ps, st, PROF_TRSM, (double)n * bs * bs / 3.0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

}  // namespace fb
