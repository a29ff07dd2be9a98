// Mixed-precision solvers: factor in low precision on the tensor cores,
// refine in FP64.
//
// Reference behaviour: dsgesv_ / dsposv_ (src/map/common/lapacksrc/f2c/
// dsgesv.c:189-412, dsposv.c:250-413): factor a single-precision copy,
// x = solve(b), then up to ITERMAX = 30 refinement steps r = b - A x (FP64),
// x += solve(r), stopping when every column has ||r||_inf <= ||x||_inf * cte
// with cte = ||A||_inf * eps * sqrt(n) (eps = DBL_EPSILON / 2, dlamch 'E');
// on failure fall back to the FP64 factorization (iter = -2 overflow, -3
// factorization failure, -31 no convergence).
//
// B200 form:
//   * the working copy of A is FP32; the panels are factored in FP64 by the
//     same kernels as the plain FP64 path (cluster LU leaves, diagonal-block
//     Cholesky) and rounded back, while every trailing update and panel
//     solve is a 16-bit (BF16 or FP16) tensor-core GEMM with FP32
//     accumulation (lp_gemm.cu), with the same one-panel lookahead on a
//     second stream;
//   * optional power-of-two equilibration (rows and columns for LU, the
//     symmetric diag(a_ii)^-1/2 for Cholesky) keeps the 16-bit operands in
//     range (required for FP16);
//   * the correction solves run in FP32 with the inverted diagonal blocks
//     formed during the factorization (two GEMMs per block);
//   * FP64 is used only for r = b - A x (DMMA GEMM), the update of x and the
//     norms;
//   * GMRES-IR: the correction equation A d = r is solved by GMRES(m) left-
//     preconditioned with the low-precision factors, in FP64, all right-hand
//     sides in lockstep (one GEMM per matrix-vector product), which carries
//     the refinement to condition numbers beyond 1/u of the factorization.
#include <algorithm>
#include <cfloat>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "dev_util.cuh"
#include "lowprec.h"
#include "mixed.h"

namespace fb {

namespace {

constexpr int MB = 128;  // block size of the low-precision factorizations
constexpr int NBO = 256;  // outer block of the low-precision Cholesky (depth of its updates)

// AT[j + i * ldt] = (float)(A[i + j * lda] * sr[i] * sc[j])   (A m x n)
__global__ void transpose_scale_kernel(const double* __restrict__ A, long lda, float* __restrict__ AT, long ldt,
                                       int m, int n, const double* __restrict__ sr, const double* __restrict__ sc) {
  __shared__ float tile[32][33];
  const int bi = blockIdx.x * 32, bj = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int i = bi + threadIdx.x, j = bj + y;
    float v = 0.f;
    if (i < m && j < n) {
      double a = A[i + (long)j * lda];
      if (sr) a *= sr[i];
      if (sc) a *= sc[j];
      v = (float)a;
    }
    tile[y][threadIdx.x] = v;
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    const int j = bj + threadIdx.x, i = bi + y;
    if (i < m && j < n) AT[j + (long)i * ldt] = tile[threadIdx.x][y];
  }
}

// F[i + j * ldf] = (float)(a(i, j) * d[i] * d[j]) for i >= j, a(i, j) from the
// stored triangle (upper: a(i, j) = A[j + i * lda]).
// (plus sigma on the diagonal: the shifted factorization of the retries)
__global__ void lower_scale_kernel(const double* __restrict__ A, long lda, float* __restrict__ F, long ldf, int n,
                                   const double* __restrict__ d, int upper, double sigma) {
  const long total = (long)n * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, j = e / n;
    if (i < j) continue;
    double a = upper ? A[j + i * lda] : A[i + j * lda];
    if (d) a *= d[i] * d[j];
    if (i == j) a += sigma;
    F[i + j * ldf] = (float)a;
  }
}

// Full symmetric copy S from the stored triangle of A.
__global__ void symmetrize_kernel(const double* __restrict__ A, long lda, double* __restrict__ S, long lds, int n,
                                  int upper) {
  const long total = (long)n * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, j = e / n;
    const bool stored = upper ? (i <= j) : (i >= j);
    S[i + j * lds] = stored ? A[i + j * lda] : A[j + i * lda];
  }
}

// out[i] = max_j |A(i, j)| * (cs ? cs[j] : 1), one thread per row (the warp
// reads 32 consecutive rows of a column: coalesced).
__global__ void row_absmax_kernel(const double* __restrict__ A, long lda, int m, int n, const double* __restrict__ cs,
                                  double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double v = 0.0;
  for (int j = 0; j < n; ++j) v = fmax(v, fabs(A[i + (long)j * lda]) * (cs ? cs[j] : 1.0));
  out[i] = v;
}
// out[j] = max_i |A(i, j)| * rs[i], one block per column.
__global__ void col_absmax_kernel(const double* __restrict__ A, long lda, int m, const double* __restrict__ rs,
                                  double* __restrict__ out) {
  __shared__ double red[256];
  const int j = blockIdx.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) v = fmax(v, fabs(A[i + (long)j * lda]) * (rs ? rs[i] : 1.0));
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = red[0];
}
// v[i] := 2^-e with v[i] = f 2^e, f in [0.5, 1): an exact power-of-two
// reciprocal (1 where v[i] is 0 or not finite).
__global__ void pow2_recip_kernel(double* v, int n, int sqrt_of) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x = v[i];
  if (!(x > 0.0) || !isfinite(x)) {
    v[i] = 1.0;
    return;
  }
  int e;
  frexp(x, &e);
  v[i] = ldexp(1.0, sqrt_of ? -(e / 2) : -e);
}
// diagonal of A into v
__global__ void diag_kernel(const double* __restrict__ A, long lda, int n, double* __restrict__ v) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] = fabs(A[i + (long)i * lda]);
}
// ||A||_inf = max_i sum_j |a_ij|, one thread per row; the maximum is taken
// with an integer atomicMax on the (non-negative) double's bits
__global__ void inf_norm_kernel(const double* __restrict__ A, long lda, int n, unsigned long long* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double s = 0.0;
  for (int j = 0; j < n; ++j) s += fabs(A[i + (long)j * lda]);
  atomicMax(out, (unsigned long long)__double_as_longlong(s));
}
// out[c] = max_i |X(i, c)|, one block per column
__global__ void colmax_kernel(const double* __restrict__ X, long ldx, int n, double* __restrict__ out) {
  __shared__ double red[256];
  const int c = blockIdx.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v = fmax(v, fabs(X[i + (long)c * ldx]));
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[c] = red[0];
}
// Y(i, c) = (TO)(X(i, c) * (s ? s[i] : 1))
template <typename TO, typename TI>
__global__ void scale_copy_kernel(const TI* __restrict__ X, long ldx, TO* __restrict__ Y, long ldy, int n, int nrhs,
                                  const double* __restrict__ s) {
  const long total = (long)n * nrhs;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, c = e / n;
    double v = (double)X[i + c * ldx];
    if (s) v *= s[i];
    Y[i + c * ldy] = (TO)v;
  }
}
// X(i, c) += sign * D(i, c)
__global__ void add_kernel(double* __restrict__ X, long ldx, const double* __restrict__ D, long ldd, int n,
                           int nrhs, double sign) {
  const long total = (long)n * nrhs;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, c = e / n;
    X[i + c * ldx] += sign * D[i + c * ldd];
  }
}
// out[q + c * nv] = sum_i V_q(i, c) W(i, c), V_q = V + q * vstride; grid (nrhs, nv)
__global__ void coldots_kernel(const double* __restrict__ V, long vstride, const double* __restrict__ W, long ld,
                               int n, int nv, double* __restrict__ out) {
  __shared__ double red[256];
  const int c = blockIdx.x, q = blockIdx.y;
  const double* v = V + q * vstride + (long)c * ld;
  const double* w = W + (long)c * ld;
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s = fma(v[i], w[i], s);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[q + (long)c * nv] = red[0];
}
// W(i, c) += sign * sum_q coef[q + c * nv] V_q(i, c)
__global__ void col_combine_kernel(double* __restrict__ W, const double* __restrict__ V, long vstride, long ld,
                                   int n, int nrhs, int nv, const double* __restrict__ coef, double sign) {
  const long total = (long)n * nrhs;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, c = e / n;
    double s = 0.0;
    for (int q = 0; q < nv; ++q) s = fma(coef[q + c * nv], V[q * vstride + i + c * ld], s);
    W[i + c * ld] += sign * s;
  }
}
// Y(i, c) = X(i, c) * f[c]
__global__ void colscale_kernel(const double* __restrict__ X, double* __restrict__ Y, long ld, int n, int nrhs,
                                const double* __restrict__ f) {
  const long total = (long)n * nrhs;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, c = e / n;
    Y[i + c * ld] = X[i + c * ld] * f[c];
  }
}

// perm[i] = source row of row i of P b: the pivot interchanges applied in
// order to the identity (one thread; the vector in shared memory when it
// fits, else in perm itself)
__global__ void perm_from_pivots_kernel(const int* __restrict__ piv, int n, int* __restrict__ perm, int use_smem) {
  extern __shared__ int sp[];
  int* v = use_smem ? sp : perm;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v[i] = i;
  __syncthreads();
  if (threadIdx.x == 0)
    for (int i = 0; i < n; ++i) {
      const int t = i + piv[i];
      const int x = v[i];
      v[i] = v[t];
      v[t] = x;
    }
  __syncthreads();
  if (use_smem)
    for (int i = threadIdx.x; i < n; i += blockDim.x) perm[i] = v[i];
}
// T(i, c) = (float)(R(perm[i], c) * s[perm[i]])
__global__ void gather_rows_kernel(const double* __restrict__ R, long ldr, const int* __restrict__ perm,
                                   const double* __restrict__ s, float* __restrict__ T, long ldt, int n, int nrhs) {
  const long total = (long)n * nrhs;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % n, c = e / n;
    const int src = perm[i];
    double v = R[src + c * ldr];
    if (s) v *= s[src];
    T[i + c * ldt] = (float)v;
  }
}

// Building blocks of the blocked triangular sweeps (FP32, 128-row blocks,
// nr <= 32 right-hand sides) of the correction solves.
// 128 x 128 block of op(P) into registers, 16 float4 per thread, every load
// in flight at once.  ROWMAJ: element (i, k) at P[k + i * ld], else
// P[i + k * ld]; the contiguous index runs in float4 steps (the caller
// guarantees 16-byte alignment and that the float4 holding the last valid
// element lies inside the allocation).  Columns k >= mk are zero (padding
// columns would otherwise multiply zeros of the right-hand block by
// whatever the workspace holds); rows i >= mi are zero too.
template <bool ROWMAJ>
__device__ __forceinline__ void block_load(const float* __restrict__ P, long ld, int mi, int mk, float4 (&v)[16]) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int e4 = threadIdx.x + j * 256;
    const int a = e4 >> 5, b4 = (e4 & 31) * 4;  // ROWMAJ: (row a, columns b4..); else (column a, rows b4..)
    const int i = ROWMAJ ? a : b4, k = ROWMAJ ? b4 : a;
    float4 x = make_float4(0.f, 0.f, 0.f, 0.f);
    if (ROWMAJ ? (i < mi && k < mk) : (k < mk && i < mi))
      x = *reinterpret_cast<const float4*>(ROWMAJ ? P + k + (long)i * ld : P + i + (long)k * ld);
    if (ROWMAJ) {
      if (k + 1 >= mk) x.y = 0.f;
      if (k + 2 >= mk) x.z = 0.f;
      if (k + 3 >= mk) x.w = 0.f;
    } else {
      if (i + 1 >= mi) x.y = 0.f;
      if (i + 2 >= mi) x.z = 0.f;
      if (i + 3 >= mi) x.w = 0.f;
    }
    v[j] = x;
  }
}
// ... and into shared memory as sF[i * 129 + k]
template <bool ROWMAJ>
__device__ __forceinline__ void block_store(float* sF, const float4 (&v)[16]) {
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    const int e4 = threadIdx.x + j * 256;
    const int a = e4 >> 5, b4 = (e4 & 31) * 4;
    if (ROWMAJ) {
      float* d = sF + a * 129 + b4;
      d[0] = v[j].x; d[1] = v[j].y; d[2] = v[j].z; d[3] = v[j].w;
    } else {
      float* d = sF + b4 * 129 + a;
      d[0] = v[j].x; d[129] = v[j].y; d[258] = v[j].z; d[387] = v[j].w;
    }
  }
}
// acc(a, b) += sum_{k < kn} sF(rg + 32 a, k) sX(k, 4 cg + b): lane rg takes
// rows rg, rg+32, rg+64, rg+96 (conflict-free scalar reads of sF, stride
// 129), warp cg takes right-hand sides 4cg..4cg+3 (one broadcast float4 of
// sX per k): 16 FMAs per 5 shared loads.
__device__ __forceinline__ void block_fma(const float* sF, const float (*sX)[36], int kn, int rg, int cg,
                                          float (&acc)[4][4]) {
#pragma unroll 8
  for (int k = 0; k < kn; ++k) {
    const float4 x = *reinterpret_cast<const float4*>(&sX[k][4 * cg]);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const float f = sF[(rg + 32 * a) * 129 + k];
      acc[a][0] = fmaf(f, x.x, acc[a][0]);
      acc[a][1] = fmaf(f, x.y, acc[a][1]);
      acc[a][2] = fmaf(f, x.z, acc[a][2]);
      acc[a][3] = fmaf(f, x.w, acc[a][3]);
    }
  }
}

constexpr int SOLVE_SMEM = (128 * 36 + 128 * 129) * 4;

__device__ __forceinline__ int ld_acquire_flag(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_flag(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Whole blocked triangular sweep in one cooperative launch (FP32, nr <= 32
// right-hand sides, 128-row blocks):
//   X_i := op(Inv_i) (Y_i - sum_j op(F)(block i, block j) X_j)
// over the blocks j solved before i (j < i forward, j > i backward).  CTA g
// owns the blocks solved g-th, (g + G)-th, ... (G = gridDim.x).  For block i,
// whose predecessor in solve order is p (i - 1 forward, i + 1 backward):
//   Z_i := op(Inv_i) (Y_i - sum_{j before p} op(F)(i, j) X_j)
// is formed while p is still being solved (the contributions are taken as
// the blocks are published), and once p is published only
//   X_i := Z_i - W_i X_p,   W_i = op(Inv_i) op(F)(i, p)
// (W precomputed per factorization, sweep_couplings) remains on the critical
// path: one block product per block of the chain.  A block is published by
// its X stores, a fence, and flags[i] := epoch.  Every block depends only on
// blocks solved earlier and every CTA takes its blocks in solve order, so
// with all CTAs resident (cooperative launch) the sweep cannot deadlock; each
// wait is bounded.  X blocks of other CTAs are read through L2
// (ld.global.cg): they were written during this launch.
// op(Inv)(i, k) = Inv[k + i * 128] when TI (else Inv[i + k * 128]);
// op(F)(r, c) = F[c + r * ldf] when TF (else F[r + c * ldf]); W_i(r, c) at
// W[i * 128 * 128 + r + c * 128].
template <bool TI, bool TF, bool BWD>
__global__ void __launch_bounds__(256) solve_sweep_kernel(const float* __restrict__ F, long ldf,
                                                          const float* __restrict__ Inv,
                                                          const float* __restrict__ W, float* X,
                                                          const float* __restrict__ Y, long ldy, int n, int nr,
                                                          int nblk, int* flags, int epoch, int* err) {
  extern __shared__ __align__(16) float sm_solve[];
  float (*sX)[36] = reinterpret_cast<float (*)[36]>(sm_solve);
  float* sF = sm_solve + 128 * 36;
  __shared__ int s_ok;
  const int tid = threadIdx.x;
  const int rg = tid & 31, cg = tid >> 5;
  // wait (thread 0, bounded) until block bj is published; CTA-uniform result
  auto wait_block = [&](int bj) -> bool {
    if (tid == 0) {
      int ok = 1;
      if (ld_acquire_flag(flags + bj) < epoch) {
        const unsigned long long t0 = globaltimer_ns();
        while (ld_acquire_flag(flags + bj) < epoch) {
          if (*((volatile int*)err) != 0 || globaltimer_ns() - t0 > kWaitLimitNs) {
            atomicExch(err, 51);
            ok = 0;
            break;
          }
        }
      }
      s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
  };
  auto load_x = [&](int c0, int w) {
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      const int e = tid + j * 256;
      const int k = e & 127, c = e >> 7;
      sX[k][c] = (k < w && c < nr) ? __ldcg(X + (long)(c0 + k) + (long)c * ldy) : 0.f;
    }
  };
  for (int q = blockIdx.x; q < nblk; q += gridDim.x) {
    const int bi = BWD ? nblk - 1 - q : q;
    const int r0 = bi * 128, wn = min(128, n - r0);
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
    float4 v[16];
    for (int t = 0; t + 1 < q; ++t) {
      const int bj = BWD ? nblk - 1 - t : t;
      const int c0 = bj * 128, w = min(128, n - c0);
      block_load<TF>(TF ? F + c0 + (long)r0 * ldf : F + r0 + (long)c0 * ldf, ldf, wn, w, v);
      if (!wait_block(bj)) return;
      load_x(c0, w);
      block_store<TF>(sF, v);
      __syncthreads();
      block_fma(sF, sX, w, rg, cg, acc);
      __syncthreads();
    }
    // Z_i := op(Inv_i) (Y_i - acc)
    block_load<TI>(Inv + (long)bi * 128 * 128, 128, wn, wn, v);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = rg + 32 * a;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int c = 4 * cg + b;
        sX[i][c] = (i < wn && c < nr) ? Y[(long)(r0 + i) + (long)c * ldy] - acc[a][b] : 0.f;
        acc[a][b] = 0.f;
      }
    }
    block_store<TI>(sF, v);
    __syncthreads();
    block_fma(sF, sX, wn, rg, cg, acc);
    if (q > 0) {
      // X_i := Z_i - W_i X_p once the predecessor p is published
      const int bp = BWD ? bi + 1 : bi - 1;
      const int c0 = bp * 128, w = min(128, n - c0);
      block_load<false>(W + (long)bi * 128 * 128, 128, wn, w, v);
      __syncthreads();
      if (!wait_block(bp)) return;
      load_x(c0, w);
      block_store<false>(sF, v);
      __syncthreads();
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = -acc[a][b];
      block_fma(sF, sX, w, rg, cg, acc);  // acc = W X_p - Z
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = -acc[a][b];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = rg + 32 * a;
      if (i < wn)
#pragma unroll
        for (int b = 0; b < 4; ++b)
          if (4 * cg + b < nr) __stcg(X + (long)(r0 + i) + (long)(4 * cg + b) * ldy, acc[a][b]);
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) st_release_flag(flags + bi, epoch);
  }
}

// Coupling blocks of the sweeps: W_i = op(Inv_i) op(F)(block i, block p),
// p the block solved just before i (i - 1 forward, i + 1 backward), one CTA
// per block, four 32-column passes of the 128 x 128 x 128 product; W_i(r, c)
// at W[i * 128 * 128 + r + c * 128].
template <bool TI, bool TF, bool BWD>
__global__ void __launch_bounds__(256) sweep_coupling_kernel(const float* __restrict__ F, long ldf,
                                                             const float* __restrict__ Inv, float* __restrict__ W,
                                                             int n, int nblk) {
  extern __shared__ __align__(16) float sm_solve[];
  float (*sX)[36] = reinterpret_cast<float (*)[36]>(sm_solve);
  float* sF = sm_solve + 128 * 36;
  const int bi = blockIdx.x;
  const int bp = BWD ? bi + 1 : bi - 1;
  if (bp < 0 || bp >= nblk) return;
  const int tid = threadIdx.x, rg = tid & 31, cg = tid >> 5;
  const int r0 = bi * 128, wn = min(128, n - r0), c0 = bp * 128, w = min(128, n - c0);
  float4 v[16];
  block_load<TI>(Inv + (long)bi * 128 * 128, 128, wn, wn, v);
  block_store<TI>(sF, v);
  for (int pc = 0; pc < 4; ++pc) {
    // sX(k, c) = op(F)(r0 + k, c0 + 32 pc + c)
    for (int e = tid; e < 128 * 32; e += 256) {
      const int k = e & 127, c = e >> 7;
      const int col = 32 * pc + c;
      sX[k][c] = (k < wn && col < w) ? (TF ? F[(c0 + col) + (long)(r0 + k) * ldf] : F[(r0 + k) + (long)(c0 + col) * ldf])
                                     : 0.f;
    }
    __syncthreads();
    float acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.f;
    block_fma(sF, sX, wn, rg, cg, acc);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = rg + 32 * a;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int c = 32 * pc + 4 * cg + b;
        W[(long)bi * 128 * 128 + i + c * 128] = (i < wn && c < w) ? acc[a][b] : 0.f;
      }
    }
    __syncthreads();
  }
}

inline int grid_for(long total) { return (int)std::min<long>(8192, (total + 255) / 256); }

}  // namespace

// ===========================================================================
// Low-precision factorizations
// ===========================================================================
namespace {

struct LpWork {
  uint16_t* PA = nullptr;   // packed A-operand (n x MB)
  uint16_t* PB = nullptr;   // packed B-operand (n x MB)
  uint16_t* PC = nullptr;   // packed operand of the side stream (n x MB)
  uint16_t* PX = nullptr;   // packed inverse block (MB x MB)
  uint16_t* PD = nullptr;   // Cholesky: packed sub-panel of the side stream (n x MB)
  uint16_t* PW[2] = {nullptr, nullptr};  // Cholesky: packed outer panels (n x NBO), ping-pong
  long plane = 0, planeX = 0;  // lo-plane offsets (LP_TF32X3: floats; LP_FP16X3: 16-bit elements)
  long planeW = 0;
  double* P64 = nullptr;    // FP64 panel (MB x n); Cholesky: the FP64 diagonal
                            // factors, block q at q MB (MB + 1), ld MB
  double* X64 = nullptr;    // FP64 inverse blocks (2 x MB x MB)
  double* Xall = nullptr;   // Cholesky: inverses of all diagonal factors (q MB MB)
};

int lp_workspace(long n, LpFactor* f, LpWork* w) {
  const size_t np = (size_t)std::max<long>(n, 1);
  f->ldf = (n + 3) & ~3L;
  f->F = (float*)ws_get(WS_LP0, sizeof(float) * (size_t)f->ldf * np);
  const size_t pk = lp_packed_bytes(LP_TF32X3, (long)np, MB), px = lp_packed_bytes(LP_TF32X3, MB, MB);
  const size_t pw = lp_packed_bytes(LP_TF32X3, (long)np, NBO);
  char* p16 = (char*)ws_get(WS_LP1, 4 * pk + px + 2 * pw + 4096);
  const size_t p64n = (size_t)(MB + 1) * (np + MB);  // P64 in either use
  char* p64 = (char*)ws_get(WS_LP3, sizeof(double) * (p64n + 2 * (size_t)MB * MB + (size_t)MB * (np + MB)) + 1024);
  const long nblk = (n + MB - 1) / MB;
  char* pinv = (char*)ws_get(WS_LP4, sizeof(float) * 2 * (size_t)nblk * MB * MB + sizeof(double) * 2 * np +
                                         sizeof(int) * 2 * np + 1024);
  if (!f->F || !p16 || !p64 || !pinv) return FLA_FAILURE;
  w->PD = (uint16_t*)(p16 + 3 * pk + px);
  w->PW[0] = (uint16_t*)(p16 + 4 * pk + px);
  w->PW[1] = (uint16_t*)(p16 + 4 * pk + px + pw);
  w->planeW = (long)NBO * (long)np;
  w->PA = (uint16_t*)p16;
  w->PB = (uint16_t*)(p16 + pk);
  w->PC = (uint16_t*)(p16 + 2 * pk);
  w->PX = (uint16_t*)(p16 + 3 * pk);
  w->plane = (long)MB * (long)np;
  w->planeX = (long)MB * MB;
  w->P64 = (double*)p64;
  w->X64 = w->P64 + p64n;
  w->Xall = w->X64 + 2 * (size_t)MB * MB;
  f->inv1 = (float*)pinv;
  f->inv2 = f->inv1 + (size_t)nblk * MB * MB;
  f->sr = (double*)(f->inv2 + (size_t)nblk * MB * MB);
  f->sc = f->sr + np;
  f->piv = (int*)(f->sc + np);
  f->perm = f->piv + np;
  f->n = n;
  return FLA_SUCCESS;
}

}  // namespace

// Coupling blocks of both correction sweeps for the current factors (see
// solve_sweep_kernel), one launch per direction.
int lp_couplings(LpFactor* f, cudaStream_t st) {
  const long n = f->n;
  const long nblk = (n + MB - 1) / MB;
  float* w = (float*)ws_get(WS_LP5, sizeof(float) * 2 * (size_t)std::max<long>(nblk, 1) * MB * MB);
  if (!w) return FLA_FAILURE;
  f->wf = w;
  f->wb = w + (size_t)nblk * MB * MB;
  static bool attr = false;
  if (!attr) {
    FB_CK(cudaFuncSetAttribute(sweep_coupling_kernel<false, false, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, SOLVE_SMEM));
    FB_CK(cudaFuncSetAttribute(sweep_coupling_kernel<true, true, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, SOLVE_SMEM));
    FB_CK(cudaFuncSetAttribute(sweep_coupling_kernel<true, true, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, SOLVE_SMEM));
    attr = true;
  }
  if (f->chol)
    sweep_coupling_kernel<false, false, false><<<(unsigned)nblk, 256, SOLVE_SMEM, st>>>(f->F, f->ldf, f->inv1,
                                                                                        f->wf, (int)n, (int)nblk);
  else
    sweep_coupling_kernel<true, true, false><<<(unsigned)nblk, 256, SOLVE_SMEM, st>>>(f->F, f->ldf, f->inv1, f->wf,
                                                                                      (int)n, (int)nblk);
  sweep_coupling_kernel<true, true, true><<<(unsigned)nblk, 256, SOLVE_SMEM, st>>>(
      f->F, f->ldf, f->chol ? f->inv1 : f->inv2, f->wb, (int)n, (int)nblk);
  count_launch(2);
  FB_CK(cudaGetLastError());
  f->coupled = true;
  return FLA_SUCCESS;
}

// LU with partial pivoting of (diag(sr) A diag(sc)) in low precision, on the
// transposed FP32 copy F = (scaled A)^T (n x n, ld ldf): the layout and the
// step structure of the FP64 driver (lu_piv_dev), with every trailing update
// and panel solve a 16-bit tensor-core GEMM.
int lp_lu_factor(DMat A, LowPrec prec, bool scale, LpFactor* f) {
  Context& cx = ctx();
  cudaStream_t st = cx.stream, sd = cx.side;
  const long n = A.m;
  LpWork w;
  if (lp_workspace(n, f, &w) != FLA_SUCCESS) return FLA_FAILURE;
  f->chol = false;
  f->prec = prec;
  f->scaled = scale;
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;
  if (scale) {
    row_absmax_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A.p, A.ld, (int)n, (int)n, nullptr, f->sr);
    pow2_recip_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(f->sr, (int)n, 0);
    col_absmax_kernel<<<(unsigned)n, 256, 0, st>>>(A.p, A.ld, (int)n, f->sr, f->sc);
    pow2_recip_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(f->sc, (int)n, 0);
    count_launch(4);
  }
  {
    dim3 grid((unsigned)((n + 31) / 32), (unsigned)((n + 31) / 32)), block(32, 8);
    transpose_scale_kernel<<<grid, block, 0, st>>>(A.p, A.ld, f->F, f->ldf, (int)n, (int)n, scale ? f->sr : nullptr,
                                                   scale ? f->sc : nullptr);
    count_launch();
    FB_CK(cudaGetLastError());
  }
  float* F = f->F;
  const long ldf = f->ldf;
  auto at = [&](long i, long j) { return F + j + i * ldf; };  // element (i, j) of the scaled A
  const long ldp = MB;
  double* X64 = w.X64;                  // inv(L11^T)
  double* Y64 = w.X64 + (size_t)MB * MB;  // inv(U11^T)

  // panel k: FP64 copy, factor, round back, the two inverse triangles
  auto panel = [&](long k, cudaStream_t s) -> int {
    const int b = (int)std::min<long>(MB, n - k);
    const long M = n - k;
    const long kb = k / MB;
    if (convert2d<double, float>(s, at(k, k), ldf, w.P64, ldp, b, M) != FLA_SUCCESS) return FLA_FAILURE;
    if (lu_panel_factor_t(w.P64, ldp, M, b, f->piv + k, (int)k, s) != FLA_SUCCESS) return FLA_FAILURE;
    if (convert2d<float, double>(s, w.P64, ldp, at(k, k), ldf, b, M) != FLA_SUCCESS) return FLA_FAILURE;
    if (tri_inverse(w.P64, ldp, b, false, true, X64, MB, s) != FLA_SUCCESS) return FLA_FAILURE;
    if (tri_inverse(w.P64, ldp, b, true, false, Y64, MB, s) != FLA_SUCCESS) return FLA_FAILURE;
    if (convert2d<float, double>(s, X64, MB, f->inv1 + kb * MB * MB, MB, b, b) != FLA_SUCCESS) return FLA_FAILURE;
    if (convert2d<float, double>(s, Y64, MB, f->inv2 + kb * MB * MB, MB, b, b) != FLA_SUCCESS) return FLA_FAILURE;
    // B operand of U12^T := A12^T inv(L11^T): B(j, kk) = X64(kk, j)
    return pack16<double>(s, prec, X64, MB, 1, w.PX, MB, b, b, 1.f, w.planeX);
  };

  cudaEvent_t ev_look = cx.ev[0], ev_panel = cx.ev[1];
  if (panel(0, st) != FLA_SUCCESS) return FLA_FAILURE;
  for (long k = 0; k < n; k += MB) {
    const int b = (int)std::min<long>(MB, n - k);
    const long nr = n - k - b;
    if (laswp_t_f32(F, ldf, (int)k, f->piv + k, b, 0, (int)k, (int)(k + b), (int)nr, st) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (nr <= 0) continue;
    // U12^T := A12^T inv(L11^T); A12^T(i, kk) = at(k + kk, k + b + i)
    if (pack16<float>(st, prec, at(k, k + b), 1, ldf, w.PA, MB, nr, b, 1.f, w.plane) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (lp_gemm(st, prec, nr, b, b, 1.f, w.PA, MB, w.PX, MB, 0.f, at(k, k + b), ldf, GEMM_FULL, 0, nullptr, INT_MAX,
                w.plane, w.planeX) != FLA_SUCCESS)
      return FLA_FAILURE;
    // trailing update  A22^T -= U12^T A21^T
    if (pack16<float>(st, prec, at(k, k + b), 1, ldf, w.PA, MB, nr, b, 1.f, w.plane) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (pack16<float>(st, prec, at(k + b, k), ldf, 1, w.PB, MB, nr, b, 1.f, w.plane) != FLA_SUCCESS)
      return FLA_FAILURE;
    const int nb2 = (int)std::min<long>(MB, nr);
    if (lp_gemm(st, prec, nb2, nr, b, -1.f, w.PA, MB, w.PB, MB, 1.f, at(k + b, k + b), ldf, GEMM_FULL, 0, nullptr,
                INT_MAX, w.plane, w.plane) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_look, st));
    FB_CK(cudaStreamWaitEvent(sd, ev_look, 0));
    if (panel(k + b, sd) != FLA_SUCCESS) return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_panel, sd));
    if (nr > nb2 && lp_gemm(st, prec, nr - nb2, nr, b, -1.f, lp_off(w.PA, prec, (size_t)nb2 * MB), MB, w.PB, MB,
                            1.f, at(k + b, k + b + nb2), ldf, GEMM_FULL, 0, nullptr, INT_MAX, w.plane,
                            w.plane) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaStreamWaitEvent(st, ev_panel, 0));
  }
  {
    const size_t sbytes = sizeof(int) * (size_t)n;
    const bool smem = sbytes <= 200 * 1024;
    if (smem) cudaFuncSetAttribute(perm_from_pivots_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    perm_from_pivots_kernel<<<1, 1024, smem ? sbytes : 0, st>>>(f->piv, (int)n, f->perm, smem ? 1 : 0);
    count_launch();
    FB_CK(cudaGetLastError());
  }
  if (lp_couplings(f, st) != FLA_SUCCESS) return FLA_FAILURE;
  int info = -1;
  if (status_read(&info) != FLA_SUCCESS) return FLA_FAILURE;
  f->info = info;
  return FLA_SUCCESS;
}

// Cholesky of diag(d) A diag(d) in low precision; F holds L (lower, FP32).
// The structure of the FP64 driver (chol_lower_enqueue): outer panels of
// NBO = 256 columns, each factored as two 128-column sub-panels on the
// second stream (FP64 diagonal block and its inverse, A21 := A21 inv(L11)^T
// as a tensor-core GEMM, the panel's later columns updated by the first
// sub-panel), then packed once into the K-major operand buffer of the
// updates (two buffers used in turn, so packing the next panel never
// overwrites the operand of an update still running); the main stream
// updates the next panel's columns first (K = 256), then the rest of the
// trailing matrix, beside the next panel.
int lp_chol_factor_shift(DMat A, bool upper, LowPrec prec, bool scale, double sigma, LpFactor* f) {
  Context& cx = ctx();
  cudaStream_t st = cx.stream, sd = cx.side;
  const long n = A.m;
  LpWork w;
  if (lp_workspace(n, f, &w) != FLA_SUCCESS) return FLA_FAILURE;
  f->chol = true;
  f->prec = prec;
  f->scaled = scale;
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;
  if (scale) {
    diag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A.p, A.ld, (int)n, f->sr);
    pow2_recip_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(f->sr, (int)n, 1);
    count_launch(2);
    FB_CK(cudaMemcpyAsync(f->sc, f->sr, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
  }
  lower_scale_kernel<<<grid_for(n * n), 256, 0, st>>>(A.p, A.ld, f->F, f->ldf, (int)n, scale ? f->sr : nullptr,
                                                      upper ? 1 : 0, sigma);
  count_launch();
  FB_CK(cudaGetLastError());
  float* F = f->F;
  const long ldf = f->ldf;
  int* info = cx.d_status + ST_INFO;
  auto at = [&](long i, long j) { return F + i + j * ldf; };

  // 128-column sub-panel at column j: diagonal block in FP64 (kept, in the
  // diagonal layout of P64, for the correction sweeps' inverses), then
  // A21 := A21 inv(L11)^T by forward substitution in FP64 in one launch
  // (rather than the inverse, two 16-bit packings and a tensor-core
  // product on the panel's critical chain)
  auto sub = [&](long j, cudaStream_t s) -> int {
    const int b = (int)std::min<long>(MB, n - j);
    double* L64 = w.P64 + (j / MB) * (long)MB * (MB + 1);
    if (convert2d<double, float>(s, at(j, j), ldf, L64, MB, b, b) != FLA_SUCCESS) return FLA_FAILURE;
    if (potrf_diag_dev(L64, MB, b, (int)j, s) != FLA_SUCCESS) return FLA_FAILURE;
    if (convert2d<float, double>(s, L64, MB, at(j, j), ldf, b, b) != FLA_SUCCESS) return FLA_FAILURE;
    const long m2 = n - j - b;
    if (m2 <= 0) return FLA_SUCCESS;
    return trsm_rlt_subst_f32(L64, MB, at(j + b, j), ldf, b, m2, info, (int)(j + b), s);
  };
  // Outer panel at column k: its sub-panels, the first one updating the
  // second's columns, then the rows below the panel packed into PW.
  auto panel = [&](long k, cudaStream_t s) -> int {
    const long kend = std::min<long>(n, k + NBO);
    for (long j = k; j < kend; j += MB) {
      if (sub(j, s) != FLA_SUCCESS) return FLA_FAILURE;
      const long j2 = j + std::min<long>(MB, n - j);
      if (j2 >= kend) break;
      if (pack16<float>(s, prec, at(j2, j), 1, ldf, w.PD, MB, n - j2, j2 - j, 1.f, w.plane) != FLA_SUCCESS)
        return FLA_FAILURE;
      if (lp_gemm(s, prec, n - j2, kend - j2, j2 - j, -1.f, w.PD, MB, w.PD, MB, 1.f, at(j2, j2), ldf, GEMM_LOWER, 0,
                  info, (int)j2, w.plane, w.plane) != FLA_SUCCESS)
        return FLA_FAILURE;
    }
    if (n > kend)
      return pack16<float>(s, prec, at(kend, k), 1, ldf, w.PW[(k / NBO) & 1], NBO, n - kend, kend - k, 1.f,
                           w.planeW);
    return FLA_SUCCESS;
  };

  cudaEvent_t ev_look = cx.ev[2], ev_panel = cx.ev[3];
  if (panel(0, st) != FLA_SUCCESS) return FLA_FAILURE;
  for (long k = 0; k < n; k += NBO) {
    const int b = (int)std::min<long>(NBO, n - k);
    const long m2 = n - k - b;
    if (m2 <= 0) break;
    const int lim = (int)(k + b);
    const int nb2 = (int)std::min<long>(NBO, m2);
    uint16_t* P = w.PW[(k / NBO) & 1];
    if (lp_gemm(st, prec, m2, nb2, b, -1.f, P, NBO, P, NBO, 1.f, at(k + b, k + b), ldf, GEMM_LOWER, 0, info, lim,
                w.planeW, w.planeW) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_look, st));
    FB_CK(cudaStreamWaitEvent(sd, ev_look, 0));
    if (panel(k + b, sd) != FLA_SUCCESS) return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_panel, sd));
    if (m2 > nb2 && lp_gemm(st, prec, m2 - nb2, m2 - nb2, b, -1.f, lp_off(P, prec, (size_t)nb2 * NBO), NBO,
                            lp_off(P, prec, (size_t)nb2 * NBO), NBO, 1.f, at(k + b + nb2, k + b + nb2), ldf,
                            GEMM_LOWER, 0, info, lim, w.planeW, w.planeW) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaStreamWaitEvent(st, ev_panel, 0));
  }
  // inverses of every diagonal factor for the correction sweeps, in one
  // launch off the factorization's chain, rounded to FP32
  const long nblk = (n + MB - 1) / MB;
  if (tri_inverse_blocks(w.P64, MB, n, true, false, w.Xall, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (convert2d<float, double>(st, w.Xall, MB, f->inv1, MB, MB, nblk * MB) != FLA_SUCCESS) return FLA_FAILURE;
  if (lp_couplings(f, st) != FLA_SUCCESS) return FLA_FAILURE;
  int inf = -1;
  if (status_read(&inf) != FLA_SUCCESS) return FLA_FAILURE;
  f->info = inf;
  return FLA_SUCCESS;
}

// Cholesky in low precision; when the 16-bit factorization breaks down
// (the rounding perturbs an ill-conditioned matrix out of the SPD cone),
// retry on the shifted diag(d) A diag(d) + sigma I with sigma = 2u, 8u, 32u,
// 128u (u the unit roundoff of the 16-bit format): the factors then
// precondition a nearby matrix and GMRES-IR restores the solution of A.
int lp_chol_factor(DMat A, bool upper, LowPrec prec, bool scale, LpFactor* f) {
  if (lp_chol_factor_shift(A, upper, prec, scale, 0.0, f) != FLA_SUCCESS) return FLA_FAILURE;
  const double u = prec == LP_FP16 ? std::ldexp(1.0, -11) : prec == LP_BF16 ? std::ldexp(1.0, -8) : std::ldexp(1.0, -21);
  // (LP_TF32X3 and LP_FP16X3 are FP32-accurate: 2^-21)
  for (int t = 0; t < 4 && f->info >= 0 && scale; ++t) {
    const double sigma = u * std::ldexp(1.0, 2 * t + 1);
    if (lp_chol_factor_shift(A, upper, prec, scale, sigma, f) != FLA_SUCCESS) return FLA_FAILURE;
    f->shift = sigma;
  }
  return FLA_SUCCESS;
}

// One triangular sweep of the correction solve in a single cooperative
// launch (solve_sweep_kernel): forward (L y = rhs) or backward (L^T x = y,
// U x = y).  The ready flags live in a workspace slot that is zeroed when it
// is (re)allocated; each sweep publishes a new epoch, so no reset is needed
// between sweeps.
int sweep(const LpFactor& f, const float* Yin, float* Xout, long n, long nrhs, bool backward, cudaStream_t st) {
  static void* last_flags = nullptr;
  static int epoch = 0;
  static int max_ctas = 0;
  const long nblk = (n + MB - 1) / MB;
  int* flags = (int*)ws_get(WS_SWEEP, sizeof(int) * (size_t)std::max<long>(nblk, 1024));
  if (!flags) return FLA_FAILURE;
  if (flags != last_flags) {
    FB_CK(cudaMemsetAsync(flags, 0, sizeof(int) * (size_t)std::max<long>(nblk, 1024), st));
    last_flags = flags;
    epoch = 0;
  }
  ++epoch;
  if (max_ctas == 0) {
    FB_CK(cudaFuncSetAttribute(solve_sweep_kernel<true, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               SOLVE_SMEM));
    FB_CK(cudaFuncSetAttribute(solve_sweep_kernel<false, false, false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize, SOLVE_SMEM));
    FB_CK(cudaFuncSetAttribute(solve_sweep_kernel<true, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               SOLVE_SMEM));
    int per_sm = 0;
    FB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, solve_sweep_kernel<true, true, true>, 256,
                                                        SOLVE_SMEM));
    max_ctas = std::max(1, per_sm) * ctx().num_sms;
  }
  const int G = (int)std::min<long>(nblk, max_ctas);
  const float* F = f.F;
  long ldf = f.ldf;
  const float* inv = backward ? (f.chol ? f.inv1 : f.inv2) : f.inv1;
  const float* Wc = backward ? f.wb : f.wf;
  float* X = Xout;
  const float* Y = Yin;
  long ldy = n;
  int ni = (int)n, nr = (int)nrhs, nb = (int)nblk, ep = epoch;
  int* err = ctx().d_status + ST_ERROR;
  void* args[] = {(void*)&F, (void*)&ldf, (void*)&inv, (void*)&Wc, (void*)&X, (void*)&Y, (void*)&ldy,
                  (void*)&ni, (void*)&nr, (void*)&nb, (void*)&flags, (void*)&ep, (void*)&err};
  void* fn;
  if (backward) fn = (void*)solve_sweep_kernel<true, true, true>;
  else fn = f.chol ? (void*)solve_sweep_kernel<false, false, false> : (void*)solve_sweep_kernel<true, true, false>;
  const int ps = prof_begin(st);
  FB_CK(cudaLaunchCooperativeKernel(fn, dim3(G), dim3(256), args, SOLVE_SMEM, st));
  prof_end(ps, st, PROF_TRSM, (double)n * (double)n * (double)nrhs);
  count_launch();
  return FLA_SUCCESS;
}

// ===========================================================================
// Correction solve with the low-precision factors: D := M^-1 R (FP64 in and
// out, FP32 inside).  T is an FP32 n x nrhs workspace, ld n.
// ===========================================================================
int lp_solve(const LpFactor& f, const double* R, long ldr, double* D, long ldd, long nrhs, float* T, float* Tb,
             cudaStream_t st) {
  const long n = f.n;
  const long nblk = (n + MB - 1) / MB;
  const float* F = f.F;
  const long ldf = f.ldf;
  // T := scale * R, rows permuted (LU)
  if (!f.chol) {
    gather_rows_kernel<<<grid_for(n * nrhs), 256, 0, st>>>(R, ldr, f.perm, f.scaled ? f.sr : nullptr, T, n, (int)n,
                                                           (int)nrhs);
  } else {
    scale_copy_kernel<float, double><<<grid_for(n * nrhs), 256, 0, st>>>(R, ldr, T, n, (int)n, (int)nrhs,
                                                                        f.scaled ? f.sr : nullptr);
  }
  count_launch();
  // Forward sweep L y = T (T -> Tb), backward sweep U x = y or L^T x = y
  // (Tb -> T): one cooperative launch each while nrhs <= 32.
  if (nrhs <= 32) {
    if (sweep(f, T, Tb, n, nrhs, false, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (sweep(f, Tb, T, n, nrhs, true, st) != FLA_SUCCESS) return FLA_FAILURE;
  } else {
    // wide right-hand sides: sgemm per block
    for (long kb = 0; kb < nblk; ++kb) {
      const long k = kb * MB;
      const int b = (int)std::min<long>(MB, n - k);
      const long rest = n - k - b;
      const float* inv = f.inv1 + kb * MB * MB;
      if (sgemm(st, !f.chol, false, b, nrhs, b, 1.f, inv, MB, T + k, n, 0.f, Tb, MB) != FLA_SUCCESS) return FLA_FAILURE;
      FB_CK(cudaMemcpy2DAsync(T + k, sizeof(float) * n, Tb, sizeof(float) * MB, sizeof(float) * b, nrhs,
                              cudaMemcpyDeviceToDevice, st));
      if (rest > 0) {
        if (!f.chol) {
          if (sgemm(st, true, false, rest, nrhs, b, -1.f, F + k + (k + b) * ldf, ldf, Tb, MB, 1.f, T + k + b, n) !=
              FLA_SUCCESS)
            return FLA_FAILURE;
        } else {
          if (sgemm(st, false, false, rest, nrhs, b, -1.f, F + (k + b) + k * ldf, ldf, Tb, MB, 1.f, T + k + b, n) !=
              FLA_SUCCESS)
            return FLA_FAILURE;
        }
      }
    }
    for (long kb = nblk - 1; kb >= 0; --kb) {
      const long k = kb * MB;
      const int b = (int)std::min<long>(MB, n - k);
      const float* inv = f.chol ? f.inv1 + kb * MB * MB : f.inv2 + kb * MB * MB;
      if (sgemm(st, true, false, b, nrhs, b, 1.f, inv, MB, T + k, n, 0.f, Tb, MB) != FLA_SUCCESS) return FLA_FAILURE;
      FB_CK(cudaMemcpy2DAsync(T + k, sizeof(float) * n, Tb, sizeof(float) * MB, sizeof(float) * b, nrhs,
                              cudaMemcpyDeviceToDevice, st));
      if (k > 0) {
        if (sgemm(st, true, false, k, nrhs, b, -1.f, F + k, ldf, Tb, MB, 1.f, T, n) != FLA_SUCCESS) return FLA_FAILURE;
      }
    }
  }
  scale_copy_kernel<double, float><<<grid_for(n * nrhs), 256, 0, st>>>(T, n, D, ldd, (int)n, (int)nrhs,
                                                                      f.scaled ? f.sc : nullptr);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// ===========================================================================
// Refinement
// ===========================================================================
namespace {

struct IrBuffers {
  double* R = nullptr;    // residual n x nrhs
  double* D = nullptr;    // correction
  double* R64 = nullptr;  // A V_j in GMRES
  float* T = nullptr;     // FP32 right-hand sides
  float* Tb = nullptr;    // FP32 block scratch (MB x nrhs)
  double* V = nullptr;    // GMRES basis (m + 1) x n x nrhs
  double* W = nullptr;    // GMRES work vector block
  double* small = nullptr;  // device: dots and norms
  double* h_small = nullptr;
};

// R := B - A X (FP64 DMMA GEMM)
int residual(const DMat& A, const DMat& B, const double* X, long ldx, double* R, long ldr, long nrhs,
             cudaStream_t st) {
  const long n = A.m;
  FB_CK(cudaMemcpy2DAsync(R, sizeof(double) * ldr, B.p, sizeof(double) * B.ld, sizeof(double) * n, nrhs,
                          cudaMemcpyDeviceToDevice, st));
  return gemm_f64(st, false, false, n, nrhs, n, -1.0, A.p, A.ld, X, ldx, 1.0, R, ldr);
}

// max-abs per column of X and R on the host; true when every column has
// ||r||_inf <= ||x||_inf * cte (dsgesv.c:330-334)
int converged(const double* X, long ldx, const double* R, long ldr, long n, long nrhs, double cte, IrBuffers& b,
              cudaStream_t st, bool* ok) {
  colmax_kernel<<<(unsigned)nrhs, 256, 0, st>>>(X, ldx, (int)n, b.small);
  colmax_kernel<<<(unsigned)nrhs, 256, 0, st>>>(R, ldr, (int)n, b.small + nrhs);
  count_launch(2);
  FB_CK(cudaMemcpyAsync(b.h_small, b.small, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, st));
  FB_CK(cudaStreamSynchronize(st));
  *ok = true;
  for (long c = 0; c < nrhs; ++c)
    if (!(b.h_small[nrhs + c] <= b.h_small[c] * cte)) *ok = false;
  return FLA_SUCCESS;
}

// GMRES(m), left-preconditioned by the low-precision factors, all columns in
// lockstep: D ~= A^-1 R.  Classical Gram-Schmidt applied twice per step.
int gmres(const DMat& A, const LpFactor& f, const double* R, double* D, long nrhs, int m, double tol, IrBuffers& b,
          cudaStream_t st, int* iters) {
  const long n = A.m;
  const long ld = (n + 1) & ~1L;  // 16-byte leading dimensions for the GEMM engine
  const long vstride = ld * nrhs;
  double* V = b.V;
  double* W = b.W;
  double* dev = b.small;         // device scratch: (m + 1) x nrhs dots, nrhs norms
  double* host = b.h_small;
  // V0 = M^-1 R, beta = ||V0||
  if (lp_solve(f, R, ld, V, ld, nrhs, b.T, b.Tb, st) != FLA_SUCCESS) return FLA_FAILURE;
  coldots_kernel<<<dim3((unsigned)nrhs, 1), 256, 0, st>>>(V, 0, V, ld, (int)n, 1, dev);
  count_launch();
  FB_CK(cudaMemcpyAsync(host, dev, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
  FB_CK(cudaStreamSynchronize(st));
  std::vector<double> beta(nrhs), inv(nrhs);
  for (long c = 0; c < nrhs; ++c) {
    beta[c] = std::sqrt(std::max(0.0, host[c]));
    inv[c] = beta[c] > 0 ? 1.0 / beta[c] : 0.0;
  }
  FB_CK(cudaMemcpyAsync(dev, inv.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, st));
  colscale_kernel<<<grid_for(n * nrhs), 256, 0, st>>>(V, V, ld, (int)n, (int)nrhs, dev);
  count_launch();
  // Hessenberg, Givens rotations and right-hand side per column (host)
  std::vector<double> H((size_t)(m + 1) * m * nrhs, 0.0), cs((size_t)m * nrhs), sn((size_t)m * nrhs),
      g((size_t)(m + 1) * nrhs, 0.0);
  for (long c = 0; c < nrhs; ++c) g[c * (m + 1)] = beta[c];
  auto Hc = [&](long c, int i, int j) -> double& { return H[(size_t)c * (m + 1) * m + i + (size_t)j * (m + 1)]; };
  int jdone = 0;
  std::vector<double> hbuf((size_t)(m + 1) * nrhs), hbuf2((size_t)(m + 1) * nrhs);
  for (int j = 0; j < m; ++j) {
    double* Vj = V + j * vstride;
    // W = M^-1 (A Vj)
    if (gemm_f64(st, false, false, n, nrhs, n, 1.0, A.p, A.ld, Vj, ld, 0.0, b.R64, ld) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (lp_solve(f, b.R64, ld, W, ld, nrhs, b.T, b.Tb, st) != FLA_SUCCESS) return FLA_FAILURE;
    // two passes of classical Gram-Schmidt against V0..Vj
    const int nv = j + 1;
    for (int pass = 0; pass < 2; ++pass) {
      coldots_kernel<<<dim3((unsigned)nrhs, (unsigned)nv), 256, 0, st>>>(V, vstride, W, ld, (int)n, nv, dev);
      col_combine_kernel<<<grid_for(n * nrhs), 256, 0, st>>>(W, V, vstride, ld, (int)n, (int)nrhs, nv, dev, -1.0);
      count_launch(2);
      FB_CK(cudaMemcpyAsync(pass == 0 ? hbuf.data() : hbuf2.data(), dev, sizeof(double) * nv * nrhs,
                            cudaMemcpyDeviceToHost, st));
    }
    coldots_kernel<<<dim3((unsigned)nrhs, 1), 256, 0, st>>>(W, 0, W, ld, (int)n, 1, dev);
    count_launch();
    FB_CK(cudaMemcpyAsync(host, dev, sizeof(double) * nrhs, cudaMemcpyDeviceToHost, st));
    FB_CK(cudaStreamSynchronize(st));
    bool all = true;
    for (long c = 0; c < nrhs; ++c) {
      for (int i = 0; i < nv; ++i) Hc(c, i, j) = hbuf[i + c * nv] + hbuf2[i + c * nv];
      const double hn = std::sqrt(std::max(0.0, host[c]));
      Hc(c, j + 1, j) = hn;
      inv[c] = hn > 0 ? 1.0 / hn : 0.0;
      // apply the previous rotations, then a new one zeroing H(j+1, j)
      for (int i = 0; i < j; ++i) {
        const double a = Hc(c, i, j), bb = Hc(c, i + 1, j);
        Hc(c, i, j) = cs[c * m + i] * a + sn[c * m + i] * bb;
        Hc(c, i + 1, j) = -sn[c * m + i] * a + cs[c * m + i] * bb;
      }
      const double a = Hc(c, j, j), bb = Hc(c, j + 1, j);
      const double r = std::hypot(a, bb);
      const double cc = r > 0 ? a / r : 1.0, ss = r > 0 ? bb / r : 0.0;
      cs[c * m + j] = cc;
      sn[c * m + j] = ss;
      Hc(c, j, j) = r;
      Hc(c, j + 1, j) = 0.0;
      const double gj = g[c * (m + 1) + j];
      g[c * (m + 1) + j] = cc * gj;
      g[c * (m + 1) + j + 1] = -ss * gj;
      if (!(std::fabs(g[c * (m + 1) + j + 1]) <= tol * beta[c])) all = false;
    }
    jdone = j + 1;
    if (all || j + 1 == m) break;
    FB_CK(cudaMemcpyAsync(dev, inv.data(), sizeof(double) * nrhs, cudaMemcpyHostToDevice, st));
    colscale_kernel<<<grid_for(n * nrhs), 256, 0, st>>>(W, V + (j + 1) * vstride, ld, (int)n, (int)nrhs, dev);
    count_launch();
  }
  // y = H^-1 g per column, D = V y
  std::vector<double> y((size_t)jdone * nrhs, 0.0);
  for (long c = 0; c < nrhs; ++c)
    for (int i = jdone - 1; i >= 0; --i) {
      double s = g[c * (m + 1) + i];
      for (int q = i + 1; q < jdone; ++q) s -= Hc(c, i, q) * y[q + c * jdone];
      const double d = Hc(c, i, i);
      y[i + c * jdone] = d != 0.0 ? s / d : 0.0;
    }
  FB_CK(cudaMemsetAsync(D, 0, sizeof(double) * ld * nrhs, st));
  FB_CK(cudaMemcpyAsync(dev, y.data(), sizeof(double) * jdone * nrhs, cudaMemcpyHostToDevice, st));
  col_combine_kernel<<<grid_for(n * nrhs), 256, 0, st>>>(D, V, vstride, ld, (int)n, (int)nrhs, jdone, dev, 1.0);
  count_launch();
  FB_CK(cudaGetLastError());
  *iters = jdone;
  return FLA_SUCCESS;
}

}  // namespace

// Refine X for A X = B with the low-precision factors f; X (n x nrhs, ld ldx)
// receives the solution.  Returns FLA_SUCCESS with res->iter >= 0 on
// convergence, res->iter = -31 (no convergence) otherwise.
int ir_refine(const DMat& A, const DMat& B, double* X, long ldx, const LpFactor& f, const IrConfig& cfg,
              IrResult* res) {
  Context& cx = ctx();
  cudaStream_t st = cx.stream;
  const long n = A.m, nrhs = B.n;
  res->iter = 0;
  res->inner = 0;
  IrBuffers b;
  const int m = std::max(1, cfg.gmres_m);
  const long ldn = (n + 1) & ~1L;  // 16-byte leading dimensions for the GEMM engine
  const size_t nb = (size_t)ldn * nrhs;
  char* w0 = (char*)ws_get(WS_IR0, sizeof(double) * 3 * nb + sizeof(float) * (2 * nb + (size_t)MB * nrhs) + 4096);
  double* v = cfg.solver == IR_GMRES ? (double*)ws_get(WS_IR1, sizeof(double) * (size_t)(m + 2) * nb) : nullptr;
  char* w2 = (char*)ws_get(WS_IR2, sizeof(double) * (size_t)(m + 2) * (nrhs + 2) + 4096);
  if (!w0 || !w2 || (cfg.solver == IR_GMRES && !v)) return FLA_FAILURE;
  b.R = (double*)w0;
  b.D = b.R + nb;
  b.R64 = b.D + nb;
  b.T = (float*)(b.R64 + nb);
  b.Tb = b.T + nb;
  b.V = v;
  b.W = v ? v + (size_t)(m + 1) * nb : nullptr;
  b.small = (double*)w2;
  std::vector<double> hs((size_t)(m + 2) * (nrhs + 2));
  b.h_small = hs.data();

  // cte = ||A||_inf * eps * sqrt(n)  (dsgesv.c:287-289)
  unsigned long long* dn = (unsigned long long*)b.small;
  FB_CK(cudaMemsetAsync(dn, 0, sizeof(unsigned long long), st));
  inf_norm_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(A.p, A.ld, (int)n, dn);
  count_launch();
  unsigned long long bits = 0;
  FB_CK(cudaMemcpyAsync(&bits, dn, sizeof(bits), cudaMemcpyDeviceToHost, st));
  FB_CK(cudaStreamSynchronize(st));
  double anrm;
  std::memcpy(&anrm, &bits, sizeof(anrm));
  const double eps = DBL_EPSILON * 0.5;
  const double cte = anrm * eps * std::sqrt((double)n);
  res->anorm = anrm;

  // x = M^-1 b
  if (lp_solve(f, B.p, B.ld, X, ldx, nrhs, b.T, b.Tb, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (residual(A, B, X, ldx, b.R, ldn, nrhs, st) != FLA_SUCCESS) return FLA_FAILURE;
  bool ok = false;
  static const bool trace = std::getenv("FLA_B200_IR_TRACE") != nullptr;
  // worst column's ||r||_inf / (||A||_inf ||x||_inf), from the last converged() call
  auto ratio = [&]() {
    double w = 0.0;
    for (long c = 0; c < nrhs; ++c) {
      const double den = anrm * b.h_small[c];
      w = std::max(w, den > 0 ? b.h_small[nrhs + c] / den : (b.h_small[nrhs + c] > 0 ? INFINITY : 0.0));
    }
    return w;
  };
  auto tlast = std::chrono::steady_clock::now();
  // timing events of the trace (the context's events are created without
  // timing)
  static cudaEvent_t tev[3] = {nullptr, nullptr, nullptr};
  if (trace && !tev[0])
    for (auto& e : tev) FB_CK(cudaEventCreate(&e));
  if (converged(X, ldx, b.R, ldn, n, nrhs, cte, b, st, &ok) != FLA_SUCCESS) return FLA_FAILURE;
  double last = ratio();
  if (trace) std::fprintf(stderr, "libflame_b200 ir: step 0  r/(|A||x|) %.3e\n", last);
  // After the dsgesv_ criterion holds, refinement goes on while each step
  // still halves the backward error, so that X reaches the backward error
  // of the FP64 factorization rather than the criterion's eps * sqrt(n).
  bool met = ok;
  int stall = 0;
  if (met && !cfg.polish) return FLA_SUCCESS;
  for (int it = 1; it <= cfg.itermax; ++it) {
    if (cfg.solver == IR_GMRES) {
      int inner = 0;
      if (gmres(A, f, b.R, b.D, nrhs, m, cfg.gmres_tol, b, st, &inner) != FLA_SUCCESS) return FLA_FAILURE;
      res->inner += inner;
    } else {
      if (trace) cudaEventRecord(tev[0], st);
      if (lp_solve(f, b.R, ldn, b.D, ldn, nrhs, b.T, b.Tb, st) != FLA_SUCCESS) return FLA_FAILURE;
      if (trace) cudaEventRecord(tev[1], st);
    }
    add_kernel<<<grid_for(n * nrhs), 256, 0, st>>>(X, ldx, b.D, ldn, (int)n, (int)nrhs, 1.0);
    count_launch();
    if (residual(A, B, X, ldx, b.R, ldn, nrhs, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (trace) cudaEventRecord(tev[2], st);
    if (converged(X, ldx, b.R, ldn, n, nrhs, cte, b, st, &ok) != FLA_SUCCESS) return FLA_FAILURE;
    const double now = ratio();
    if (trace) {
      const auto tnow = std::chrono::steady_clock::now();
      float ms_solve = 0.f, ms_res = 0.f;
      if (cfg.solver != IR_GMRES) {
        cudaEventElapsedTime(&ms_solve, tev[0], tev[1]);
        cudaEventElapsedTime(&ms_res, tev[1], tev[2]);
      }
      std::fprintf(stderr, "libflame_b200 ir: step %d  r/(|A||x|) %.3e  gmres %d  %.3f ms (solve %.3f, update + "
                   "residual %.3f)\n", it, now, res->inner,
                   std::chrono::duration<double, std::milli>(tnow - tlast).count(), ms_solve, ms_res);
      tlast = tnow;
    }
    if (met && !(now < 0.5 * last)) {
      // no longer improving: keep the better of the last two iterates
      if (now > last) {
        add_kernel<<<grid_for(n * nrhs), 256, 0, st>>>(X, ldx, b.D, ldn, (int)n, (int)nrhs, -1.0);
        count_launch();
      }
      res->iter = it;
      return FLA_SUCCESS;
    }
    if (ok && (!cfg.polish || met)) {
      res->iter = it;
      return FLA_SUCCESS;
    }
    if (ok) met = true;
    // stagnation: three steps in a row without halving the backward error
    // (adaptive solver: one step without a fourfold reduction)
    stall = (now < 0.5 * last) ? 0 : stall + 1;
    if (!met && cfg.solver == IR_AUTO && !(now < 0.25 * last)) stall = 3;
    if (!met && stall >= 3) {
      res->iter = -(cfg.itermax + 1);
      res->stalled = true;
      return FLA_SUCCESS;
    }
    last = std::min(last, now);
  }
  if (met) {
    res->iter = cfg.itermax;
    return FLA_SUCCESS;
  }
  res->iter = -(cfg.itermax + 1);
  return FLA_SUCCESS;
}

// Full symmetric FP64 copy of the stored triangle (residuals of the
// Cholesky solvers need the whole matrix).
int symmetrize(const DMat& A, bool upper, double* S, long lds, cudaStream_t st) {
  symmetrize_kernel<<<grid_for(A.m * A.m), 256, 0, st>>>(A.p, A.ld, S, lds, (int)A.m, upper ? 1 : 0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

IrConfig ir_default_config() {
  IrConfig c;
  if (const char* e = std::getenv("FLA_B200_IR_PREC")) {
    const std::string s(e);
    if (s == "bf16") c.prec = LP_BF16;
    if (s == "fp16") c.prec = LP_FP16;
    if (s == "tf32x3") c.prec = LP_TF32X3;
    if (s == "fp16x3") c.prec = LP_FP16X3;
  }
  if (const char* e = std::getenv("FLA_B200_IR_SOLVER")) {
    const std::string s(e);
    if (s == "ir") c.solver = IR_CLASSIC;
    if (s == "gmres") c.solver = IR_GMRES;
    if (s == "auto") c.solver = IR_AUTO;
  }
  return c;
}

}  // namespace fb
