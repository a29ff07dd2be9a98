// Reverse-mode differentiation of the Cholesky factorization and of the
// operations a Gaussian-process likelihood builds on it (no counterpart in
// the reference; the forward operations are FLA_Chol,
// src/lapack/dec/chol/front/flamec/FLA_Chol.c:16-29, and FLA_Trsm,
// src/base/flamec/blas/3/trsm/front/flamec/FLA_Trsm.c:15-26).
//
// Cholesky adjoint, blocked, right to left, in place over Lbar (Murray 2016,
// "Differentiation of the Cholesky decomposition", level-3 reverse mode).
// For the block column J (rows/columns j0 .. j0+w) write
//   R = L(J, 0:j0), D = L(J, J), B = L(below, 0:j0), C = L(below, J)
// and the same names with a bar for the adjoints stored in Lbar:
//   Cbar := Cbar inv(D)                         (GEMM with inv(D))
//   Bbar := Bbar - Cbar R                        (DMMA GEMM)
//   Dbar := Dbar - tril(Cbar^T C)                (DMMA GEMM, lower part)
//   Dbar := unblocked adjoint of chol(D)         (chol_adj_diag_kernel)
//   Rbar := Rbar - Cbar^T B - (Dbar + Dbar^T) R  (DMMA GEMMs)
// On return the lower triangle of Lbar holds Abar, the adjoint of the lower
// entries of A that the forward factorization reads; the gradient with
// respect to a symmetric A is (Abar + Abar^T) / 2.
//
// Unblocked adjoint of one diagonal block (reverse of the left-looking
// column step s_ij = a_ij - sum_k<j l_ik l_jk, l_jj = sqrt(s_jj),
// l_ij = s_ij / l_jj), columns from last to first:
//   lbar_ij /= l_jj (i > j);  lbar_jj = (lbar_jj - sum_i>j lbar_ij l_ij) / (2 l_jj)
//   lbar_jk -= 2 lbar_jj l_jk + sum_i>j lbar_ij l_ik   (k < j)
//   lbar_ik -= lbar_ij l_jk                              (i > j, k < j)
#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <vector>

#include "common.h"

namespace fb {

namespace {

constexpr int AB = 128;          // block size
constexpr int ADJ_THREADS = 512;
constexpr int PACKED = AB * (AB + 1) / 2;
constexpr size_t ADJ_SMEM = sizeof(double) * 2 * PACKED;

// packed lower, column-major: (i, j), i >= j
__device__ __forceinline__ int pk(int i, int j) { return i + j * (2 * AB - j - 1) / 2; }

__global__ void __launch_bounds__(ADJ_THREADS) chol_adj_diag_kernel(const double* __restrict__ L, double* Lb, long ld,
                                                                    int w) {
  extern __shared__ double asm_[];
  double* sD = asm_;
  double* sB = asm_ + PACKED;
  __shared__ double red[ADJ_THREADS / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int e = tid; e < w * w; e += ADJ_THREADS) {
    const int i = e % w, j = e / w;
    if (i >= j) {
      sD[pk(i, j)] = L[i + (long)j * ld];
      sB[pk(i, j)] = Lb[i + (long)j * ld];
    }
  }
  __syncthreads();
  for (int j = w - 1; j >= 0; --j) {
    const double d = sD[pk(j, j)];
    const double dinv = 1.0 / d;
    // lbar_ij /= l_jj, and the partial sums of lbar_ij l_ij
    double part = 0.0;
    for (int i = j + 1 + tid; i < w; i += ADJ_THREADS) {
      const double v = sB[pk(i, j)] * dinv;
      sB[pk(i, j)] = v;
      part = fma(v, sD[pk(i, j)], part);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
    if (lane == 0) red[warp] = part;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int q = 0; q < ADJ_THREADS / 32; ++q) s += red[q];
      sB[pk(j, j)] = (sB[pk(j, j)] - s) * (0.5 * dinv);
    }
    __syncthreads();
    const double bjj = sB[pk(j, j)];
    // row j, columns k < j: one thread per k
    for (int k = tid; k < j; k += ADJ_THREADS) {
      double s = 2.0 * bjj * sD[pk(j, k)];
      for (int i = j + 1; i < w; ++i) s = fma(sB[pk(i, j)], sD[pk(i, k)], s);
      sB[pk(j, k)] -= s;
    }
    // rectangle i > j, k < j
    const int rows = w - 1 - j;
    for (int e = tid; e < rows * j; e += ADJ_THREADS) {
      const int i = j + 1 + e % rows, k = e / rows;
      sB[pk(i, k)] -= sB[pk(i, j)] * sD[pk(j, k)];
    }
    __syncthreads();
  }
  for (int e = tid; e < w * w; e += ADJ_THREADS) {
    const int i = e % w, j = e / w;
    if (i >= j) Lb[i + (long)j * ld] = sB[pk(i, j)];
  }
}

// S := (Db + Db^T) with Db lower (w x w), into S (ld lds)
__global__ void symmetric_sum_kernel(const double* __restrict__ Db, long ld, double* __restrict__ S, long lds, int w) {
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < w * w; e += gridDim.x * blockDim.x) {
    const int i = e % w, j = e / w;
    const double a = (i >= j) ? Db[i + (long)j * ld] : 0.0;
    const double b = (j >= i) ? Db[j + (long)i * ld] : 0.0;
    S[i + (long)j * lds] = a + b;
  }
}

// Lbar(i, i) += scale / L(i, i)
__global__ void logdet_adj_kernel(const double* __restrict__ L, double* __restrict__ Lb, long ld, long n,
                                  double scale) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) Lb[i + i * ld] += scale / L[i + i * ld];
}
// partial sums of log L(i, i)
__global__ void logdet_kernel(const double* __restrict__ L, long ld, long n, double* out) {
  __shared__ double red[256];
  double s = 0.0;
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    s += log(L[i + i * ld]);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if (threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(out, red[0]);
}

bool g_adj_attr = false;

}  // namespace

// Scratch of chol_adjoint_dev for order n: Dinv (AB x AB) then W (ldw x AB)
// and S (AB x AB), in doubles.
size_t chol_adjoint_scratch(long n) { return (size_t)AB * AB * 2 + (size_t)((n + 1) & ~1L) * AB; }

// In place over Lb (lower triangle); L lower Cholesky factor; n x n, ld.
// scratch: chol_adjoint_scratch(n) doubles of device memory, or nullptr for
// the library's workspace (then calls must not overlap).
int chol_adjoint_dev(const double* L, double* Lb, long ld, long n, cudaStream_t st, double* scratch) {
  if (n <= 0) return FLA_SUCCESS;
  if (!g_adj_attr) {
    FB_CK(cudaFuncSetAttribute(chol_adj_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ADJ_SMEM));
    g_adj_attr = true;
  }
  const long nblk = (n + AB - 1) / AB;
  const long ldw = (n + 1) & ~1L;
  double* Dinv = scratch ? scratch : (double*)ws_get(WS_MISC, sizeof(double) * AB * AB);
  double* W = scratch ? scratch + (size_t)AB * AB
                      : (double*)ws_get(WS_MISC2, sizeof(double) * (size_t)ldw * AB + sizeof(double) * AB * AB);
  if (!Dinv || !W) return FLA_FAILURE;
  double* S = W + (size_t)ldw * AB;  // (Dbar + Dbar^T), AB x AB
  auto Lat = [&](long i, long j) { return L + i + j * ld; };
  auto Bat = [&](long i, long j) { return Lb + i + j * ld; };
  for (long q = nblk - 1; q >= 0; --q) {
    const long j0 = q * AB;
    const int w = (int)std::min<long>(AB, n - j0);
    const long m = n - j0 - w;  // rows below the block
    if (m > 0) {
      // Cbar := Cbar inv(D)
      if (tri_inverse(Lat(j0, j0), ld, w, true, false, Dinv, AB, st) != FLA_SUCCESS) return FLA_FAILURE;
      FB_CK(cudaMemcpy2DAsync(W, sizeof(double) * ldw, Bat(j0 + w, j0), sizeof(double) * ld, sizeof(double) * m, w,
                              cudaMemcpyDeviceToDevice, st));
      if (gemm_f64(st, false, false, m, w, w, 1.0, W, ldw, Dinv, AB, 0.0, Bat(j0 + w, j0), ld) != FLA_SUCCESS)
        return FLA_FAILURE;
      // Bbar := Bbar - Cbar R
      if (j0 > 0 &&
          gemm_f64(st, false, false, m, j0, w, -1.0, Bat(j0 + w, j0), ld, Lat(j0, 0), ld, 1.0, Bat(j0 + w, 0), ld) !=
              FLA_SUCCESS)
        return FLA_FAILURE;
      // Dbar := Dbar - tril(Cbar^T C)
      if (gemm_f64(st, true, false, w, w, m, -1.0, Bat(j0 + w, j0), ld, Lat(j0 + w, j0), ld, 1.0, Bat(j0, j0), ld,
                   GEMM_LOWER, 0) != FLA_SUCCESS)
        return FLA_FAILURE;
    }
    chol_adj_diag_kernel<<<1, ADJ_THREADS, ADJ_SMEM, st>>>(Lat(j0, j0), Bat(j0, j0), ld, w);
    count_launch();
    FB_CK(cudaGetLastError());
    if (j0 > 0) {
      // Rbar := Rbar - Cbar^T B - (Dbar + Dbar^T) R
      if (m > 0 &&
          gemm_f64(st, true, false, w, j0, m, -1.0, Bat(j0 + w, j0), ld, Lat(j0 + w, 0), ld, 1.0, Bat(j0, 0), ld) !=
              FLA_SUCCESS)
        return FLA_FAILURE;
      symmetric_sum_kernel<<<64, 256, 0, st>>>(Bat(j0, j0), ld, S, AB, w);
      count_launch();
      if (gemm_f64(st, false, false, w, j0, w, -1.0, S, AB, Lat(j0, 0), ld, 1.0, Bat(j0, 0), ld) != FLA_SUCCESS)
        return FLA_FAILURE;
    }
  }
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// Lbar += scale * diag(1 / L_ii): adjoint of scale * sum_i log L_ii.
int logdet_adjoint_dev(const double* L, double* Lb, long ld, long n, double scale, cudaStream_t st) {
  if (n <= 0) return FLA_SUCCESS;
  logdet_adj_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(L, Lb, ld, n, scale);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

int logdet_dev(const double* L, long ld, long n, double* h_out, cudaStream_t st) {
  double* d = (double*)ws_get(WS_IR2, sizeof(double) * 8);
  if (!d) return FLA_FAILURE;
  FB_CK(cudaMemsetAsync(d, 0, sizeof(double), st));
  logdet_kernel<<<(unsigned)std::min<long>(1024, (n + 255) / 256), 256, 0, st>>>(L, ld, n, d);
  count_launch();
  FB_CK(cudaMemcpyAsync(h_out, d, sizeof(double), cudaMemcpyDeviceToHost, st));
  FB_CK(cudaStreamSynchronize(st));
  return FLA_SUCCESS;
}

// Adjoint of X = inv(L) B (L lower, non-unit, n x n; X, B n x k):
//   Bbar := inv(L)^T Xbar (in place over Xbar), Lbar -= tril(Bbar X^T).
int trsm_adjoint_dev(DMat L, DMat X, DMat Xbar, double* Lb, long ldlb, cudaStream_t st) {
  if (trsm_left_dev(L, Xbar, true, true, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  return gemm_f64(st, false, true, L.m, L.m, X.n, -1.0, Xbar.p, Xbar.ld, X.p, X.ld, 1.0, Lb, ldlb, GEMM_LOWER, 0);
}

}  // namespace fb

using namespace fb;

extern "C" {

// No counterpart in the reference.  Adjoint of the lower Cholesky
// factorization A = L L^T (FLA_Chol): L holds the factor, Lbar (same order)
// the adjoint of L in its lower triangle; on return the lower triangle of
// Lbar holds Abar, the adjoint of the lower entries of A (the gradient with
// respect to a symmetric A is (Abar + Abar^T)/2).  Only the lower triangles
// are read or written.  FLA_DOUBLE objects, device or host buffers.
FLA_Error FLA_Chol_adjoint(FLA_Uplo uplo, FLA_Obj L, FLA_Obj Lbar) {
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(uplo == FLA_LOWER_TRIANGULAR, "FLA_Chol_adjoint", "only FLA_LOWER_TRIANGULAR is provided");
  FB_REQUIRE(L.base && Lbar.base && L.base->datatype == FLA_DOUBLE && Lbar.base->datatype == FLA_DOUBLE,
             "FLA_Chol_adjoint", "objects must be FLA_DOUBLE");
  FB_REQUIRE(L.m == L.n && Lbar.m == L.m && Lbar.n == L.n, "FLA_Chol_adjoint", "nonconformal objects");
  if (L.m == 0) return FLA_SUCCESS;
  Staged sl, sb;
  if (stage(L, WS_STAGE_A, &sl) != FLA_SUCCESS || stage(Lbar, WS_STAGE_B, &sb) != FLA_SUCCESS) return FLA_FAILURE;
  if (sl.ld != sb.ld) {
    set_last_error("FLA_Chol_adjoint: L and Lbar need the same leading dimension");
    return FLA_FAILURE;
  }
  cudaStream_t st = ctx().stream;
  op_begin(st);
  if (chol_adjoint_dev((const double*)sl.dev, (double*)sb.dev, sl.ld, (long)L.m, st, nullptr) != FLA_SUCCESS)
    return FLA_FAILURE;
  op_end(st);
  if (unstage(sb) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// Lbar += scale * diag(1/L(i,i)), the adjoint of scale * sum_i log L(i,i)
// (log det A = 2 sum_i log L(i,i)); *logdet (optional) receives
// sum_i log L(i,i).
FLA_Error FLA_B200_Chol_logdet_adjoint(FLA_Obj L, FLA_Obj Lbar, double scale, double* logdet) {
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(L.base && Lbar.base && L.m == L.n && Lbar.m == L.m && Lbar.n == L.n, "FLA_B200_Chol_logdet_adjoint",
             "nonconformal objects");
  Staged sl, sb;
  if (stage(L, WS_STAGE_A, &sl) != FLA_SUCCESS || stage(Lbar, WS_STAGE_B, &sb) != FLA_SUCCESS) return FLA_FAILURE;
  if (sl.ld != sb.ld) {
    set_last_error("FLA_B200_Chol_logdet_adjoint: L and Lbar need the same leading dimension");
    return FLA_FAILURE;
  }
  cudaStream_t st = ctx().stream;
  op_begin(st);
  if (logdet && logdet_dev((const double*)sl.dev, sl.ld, (long)L.m, logdet, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (logdet_adjoint_dev((const double*)sl.dev, (double*)sb.dev, sb.ld, (long)L.m, scale, st) != FLA_SUCCESS)
    return FLA_FAILURE;
  op_end(st);
  if (unstage(sb) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// Adjoint of X = inv(L) B (FLA_Trsm left, lower, no transpose, non-unit):
// given X and Xbar (n x k), Xbar := Bbar = inv(L)^T Xbar and Lbar -=
// tril(Bbar X^T).
FLA_Error FLA_B200_Trsm_llnn_adjoint(FLA_Obj L, FLA_Obj X, FLA_Obj Xbar, FLA_Obj Lbar) {
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(L.base && X.base && Xbar.base && Lbar.base && L.m == L.n && X.m == L.m && Xbar.m == L.m &&
                 Xbar.n == X.n && Lbar.m == L.m && Lbar.n == L.n,
             "FLA_B200_Trsm_llnn_adjoint", "nonconformal objects");
  Staged sl, sx, sxb, slb;
  if (stage(L, WS_STAGE_A, &sl) != FLA_SUCCESS || stage(X, WS_STAGE_B, &sx) != FLA_SUCCESS ||
      stage(Xbar, WS_STAGE_X, &sxb) != FLA_SUCCESS || stage(Lbar, WS_FB, &slb) != FLA_SUCCESS)
    return FLA_FAILURE;
  cudaStream_t st = ctx().stream;
  auto dm = [](const Staged& s) {
    DMat d;
    d.p = (double*)s.dev;
    d.ld = s.ld;
    d.m = s.m;
    d.n = s.n;
    return d;
  };
  op_begin(st);
  if (trsm_adjoint_dev(dm(sl), dm(sx), dm(sxb), (double*)slb.dev, slb.ld, st) != FLA_SUCCESS) return FLA_FAILURE;
  op_end(st);
  if (unstage(sxb) != FLA_SUCCESS || unstage(slb) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// No counterpart in the reference.  FLA_Chol_adjoint over a batch: for each
// i, L[i] (device, order n[i], leading dimension ld[i]) holds a lower
// Cholesky factor and Lbar[i] (device, same order and leading dimension)
// the adjoint of L[i]; first Lbar[i](j, j) += logdet_scale / L[i](j, j) (the
// adjoint of logdet_scale * sum_j log L(j, j); 0 skips it), then Lbar[i]'s
// lower triangle is replaced by Abar[i] as FLA_Chol_adjoint does.  Each
// matrix runs the blocked adjoint; the matrices, largest first, are spread
// round-robin over a pool of streams with a scratch area each, so the small
// per-block kernels of different matrices overlap.
FLA_Error FLA_Chol_adjoint_batched(int count, const int* n, double** L, const int* ld, double** Lbar,
                                   double logdet_scale) {
  if (!ctx().initialized) FLA_Init();
  long maxn = 0;
  for (int i = 0; i < count; ++i) {
    FB_REQUIRE(n[i] >= 0 && ld[i] >= std::max(1, n[i]), "FLA_Chol_adjoint_batched", "bad order or leading dimension");
    if (n[i] > 0 && (!is_device_ptr(L[i]) || !is_device_ptr(Lbar[i]))) {
      set_last_error("FLA_Chol_adjoint_batched: matrix " + std::to_string(i) + ": buffers must be device memory");
      return FLA_FAILURE;
    }
    maxn = std::max<long>(maxn, n[i]);
  }
  if (count <= 0 || maxn == 0) return FLA_SUCCESS;
  constexpr int NS = 8;
  static cudaStream_t pool[NS];
  static cudaEvent_t ev[NS + 1];
  static bool made = false;
  if (!made) {
    for (int q = 0; q < NS; ++q) FB_CK(cudaStreamCreateWithFlags(&pool[q], cudaStreamNonBlocking));
    for (int q = 0; q <= NS; ++q) FB_CK(cudaEventCreateWithFlags(&ev[q], cudaEventDisableTiming));
    made = true;
  }
  const size_t per = chol_adjoint_scratch(maxn);
  double* scr = (double*)ws_get(WS_ADJ, sizeof(double) * per * NS);
  if (!scr) return FLA_FAILURE;
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return n[x] > n[y]; });
  cudaStream_t st = ctx().stream;
  op_begin(st);
  FB_CK(cudaEventRecord(ev[NS], st));
  for (int q = 0; q < NS; ++q) FB_CK(cudaStreamWaitEvent(pool[q], ev[NS], 0));
  // orders above 2048 reach the GEMM engine's split-K workspace, which the
  // streams of the pool would share: one stream then
  const int ns = maxn > 2048 ? 1 : NS;
  for (int k = 0; k < count; ++k) {
    const int i = order[k], q = k % ns;
    if (n[i] == 0) continue;
    if (logdet_scale != 0.0 && logdet_adjoint_dev(L[i], Lbar[i], ld[i], n[i], logdet_scale, pool[q]) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (chol_adjoint_dev(L[i], Lbar[i], ld[i], n[i], pool[q], scr + per * q) != FLA_SUCCESS) return FLA_FAILURE;
  }
  for (int q = 0; q < NS; ++q) {
    FB_CK(cudaEventRecord(ev[q], pool[q]));
    FB_CK(cudaStreamWaitEvent(st, ev[q], 0));
  }
  op_end(st);
  return sync_all();
}

}  // extern "C"
