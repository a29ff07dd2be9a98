// QR factorization via the UT transform (FLA_QR_UT) and the application of
// Q (FLA_Apply_Q_UT) on the GPU; dgeqrf_ on top.
//
// Reference: src/lapack/dec/q/qrut/vars/flamec/FLA_QR_UT_blk_var1.c:13-102
// (blocks of b_alg = length(T) columns: panel QR into the b_alg x b_alg
// block of T, then Q1^T applied to the trailing columns through
// FLA_Apply_Q_UT lhfc var1, src/lapack/util/app/qut/lhfc/flamec/
// FLA_Apply_Q_UT_lhfc_blk_var1.c:148-182), with the unblocked leaf
// FLA_QR_UT_opt_var2.c:161-226 and the Householder vector of
// src/base/flamec/util/lapack/FLA_Househ2_UT.c:274-386:
//   alpha = -sign(chi1) ||[chi1; x2]||,  u2 = x2 / (chi1 - alpha),
//   tau = 1/2 + 1/2 (||x2|| / |chi1 - alpha|)^2,  chi1 := alpha
//   (||x2|| = 0: tau = 1/2, chi1 := -chi1),
// and T = striu(U^T U) + diag(tau) per block.
//
// GPU structure: panels of NBQ = (64 / b_alg) * b_alg columns are factored
// by a cooperative kernel (row slabs in SMEM, two grid barriers per column:
// one for ||x2||, one for the dot products that give both the update row w
// and the T column); the NBQ x NBQ triangular factor of the whole panel is
// formed on the way and its b_alg x b_alg diagonal blocks are the T blocks
// the reference's interface stores.  The trailing columns get
// B := (I - U T^-T U^T) B as two GEMM-engine calls and a triangular solve.
#include <climits>
#include <cstring>

#include "common.h"
#include "dev_util.cuh"

namespace fb {

namespace {

constexpr int QR_THREADS = 256;
constexpr int QR_NBMAX = 64;  // widest panel of the cooperative kernel
constexpr int QR_NB = 128;     // panel width of the blocked factorization (T blocks per panel: 128 / b_alg)
constexpr size_t QR_SMEM_CAP = 200 * 1024;

struct QrPanelArgs {
  double* P;       // panel, column-major (row k, col k of A)
  long ld;
  int M, nb;       // panel rows, columns
  int R, lds, G;   // rows per CTA, SMEM stride, CTAs
  double* Tbig;    // out: nb x nb (ld ldt), upper triangle with diagonal
  long ldt;
  double* part_ss; // [2][G]      partial ||x2||^2 per CTA
  double* part;    // [2][G][nb]  partial dot products per CTA
  double* rowj;    // [2][nb + 1] row j (and chi1 at [nb])
  unsigned* bar;
  int* err;
};

// Deterministic CTA-wide sum (fixed thread -> partial mapping, fixed tree).
__device__ __forceinline__ double block_sum(double v, double* sred) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  if (lane == 0) sred[warp] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < QR_THREADS / 32; ++w) t += sred[w];
    sred[QR_THREADS / 32] = t;
  }
  __syncthreads();
  return sred[QR_THREADS / 32];
}

__global__ void __launch_bounds__(QR_THREADS) qr_panel_kernel(QrPanelArgs a) {
  extern __shared__ double S[];  // slab S[i + c*lds]; then w[nb]
  __shared__ double sred[QR_THREADS / 32 + 1];
  __shared__ double s_scale, s_alpha, s_tau, s_rtau;
  __shared__ int s_trivial;
  double* sw = S + (size_t)a.lds * a.nb;  // per-column d_c / w_c
  const int c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = c * a.R, rows = min(a.R, a.M - r0);
  const int nb = a.nb, lds = a.lds, G = a.G;

  for (int col = 0; col < nb; ++col)
    for (int i = tid; i < rows; i += QR_THREADS) S[i + col * lds] = a.P[(long)(r0 + i) + (long)col * a.ld];
  __syncthreads();

  const int mn = min(a.M, nb);
  for (int j = 0; j < mn; ++j) {
    const int par = j & 1;
    double* part = a.part + (size_t)par * G * nb;
    double* part_ss = a.part_ss + (size_t)par * G;
    double* rowj = a.rowj + (size_t)par * (nb + 1);
    const bool own_j = (j >= r0 && j < r0 + rows);
    // ---- A: ||x2||^2 partial over rows > j, chi1 from the owner of row j
    double ss = 0.0;
    for (int i = tid; i < rows; i += QR_THREADS)
      if (r0 + i > j) {
        const double x = S[i + j * lds];
        ss = fma(x, x, ss);
      }
    ss = block_sum(ss, sred);
    if (tid == 0) __stcg(part_ss + c, ss);
    if (own_j && tid == 0) __stcg(rowj + nb, S[(j - r0) + j * lds]);
    if (!grid_barrier(a.bar, (unsigned)G, (unsigned)(2 * j + 1), a.err, 31)) return;
    // ---- B: Householder vector (every CTA computes the same values)
    if (warp == 0) {
      double t = 0.0;
      for (int g = lane; g < G; g += 32) t += __ldcg(part_ss + g);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
      if (lane == 0) {
        const double chi1 = __ldcg(rowj + nb);
        const double nx2 = sqrt(t);
        if (nx2 == 0.0) {
          s_trivial = 1;
          s_scale = 1.0;
          s_alpha = -chi1;
          s_tau = 0.5;
        } else {
          const double nx = hypot(fabs(chi1), nx2);
          const double alpha = -((chi1 < 0.0) ? -1.0 : 1.0) * nx;
          const double cma = chi1 - alpha;
          const double q = nx2 / fabs(cma);
          s_trivial = 0;
          s_scale = 1.0 / cma;
          s_alpha = alpha;
          s_tau = 0.5 + 0.5 * (q * q);
        }
        s_rtau = 1.0 / s_tau;
      }
    }
    __syncthreads();
    if (!s_trivial)
      for (int i = tid; i < rows; i += QR_THREADS)
        if (r0 + i > j) S[i + j * lds] *= s_scale;
    if (own_j && tid == 0) S[(j - r0) + j * lds] = s_alpha;
    __syncthreads();
    // dot products d_col = sum_{rows > j} u_i a(i, col), all col != j
    for (int col = warp; col < nb; col += QR_THREADS / 32) {
      double d = 0.0;
      if (col != j)
        for (int i = lane; i < rows; i += 32)
          if (r0 + i > j) d = fma(S[i + j * lds], S[i + col * lds], d);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
      if (lane == 0) __stcg(part + (size_t)c * nb + col, d);
    }
    if (own_j)
      for (int col = tid; col < nb; col += QR_THREADS) __stcg(rowj + col, S[(j - r0) + col * lds]);
    if (!grid_barrier(a.bar, (unsigned)G, (unsigned)(2 * j + 2), a.err, 32)) return;
    // ---- C: apply H_j to the columns right of j; T column j
    for (int col = warp; col < nb; col += QR_THREADS / 32) {
      double d = 0.0;
      for (int g = lane; g < G; g += 32) d += __ldcg(part + (size_t)g * nb + col);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
      if (lane == 0) {
        const double rj = __ldcg(rowj + col);
        if (col > j) {
          sw[col] = (rj + d) * s_rtau;  // w = (a1t + A2^T u2) / tau
        } else if (col < j) {
          if (c == 0) a.Tbig[col + (long)j * a.ldt] = rj + d;  // t01 = a10t^T + A20^T u21
        } else if (c == 0) {
          a.Tbig[j + (long)j * a.ldt] = s_tau;
        }
      }
    }
    __syncthreads();
    for (int col = j + 1; col < nb; ++col) {
      const double wc = sw[col];
      for (int i = tid; i < rows; i += QR_THREADS) {
        const int gi = r0 + i;
        if (gi > j) S[i + col * lds] = fma(-S[i + j * lds], wc, S[i + col * lds]);
        else if (gi == j) S[i + col * lds] -= wc;
      }
    }
    __syncthreads();
  }
  for (int col = 0; col < nb; ++col)
    for (int i = tid; i < rows; i += QR_THREADS) a.P[(long)(r0 + i) + (long)col * a.ld] = S[i + col * lds];
}

// Uw (M x b, ld ldu) := unit lower trapezoid of P (M x b): ones on the
// diagonal, zeros above, P below.
__global__ void form_unit_lower_kernel(const double* __restrict__ P, long ldp, double* __restrict__ U,
                                       long ldu, int M, int b) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)M * b;
  if (idx >= total) return;
  const int col = (int)(idx / M), row = (int)(idx % M);
  double v = 0.0;
  if (row > col) v = P[row + (long)col * ldp];
  else if (row == col) v = 1.0;
  U[row + (long)col * ldu] = v;
}

// Copy the b_alg x b_alg diagonal blocks of Tbig (cols x cols, ld ldb)
// into T's columns [k, k+cols) (T is b_alg x n, ld ldt); only the upper
// triangles.
__global__ void extract_t_blocks_kernel(const double* __restrict__ Tbig, long ldb, int cols, double* T,
                                        long ldt, int b_alg) {
  const int j = blockIdx.x;           // panel column
  if (j >= cols) return;
  const int blk0 = (j / b_alg) * b_alg;
  for (int i = threadIdx.x; i < b_alg; i += blockDim.x) {
    const int r = blk0 + i;           // row of Tbig
    if (r <= j) T[i + (long)j * ldt] = Tbig[r + (long)j * ldb];
  }
}

// t[j] := T(j mod b_alg, j) (FLA_QR_UT_recover_tau), optionally 1/t[j]
// (FLAME_invert_dtau, src/map/lapack2flamec/FLA_lapack2flame_util.c:96-113).
__global__ void recover_tau_kernel(const double* T, long ldt, int b_alg, int k, double* t, long inct,
                                   int invert) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  double v = T[(j % b_alg) + (long)j * ldt];
  if (invert && v != 0.0) v = 1.0 / v;
  t[(long)j * inct] = v;
}

bool g_qr_attrs = false;
void set_qr_attrs() {
  if (g_qr_attrs) return;
  cudaFuncSetAttribute(qr_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(220 * 1024));
  g_qr_attrs = true;
}

struct QrGeom {
  int R, G, lds;
};
QrGeom qr_geom(long M, int nb) {
  QrGeom g;
  long r = std::max<long>(std::min<long>(M, 32), (M + 63) / 64);
  if ((size_t)(r | 1) * nb * 8 + nb * 8 > QR_SMEM_CAP)
    r = std::max<long>(std::min<long>(M, 32), (M + ctx().num_sms - 1) / ctx().num_sms);
  g.R = (int)r;
  g.G = (int)((M + r - 1) / r);
  g.lds = g.R | 1;
  return g;
}

long even_up(long x) { return (x + 1) & ~1L; }

}  // namespace

// One M x nb panel (nb <= 64) by the cooperative kernel: two grid barriers
// per column; for pieces taller than any cluster leaf holds.  Tb (ld ldtb)
// receives the panel's nb x nb T.
int qr_coop_panel(double* P, long ld, long M, int nb, double* Tb, long ldtb, cudaStream_t st) {
  set_qr_attrs();
  Context& cx = ctx();
  QrGeom g = qr_geom(M, nb);
  if (nb > QR_NBMAX || (size_t)g.lds * nb * 8 + nb * 8 > QR_SMEM_CAP || g.G > cx.num_sms) {
    set_last_error("FLA_QR_UT: panel too tall for the cooperative panel kernel");
    return FLA_FAILURE;
  }
  const int GMAX = cx.num_sms;
  const size_t b_part = sizeof(double) * (size_t)2 * GMAX * (QR_NBMAX + 1);
  const size_t b_rowj = sizeof(double) * 2 * (QR_NBMAX + 1);
  char* ws = (char*)ws_get(WS_PANEL, b_part + b_rowj + 256);
  if (!ws) return FLA_FAILURE;
  QrPanelArgs pa;
  pa.P = P;
  pa.ld = ld;
  pa.M = (int)M;
  pa.nb = nb;
  pa.R = g.R;
  pa.lds = g.lds;
  pa.G = g.G;
  pa.Tbig = Tb;
  pa.ldt = ldtb;
  pa.part = (double*)ws;
  pa.part_ss = pa.part + (size_t)2 * GMAX * nb;
  pa.rowj = (double*)(ws + b_part);
  pa.bar = (unsigned*)(cx.d_status + ST_BAR);
  pa.err = cx.d_status + ST_ERROR;
  FB_CK(cudaMemsetAsync(pa.bar, 0, sizeof(unsigned), st));
  const size_t smem = (size_t)g.lds * nb * 8 + (size_t)nb * 8;
  void* args[] = {&pa};
  const int ps = prof_begin(st);
  FB_CK(cudaLaunchCooperativeKernel((void*)qr_panel_kernel, dim3(g.G), dim3(QR_THREADS), args, smem, st));
  prof_end(ps, st, PROF_PANEL, 0.0);
  count_launch();
  return FLA_SUCCESS;
}

// qr_panel.cu
int qr_panel_factor(double* P, long ld, long M, int w, double* Tb, long ldtb, double* U, long ldu, double* Wk,
                    long ldw, cudaStream_t st);
int unit_lower_copy(const double* P, long ldp, double* U, long ldu, long M, int b, cudaStream_t st);

namespace {

// B := (I - U T^-T U^T) B, U the M x b unit lower trapezoid (explicit,
// ld ldu), B M x nc, with Ti = T^-1 (ld ldti) precomputed: W := U^T B,
// W2 := Ti^T W, B -= U W2 (W and W2 b x nc, ld ldw, scratch).  The
// explicit inverse turns the b-step triangular solve into a GEMM.  The
// k = M product is split into slices of at most 1024 rows so that its
// tiles leave SMs often enough for the cluster leaves of the next panel.
int apply_block_qt(const double* U, long ldu, const double* Ti, long ldti, long M, int b, double* B, long ldb,
                   long nc, double* W, double* W2, long ldw, cudaStream_t st) {
  if (nc <= 0) return FLA_SUCCESS;
  if (gemm_f64(st, true, false, b, nc, M, 1.0, U, ldu, B, ldb, 0.0, W, ldw, GEMM_FULL, 0, nullptr, 0x7fffffff,
               1024) != FLA_SUCCESS)
    return FLA_FAILURE;
  if (gemm_f64(st, true, false, b, nc, b, 1.0, Ti, ldti, W, ldw, 0.0, W2, ldw) != FLA_SUCCESS) return FLA_FAILURE;
  return gemm_f64(st, false, false, M, nc, b, -1.0, U, ldu, W2, ldw, 1.0, B, ldb);
}

}  // namespace

// A := QR in place (A m x n); T (b_alg x n, ld ldt) receives the T blocks.
// Panels of NBQ = (128 / b_alg) b_alg columns (recursive cluster panels,
// qr_panel.cu) on the side stream, one panel ahead: after panel k, the
// main stream first updates panel k+1's columns, then the side stream
// factors panel k+1 while the main stream updates the remaining columns
// with the UT transform of panel k (two GEMMs and a triangular solve with
// its T).
int qr_ut_dev(DMat A, DMat T, int b_alg) {
  set_qr_attrs();
  Context& cx = ctx();
  cudaStream_t st = cx.stream, sd = cx.side;
  const long m = A.m, n = A.n, mn = std::min(m, n);
  if (mn == 0) return FLA_SUCCESS;
  const int NBQ = std::max(1, QR_NB / b_alg) * b_alg;
  const long ldu = even_up(m), ldtb = even_up(NBQ), ldw = even_up(NBQ);
  double* Tb2 = (double*)ws_get(WS_QR_T, sizeof(double) * 4 * (size_t)ldtb * NBQ);  // T, T^-1 of two panels
  double* Wt = (double*)ws_get(WS_MISC2, sizeof(double) * 2 * (size_t)ldw * std::max<long>(n, 1));
  double* Up2 = (double*)ws_get(WS_QR_U, sizeof(double) * 2 * (size_t)ldu * NBQ);  // U of two panels
  double* Wp = (double*)ws_get(WS_QR_W, sizeof(double) * 3 * (size_t)ldw * NBQ);
  if (!Tb2 || !Wt || !Up2 || !Wp) return FLA_FAILURE;
  double* Wt2 = Wt + (size_t)ldw * std::max<long>(n, 1);
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;
  cudaEvent_t ev_look = cx.ev[0], ev_panel = cx.ev[1];
  auto a_at = [&](long i, long j) { return A.p + i + j * A.ld; };
  auto tb = [&](long k) { return Tb2 + (size_t)((k / NBQ) & 1) * ldtb * NBQ; };
  auto ti = [&](long k) { return Tb2 + (size_t)(2 + ((k / NBQ) & 1)) * ldtb * NBQ; };
  auto up = [&](long k) { return Up2 + (size_t)((k / NBQ) & 1) * ldu * NBQ; };
  auto panel = [&](long k, int b, cudaStream_t s) -> int {
    if (qr_panel_factor(a_at(k, k), A.ld, m - k, b, tb(k), ldtb, up(k), ldu, Wp, ldw, s) != FLA_SUCCESS)
      return FLA_FAILURE;
    extract_t_blocks_kernel<<<b, std::min(std::max(32, b_alg), 1024), 0, s>>>(tb(k), ldtb, b, T.p + k * T.ld,
                                                                            T.ld, b_alg);
    count_launch();
    if (k + b >= n) return FLA_SUCCESS;  // no trailing columns: T^-1 unused
    return tri_inverse(tb(k), ldtb, b, false, false, ti(k), ldtb, s);
  };
  if (panel(0, (int)std::min<long>(NBQ, mn), st) != FLA_SUCCESS) return FLA_FAILURE;
  for (long k = 0; k < mn; k += NBQ) {
    const int b = (int)std::min<long>(NBQ, mn - k);
    const long M = m - k, n2 = n - k - b;
    if (n2 <= 0) break;
    double* Uk = up(k);
    const int nb2 = (int)std::min<long>(NBQ, mn - k - b);  // next panel's width (0: none)
    if (nb2 > 0) {
      if (apply_block_qt(Uk, ldu, ti(k), ldtb, M, b, a_at(k, k + b), A.ld, nb2, Wt, Wt2, ldw, st) != FLA_SUCCESS)
        return FLA_FAILURE;
      FB_CK(cudaEventRecord(ev_look, st));
      FB_CK(cudaStreamWaitEvent(sd, ev_look, 0));
      if (panel(k + b, nb2, sd) != FLA_SUCCESS) return FLA_FAILURE;
      FB_CK(cudaEventRecord(ev_panel, sd));
    }
    if (apply_block_qt(Uk, ldu, ti(k), ldtb, M, b, a_at(k, k + b + nb2), A.ld, n2 - nb2, Wt, Wt2, ldw, st) !=
        FLA_SUCCESS)
      return FLA_FAILURE;
    if (nb2 > 0) FB_CK(cudaStreamWaitEvent(st, ev_panel, 0));
  }
  int info;
  return status_read(&info);
}

namespace {

// The s x s triangular factor of a super-block of s / b_alg consecutive
// UT blocks: the stored b_alg x b_alg T blocks on the diagonal, the Gram
// blocks U_i^T U_j of G (ld ldg) above them; below the diagonal is unused.
__global__ void assemble_t_kernel(const double* __restrict__ T, long ldt, int b_alg, const double* __restrict__ G,
                                  long ldg, int s, double* __restrict__ Ts, long ldts) {
  const int j = blockIdx.x;
  for (int i = threadIdx.x; i <= j && i < s; i += blockDim.x) {
    const bool diag_blk = (i / b_alg) == (j / b_alg);
    Ts[i + (long)j * ldts] = diag_blk ? T[(i % b_alg) + (long)j * ldt] : G[i + (long)j * ldg];
  }
}

}  // namespace

// B := Q^T B (transpose_q) or Q B for Q = H(0) H(1) ... from the UT
// representation in U (m x k, below the diagonal) and T (b_alg x k), the
// blocks of FLA_Apply_Q_UT_lhfc/lhfc var1
// (src/lapack/util/app/qut/lhfc/flamec/FLA_Apply_Q_UT_lhfc_blk_var1.c:
// 148-182), grouped into super-blocks of S = (128 / b_alg) b_alg columns:
// one GEMM U^T [U | B] gives both the Gram blocks that complete the
// super-block's triangular factor (its diagonal blocks are the stored T
// blocks) and W = U^T B; then W2 := Ts^-T W (Q^T) or Ts^-1 W (Q), through
// the explicit inverse of Ts, and B -= U W2.  The product of the super-block's UT transforms is the single
// UT transform with that factor, so the result is the block-by-block one up
// to rounding.
int apply_q_dev(DMat U, DMat T, int b_alg, DMat B, bool transpose_q) {
  Context& cx = ctx();
  cudaStream_t st = cx.stream;
  const long m = U.m, k = std::min(U.m, U.n), nr = B.n;
  if (k == 0 || nr == 0) return FLA_SUCCESS;
  const int S = std::max(1, QR_NB / b_alg) * b_alg;
  const long ldy = even_up(m), ldg = even_up(S);
  double* Y = (double*)ws_get(WS_QR_U, sizeof(double) * (size_t)ldy * (size_t)(S + nr));  // [U | B]
  // [Gram | W], Ts, Ts^-1, W2
  double* G = (double*)ws_get(WS_QR_W, sizeof(double) * (size_t)ldg * (size_t)(3 * S + 2 * nr));
  if (!Y || !G) return FLA_FAILURE;
  double* Ts = G + (size_t)ldg * (S + nr);
  double* Tsi = Ts + (size_t)ldg * S;
  double* W2 = Tsi + (size_t)ldg * S;
  op_begin(st);
  const long nsb = (k + S - 1) / S;
  for (long bi = 0; bi < nsb; ++bi) {
    const long jb = transpose_q ? bi * S : (nsb - 1 - bi) * S;
    const int s = (int)std::min<long>(S, k - jb);
    const long M = m - jb;
    double* Bj = B.p + jb;
    if (unit_lower_copy(U.p + jb + jb * U.ld, U.ld, Y, ldy, M, s, st) != FLA_SUCCESS) return FLA_FAILURE;
    FB_CK(cudaMemcpy2DAsync(Y + (size_t)ldy * s, sizeof(double) * ldy, Bj, sizeof(double) * B.ld,
                            sizeof(double) * M, nr, cudaMemcpyDeviceToDevice, st));
    if (gemm_f64(st, true, false, s, s + nr, M, 1.0, Y, ldy, Y, ldy, 0.0, G, ldg) != FLA_SUCCESS)
      return FLA_FAILURE;
    assemble_t_kernel<<<s, 128, 0, st>>>(T.p + jb * T.ld, T.ld, b_alg, G, ldg, s, Ts, ldg);
    count_launch();
    // W2 := Ts^-T W (Q^T) or Ts^-1 W (Q), through the explicit inverse
    double* W = G + (size_t)ldg * s;
    if (tri_inverse(Ts, ldg, s, false, false, Tsi, ldg, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (gemm_f64(st, transpose_q, false, s, nr, s, 1.0, Tsi, ldg, W, ldg, 0.0, W2, ldg) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (gemm_f64(st, false, false, M, nr, s, -1.0, Y, ldy, W2, ldg, 1.0, Bj, B.ld) != FLA_SUCCESS)
      return FLA_FAILURE;
  }
  op_end(st);
  return FLA_SUCCESS;
}

int recover_tau_dev(DMat T, int b_alg, long k, double* t, long inct, bool invert, cudaStream_t st) {
  if (k <= 0) return FLA_SUCCESS;
  recover_tau_kernel<<<(unsigned)((k + 127) / 128), 128, 0, st>>>(T.p, T.ld, b_alg, (int)k, t, inct,
                                                                 invert ? 1 : 0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

}  // namespace fb

using namespace fb;

namespace {
void qr_ensure_init() {
  if (!ctx().initialized) FLA_Init();
}
DMat dm(const Staged& s) {
  DMat d;
  d.p = (double*)s.dev;
  d.ld = s.ld;
  d.m = s.m;
  d.n = s.n;
  return d;
}
}  // namespace

extern "C" {

// src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_create_T.c:13-51
FLA_Error FLA_QR_UT_create_T(FLA_Obj A, FLA_Obj* T) {
  qr_ensure_init();
  FB_REQUIRE(A.base != nullptr && T != nullptr, "FLA_QR_UT_create_T", "null object");
  dim_t mn = A.m < A.n ? A.m : A.n;
  dim_t b_alg = (dim_t)(128 * 0.25);  // FLA_Query_blocksize * FLA_QR_INNER_TO_OUTER_B_RATIO
  if (b_alg > mn) b_alg = mn;
  return FLA_Obj_create(A.base->datatype, b_alg, A.n, 0, 0, T);
}

// src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT.c:15-28 (+ FLA_QR_UT_check:
// T is b x width(A), b >= 1 when A is not empty).
FLA_Error FLA_QR_UT(FLA_Obj A, FLA_Obj T) {
  qr_ensure_init();
  FB_REQUIRE(A.base && T.base, "FLA_QR_UT", "null object");
  FB_REQUIRE(A.base->datatype == FLA_DOUBLE && T.base->datatype == FLA_DOUBLE, "FLA_QR_UT",
             "objects must be FLA_DOUBLE");
  FB_REQUIRE(T.n == A.n, "FLA_QR_UT", "width of T must equal width of A");
  const long mn = std::min<long>(A.m, A.n);
  if (mn == 0) return FLA_SUCCESS;
  FB_REQUIRE(T.m >= 1, "FLA_QR_UT", "T must have at least one row");
  Staged sa, stt;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(T, WS_STAGE_B, &stt, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (qr_ut_dev(dm(sa), dm(stt), (int)T.m) != FLA_SUCCESS) return FLA_FAILURE;
  if (unstage(sa) != FLA_SUCCESS || unstage(stt) != FLA_SUCCESS || sync_all() != FLA_SUCCESS)
    return FLA_FAILURE;
  return FLA_SUCCESS;
}

// src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_recover_tau.c
FLA_Error FLA_QR_UT_recover_tau(FLA_Obj T, FLA_Obj t) {
  qr_ensure_init();
  FB_REQUIRE(T.base && t.base, "FLA_QR_UT_recover_tau", "null object");
  const long k = (long)(t.m * t.n);
  if (k == 0) return FLA_SUCCESS;
  FB_REQUIRE(k <= (long)T.n, "FLA_QR_UT_recover_tau", "t longer than the width of T");
  Staged stt, sv;
  if (stage(T, WS_STAGE_B, &stt, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(t, WS_STAGE_P, &sv, false, false) != FLA_SUCCESS) return FLA_FAILURE;
  long inc = (t.n == 1) ? 1 : sv.ld;
  if (recover_tau_dev(dm(stt), (int)T.m, k, (double*)sv.dev, inc, false, ctx().stream) != FLA_SUCCESS)
    return FLA_FAILURE;
  if (unstage(sv) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// src/lapack/util/app/qut/front/flamec/FLA_Apply_Q_UT_create_workspace.c:13-25
FLA_Error FLA_Apply_Q_UT_create_workspace(FLA_Obj T, FLA_Obj B, FLA_Obj* W) {
  qr_ensure_init();
  FB_REQUIRE(T.base && B.base && W, "FLA_Apply_Q_UT_create_workspace", "null object");
  dim_t nW = B.m > B.n ? B.m : B.n;
  return FLA_Obj_create(T.base->datatype, T.m, nW, 0, 0, W);
}

// src/lapack/util/app/qut/front/flamec/FLA_Apply_Q_UT.c:16-28
FLA_Error FLA_Apply_Q_UT(FLA_Side side, FLA_Trans trans, FLA_Direct direct, FLA_Store storev,
                         FLA_Obj A, FLA_Obj T, FLA_Obj W, FLA_Obj B) {
  qr_ensure_init();
  (void)W;
  FB_REQUIRE(side == FLA_LEFT, "FLA_Apply_Q_UT", "only side = FLA_LEFT is supported");
  FB_REQUIRE(direct == FLA_FORWARD && storev == FLA_COLUMNWISE, "FLA_Apply_Q_UT",
             "only FLA_FORWARD / FLA_COLUMNWISE (QR_UT storage) is supported");
  FB_REQUIRE(trans == FLA_NO_TRANSPOSE || trans == FLA_TRANSPOSE || trans == FLA_CONJ_TRANSPOSE,
             "FLA_Apply_Q_UT", "invalid trans value");
  FB_REQUIRE(A.base && T.base && B.base, "FLA_Apply_Q_UT", "null object");
  FB_REQUIRE(A.base->datatype == FLA_DOUBLE && T.base->datatype == FLA_DOUBLE &&
                 B.base->datatype == FLA_DOUBLE,
             "FLA_Apply_Q_UT", "objects must be FLA_DOUBLE");
  FB_REQUIRE(B.m == A.m && T.n >= std::min(A.m, A.n), "FLA_Apply_Q_UT", "nonconformal objects");
  if (B.n == 0 || std::min(A.m, A.n) == 0) return FLA_SUCCESS;
  Staged sa, stt, sb;
  if (stage(A, WS_STAGE_A, &sa, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(T, WS_STAGE_P, &stt, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS) return FLA_FAILURE;
  if (apply_q_dev(dm(sa), dm(stt), (int)T.m, dm(sb), trans != FLA_NO_TRANSPOSE) != FLA_SUCCESS)
    return FLA_FAILURE;
  if (unstage(sb) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// src/map/lapack2flamec/FLA_geqrf.c:24-88 with dgeqrf_check
// (src/map/common/lapackcheck/dgeqrf_check.c): tau is LAPACK's, i.e. the
// reciprocal of the UT transform's diagonal of T.
int dgeqrf_(int* m, int* n, double* a, int* lda, double* tau, double* work, int* lwork, int* info) {
  *info = 0;
  const int nb = 32;
  if (work) work[0] = (double)((*n > 0 ? *n : 1) * nb);
  const bool lquery = (*lwork == -1);
  if (*m < 0) { *info = -1; }
  else if (*n < 0) { *info = -2; }
  else if (*lda < std::max(1, *m)) { *info = -4; }
  else if (*lwork < std::max(1, *n) && !lquery) { *info = -7; }
  if (*info != 0) {
    std::printf("lapack2flame: On entry to %6s, parameter number %2i had an illegal value\n", "DGEQRF",
                -*info);
    return FLA_FAILURE;
  }
  if (lquery) return 0;
  const int k = std::min(*m, *n);
  if (k == 0) {
    if (work) work[0] = 1.0;
    return 0;
  }
  qr_ensure_init();
  FLA_Base_obj ba;
  std::memset(&ba, 0, sizeof(ba));
  ba.datatype = FLA_DOUBLE;
  ba.elemtype = FLA_SCALAR;
  ba.m = *m;
  ba.n = *n;
  ba.rs = 1;
  ba.cs = *lda;
  ba.buffer = a;
  FLA_Obj A;
  A.offm = A.offn = 0;
  A.m = *m;
  A.n = *n;
  A.m_inner = A.m;
  A.n_inner = A.n;
  A.base = &ba;
  Staged sa;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS) return FLA_FAILURE;
  const int b_alg = std::min(32, k);
  const long ldt = even_up(b_alg);
  double* T = (double*)ws_get(WS_STAGE_B, sizeof(double) * (size_t)ldt * (*n));
  const bool host_tau = !is_device_ptr(tau);
  double* dtau = host_tau ? (double*)ws_get(WS_STAGE_P, sizeof(double) * k) : tau;
  if (!T || !dtau) return FLA_FAILURE;
  FB_CK(cudaMemsetAsync(T, 0, sizeof(double) * (size_t)ldt * (*n), ctx().stream));
  DMat Tm;
  Tm.p = T;
  Tm.ld = ldt;
  Tm.m = b_alg;
  Tm.n = *n;
  if (qr_ut_dev(dm(sa), Tm, b_alg) != FLA_SUCCESS) return FLA_FAILURE;
  if (recover_tau_dev(Tm, b_alg, k, dtau, 1, true, ctx().stream) != FLA_SUCCESS) return FLA_FAILURE;
  if (unstage(sa) != FLA_SUCCESS) return FLA_FAILURE;
  if (host_tau) FB_CK(cudaMemcpyAsync(tau, dtau, sizeof(double) * k, cudaMemcpyDeviceToHost, ctx().stream));
  if (sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return 0;
}

}  // extern "C"
