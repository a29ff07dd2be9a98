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
constexpr int QR_NBMAX = 64;
constexpr size_t QR_SMEM_CAP = 200 * 1024;

struct QrPanelArgs {
  double* P;       // panel, column-major (row k, col k of A)
  long ld;
  int M, nb;       // panel rows, columns
  int R, lds, G;   // rows per CTA, SMEM stride, CTAs
  double* Tbig;    // out: nb x nb (ld nb), upper triangle with diagonal
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
          if (c == 0) a.Tbig[col + (long)j * nb] = rj + d;  // t01 = a10t^T + A20^T u21
        } else if (c == 0) {
          a.Tbig[j + (long)j * nb] = s_tau;
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

// Copy the b_alg x b_alg diagonal blocks of Tbig (nb x nb) into T's columns
// [k, k+nb) (T is b_alg x n, ld ldt); only the upper triangles.
__global__ void extract_t_blocks_kernel(const double* __restrict__ Tbig, int nb, int cols, double* T,
                                        long ldt, int b_alg) {
  const int j = blockIdx.x;           // panel column
  const int i = threadIdx.x;          // row within its T block
  if (j >= cols || i >= b_alg) return;
  const int blk0 = (j / b_alg) * b_alg;
  const int r = blk0 + i;             // row of Tbig
  if (r <= j) T[i + (long)j * ldt] = Tbig[r + (long)j * nb];
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

// A := QR in place (A m x n); T (b_alg x n, ld ldt) receives the T blocks.
int qr_ut_dev(DMat A, DMat T, int b_alg) {
  set_qr_attrs();
  Context& cx = ctx();
  cudaStream_t st = cx.stream;
  const long m = A.m, n = A.n, mn = std::min(m, n);
  if (mn == 0) return FLA_SUCCESS;
  const int NBQ = std::max(1, QR_NBMAX / b_alg) * b_alg;
  QrGeom g0 = qr_geom(m, NBQ);
  if ((size_t)g0.lds * NBQ * 8 + NBQ * 8 > QR_SMEM_CAP || g0.G > cx.num_sms) {
    set_last_error("FLA_QR_UT: panel too tall for the cooperative panel kernel");
    return FLA_FAILURE;
  }
  // workspace: panel exchange, Tbig, Uw (m x NBQ), W (NBQ x n)
  const int GMAX = cx.num_sms;
  size_t b_part = sizeof(double) * (size_t)2 * GMAX * (NBQ + 1);
  size_t b_rowj = sizeof(double) * 2 * (NBQ + 1);
  size_t b_tbig = sizeof(double) * NBQ * NBQ;
  char* ws = (char*)ws_get(WS_PANEL, b_part + b_rowj + b_tbig + 1024);
  const long ldu = even_up(m);
  const long ldw = even_up(NBQ);
  double* Uw = (double*)ws_get(WS_MISC, sizeof(double) * (size_t)ldu * NBQ);
  double* W = (double*)ws_get(WS_MISC2, sizeof(double) * (size_t)ldw * std::max<long>(n, 1));
  if (!ws || !Uw || !W) return FLA_FAILURE;
  double* part = (double*)ws;
  double* part_ss = part + (size_t)2 * GMAX * NBQ;
  double* rowj = (double*)(ws + b_part);
  double* Tbig = (double*)(ws + b_part + b_rowj + 256 - ((b_part + b_rowj) % 256));
  unsigned* bar = (unsigned*)(cx.d_status + ST_BAR);
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;

  for (long k = 0; k < mn; k += NBQ) {
    const int b = (int)std::min<long>(NBQ, mn - k);
    const long M = m - k;
    QrGeom g = qr_geom(M, NBQ);
    QrPanelArgs pa;
    pa.P = A.p + k + k * A.ld;
    pa.ld = A.ld;
    pa.M = (int)M;
    pa.nb = b;
    pa.R = g.R;
    pa.lds = g.lds;
    pa.G = g.G;
    pa.Tbig = Tbig;
    pa.part = part;
    pa.part_ss = part_ss;
    pa.rowj = rowj;
    pa.bar = bar;
    pa.err = cx.d_status + ST_ERROR;
    FB_CK(cudaMemsetAsync(bar, 0, sizeof(unsigned), st));
    const size_t smem = (size_t)g.lds * b * 8 + (size_t)b * 8;
    void* args[] = {&pa};
    const int ps = prof_begin(st);
    FB_CK(cudaLaunchCooperativeKernel((void*)qr_panel_kernel, dim3(g.G), dim3(QR_THREADS), args, smem, st));
    prof_end(ps, st, PROF_PANEL, 0.0);
    count_launch();
    extract_t_blocks_kernel<<<b, std::max(32, b_alg), 0, st>>>(Tbig, b, b, T.p + k * T.ld, T.ld, b_alg);
    count_launch();
    const long n2 = n - k - b;
    if (n2 <= 0) continue;
    // B := (I - U Tbig^-T U^T) B for B = A(k:m, k+b:n)
    const unsigned nthr = 256;
    form_unit_lower_kernel<<<(unsigned)((M * b + nthr - 1) / nthr), nthr, 0, st>>>(pa.P, A.ld, Uw, ldu,
                                                                                   (int)M, b);
    count_launch();
    double* B = A.p + k + (k + b) * A.ld;
    if (gemm_f64(st, true, false, b, n2, M, 1.0, Uw, ldu, B, A.ld, 0.0, W, ldw) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (trsm_block(Tbig, b, W, ldw, b, n2, false, true, false, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (gemm_f64(st, false, false, M, n2, b, -1.0, Uw, ldu, W, ldw, 1.0, B, A.ld) != FLA_SUCCESS)
      return FLA_FAILURE;
  }
  int info;
  return status_read(&info);
}

// B := Q^T B (transpose_q) or Q B for Q = H(0) H(1) ... from the UT
// representation in U (m x k, below the diagonal) and T (b_alg x k).
int apply_q_dev(DMat U, DMat T, int b_alg, DMat B, bool transpose_q) {
  Context& cx = ctx();
  cudaStream_t st = cx.stream;
  const long m = U.m, k = std::min(U.m, U.n), nr = B.n;
  if (k == 0 || nr == 0) return FLA_SUCCESS;
  const long ldu = even_up(m), ldw = even_up(b_alg);
  double* Uw = (double*)ws_get(WS_MISC, sizeof(double) * (size_t)ldu * b_alg);
  double* W = (double*)ws_get(WS_MISC2, sizeof(double) * (size_t)ldw * nr);
  if (!Uw || !W) return FLA_FAILURE;
  op_begin(st);
  const long nblk = (k + b_alg - 1) / b_alg;
  for (long bi = 0; bi < nblk; ++bi) {
    const long jb = transpose_q ? bi * b_alg : (nblk - 1 - bi) * b_alg;
    const int b = (int)std::min<long>(b_alg, k - jb);
    const long M = m - jb;
    const unsigned nthr = 256;
    form_unit_lower_kernel<<<(unsigned)((M * b + nthr - 1) / nthr), nthr, 0, st>>>(
        U.p + jb + jb * U.ld, U.ld, Uw, ldu, (int)M, b);
    count_launch();
    double* Bj = B.p + jb;
    if (gemm_f64(st, true, false, b, nr, M, 1.0, Uw, ldu, Bj, B.ld, 0.0, W, ldw) != FLA_SUCCESS)
      return FLA_FAILURE;
    // W := T^-T W (Q^T) or T^-1 W (Q); T block upper triangular
    if (trsm_block(T.p + jb * T.ld, T.ld, W, ldw, b, nr, false, transpose_q, false, st) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (gemm_f64(st, false, false, M, nr, b, -1.0, Uw, ldu, W, ldw, 1.0, Bj, B.ld) != FLA_SUCCESS)
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
  ba.elemtype = FLA_MATRIX;
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
