// The user-side steps after FLA_QR_UT: least-squares solve, explicit Q,
// the T blocks of a LAPACK tau vector, and the lapack2flame dormqr_ /
// dorgqr_ entry points.  All run on the Apply_Q_UT engine of qr.cu (block
// reflectors applied with two DMMA GEMMs and a small triangular solve per
// 32-column block) and the blocked triangular solve of lu.cu.
//
// Reference interfaces:
//   FLA_QR_UT_solve   src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_solve.c:13-49
//   FLA_QR_UT_form_Q  src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_form_Q.c:13-86
//   FLA_Accum_T_UT    src/lapack/util/accum/tut/front/flamec/FLA_Accum_T_UT.c:13
//                     (T = striu(U^T U) + diag(t))
//   dormqr_           src/map/lapack2flamec/FLA_ormqr.c:35-97
//   dorgqr_           src/map/lapack2flamec/FLA_orgqr.c:30-80
#include <algorithm>
#include <cstring>

#include "common.h"

namespace fb {

int apply_q_dev(DMat U, DMat T, int b_alg, DMat B, bool transpose_q);

namespace {

constexpr int ACC_THREADS = 256;

// T(:, c) for one column c of the reflector block holding it: T(r - c0, c)
// = u_r^T u_c for the earlier columns r of the block (u_j unit at row j, A
// below, zero above), T(c - c0, c) = t[c] (libflame's tau, the reciprocal of
// LAPACK's), zeros below the diagonal of the block.
__global__ void __launch_bounds__(ACC_THREADS) accum_t_kernel(const double* __restrict__ A, long lda, long m,
                                                               const double* __restrict__ t, long inct,
                                                               int invert_tau, double* T, long ldt, int b) {
  const int c = blockIdx.x;
  const int c0 = (c / b) * b;
  __shared__ double red[ACC_THREADS / 32];
  for (int r = c0; r < c; ++r) {
    double s = 0.0;
    for (long i = c + 1 + threadIdx.x; i < m; i += ACC_THREADS) s = fma(A[i + r * lda], A[i + (long)c * lda], s);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double v = 0.0;
      for (int w = 0; w < ACC_THREADS / 32; ++w) v += red[w];
      T[(r - c0) + (long)c * ldt] = A[c + r * lda] + v;  // u_r(c) * 1 + sum below
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < b; i += ACC_THREADS) {
    const int row = c0 + i;
    if (row == c) {
      double v = t[(long)c * inct];
      if (invert_tau && v != 0.0) v = 1.0 / v;
      T[i + (long)c * ldt] = v;
    } else if (row > c) {
      T[i + (long)c * ldt] = 0.0;
    }
  }
}

// X := the first n columns of the m x m identity.
__global__ void set_identity_kernel(double* X, long ldx, long m, long n) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= m * n) return;
  const long j = idx / m, i = idx - j * m;
  X[i + j * ldx] = (i == j) ? 1.0 : 0.0;
}

__global__ void copy_cols_kernel(const double* __restrict__ S, long lds, double* __restrict__ D, long ldd, long m,
                                 long n) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= m * n) return;
  const long j = idx / m, i = idx - j * m;
  D[i + j * ldd] = S[i + j * lds];
}

long even_up(long x) { return (x + 1) & ~1L; }

void ensure_init() {
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

DMat dmat(double* p, long ld, long m, long n) {
  DMat d;
  d.p = p;
  d.ld = ld;
  d.m = m;
  d.n = n;
  return d;
}

}  // namespace

int set_identity_dev(DMat X, cudaStream_t st) {
  const long total = X.m * X.n;
  if (total <= 0) return FLA_SUCCESS;
  set_identity_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(X.p, X.ld, X.m, X.n);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

int copy_dev(const DMat& S, DMat D, cudaStream_t st) {
  const long total = S.m * S.n;
  if (total <= 0) return FLA_SUCCESS;
  copy_cols_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(S.p, S.ld, D.p, D.ld, S.m, S.n);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// T (b x k) := the UT-transform blocks of the k reflectors stored below the
// diagonal of U (m x k) with scalars t (LAPACK's tau when invert_tau).
int accum_t_dev(DMat U, const double* t, long inct, bool invert_tau, DMat T, int b, cudaStream_t st) {
  const long k = std::min(U.m, U.n);
  if (k <= 0) return FLA_SUCCESS;
  accum_t_kernel<<<(unsigned)k, ACC_THREADS, 0, st>>>(U.p, U.ld, U.m, t, inct, invert_tau ? 1 : 0, T.p, T.ld, b);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// C := op(Q) C (left) or C op(Q) (right) for the Q of the k reflectors in
// U (order = rows of U) and T blocks; the right side runs as the left
// product on C^T, transposed into a workspace and back.
int apply_q_side_dev(bool left, bool transpose_q, DMat U, DMat T, int b, DMat C, cudaStream_t st) {
  if (left) return apply_q_dev(U, T, b, C, transpose_q);
  // C Q = (Q^T C^T)^T, C Q^T = (Q C^T)^T
  const long m = C.m, n = C.n;
  const long ldw = even_up(n);
  double* W = (double*)ws_get(WS_FB, sizeof(double) * (size_t)ldw * (size_t)std::max<long>(m, 1));
  if (!W) return FLA_FAILURE;
  if (transpose_dev(C.p, C.ld, W, ldw, m, n, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (apply_q_dev(U, T, b, dmat(W, ldw, n, m), !transpose_q) != FLA_SUCCESS) return FLA_FAILURE;
  return transpose_dev(W, ldw, C.p, C.ld, n, m, false, st);
}

}  // namespace fb

using namespace fb;

extern "C" {

// src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_solve.c:13-49 (+
// FLA_QR_UT_solve_check): Y := Q^T B; X := inv(triu(A_T)) Y_T, A_T the top
// n x n block of the m x n factor (m >= n).  B is left unchanged.
FLA_Error FLA_QR_UT_solve(FLA_Obj A, FLA_Obj T, FLA_Obj B, FLA_Obj X) {
  ensure_init();
  FB_REQUIRE(A.base && T.base && B.base && X.base, "FLA_QR_UT_solve", "null object");
  FB_REQUIRE(A.base->datatype == FLA_DOUBLE && T.base->datatype == FLA_DOUBLE &&
                 B.base->datatype == FLA_DOUBLE && X.base->datatype == FLA_DOUBLE,
             "FLA_QR_UT_solve", "objects must be FLA_DOUBLE");
  FB_REQUIRE(T.n == std::min(A.m, A.n), "FLA_QR_UT_solve", "width of T must equal min_dim(A)");
  FB_REQUIRE(X.m == A.n && B.m == A.m && X.n == B.n, "FLA_QR_UT_solve", "nonconformal objects");
  FB_REQUIRE(A.m >= A.n, "FLA_QR_UT_solve", "A must have at least as many rows as columns");
  const long m = A.m, n = A.n, nr = B.n;
  if (nr == 0 || n == 0) return FLA_SUCCESS;
  Staged sa, stt, sx;
  if (stage(A, WS_STAGE_A, &sa, true, true) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(T, WS_STAGE_P, &stt, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(X, WS_STAGE_X, &sx, false, true) != FLA_SUCCESS) return FLA_FAILURE;
  cudaStream_t st = ctx().stream;
  op_begin(st);
  // Y := B in a workspace (B may be a host buffer)
  const long ldy = even_up(m);
  double* Y = (double*)ws_get(WS_STAGE_B, sizeof(double) * (size_t)ldy * (size_t)nr);
  if (!Y) return FLA_FAILURE;
  FB_CK(cudaMemcpy2DAsync(Y, sizeof(double) * ldy, FLA_Obj_buffer_at_view(B), sizeof(double) * B.base->cs,
                          sizeof(double) * m, nr, cudaMemcpyDefault, st));
  DMat a = dm(sa), y = dmat(Y, ldy, m, nr);
  if (apply_q_dev(a, dm(stt), (int)T.m, y, true) != FLA_SUCCESS) return FLA_FAILURE;
  if (trsm_left_dev(a.sub(0, 0, n, n), y.sub(0, 0, n, nr), false, false, false, st) != FLA_SUCCESS)
    return FLA_FAILURE;
  if (copy_dev(y.sub(0, 0, n, nr), dm(sx), st) != FLA_SUCCESS) return FLA_FAILURE;
  op_end(st);
  if (unstage(sx) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_form_Q.c:13-86 (+
// FLA_QR_UT_form_Q_check: Q has as many rows as A): Q := the first
// width(Q) columns of H(0) H(1) ... H(k-1), k = width(T).  Q may be (a view
// of) A itself: the reflectors are then copied out first.
FLA_Error FLA_QR_UT_form_Q(FLA_Obj A, FLA_Obj T, FLA_Obj Q) {
  ensure_init();
  FB_REQUIRE(A.base && T.base && Q.base, "FLA_QR_UT_form_Q", "null object");
  FB_REQUIRE(A.base->datatype == FLA_DOUBLE && T.base->datatype == FLA_DOUBLE &&
                 Q.base->datatype == FLA_DOUBLE,
             "FLA_QR_UT_form_Q", "objects must be FLA_DOUBLE");
  FB_REQUIRE(Q.m == A.m, "FLA_QR_UT_form_Q", "Q must have as many rows as A");
  const long m = A.m;
  const long k = std::min<long>((long)T.n, std::min<long>(A.m, A.n));
  if (Q.n == 0 || m == 0) return FLA_SUCCESS;
  Staged sa, stt, sq;
  if (stage(A, WS_STAGE_A, &sa, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(T, WS_STAGE_P, &stt, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  const bool same_base = (A.base == Q.base);
  cudaStream_t st = ctx().stream;
  DMat u = dm(sa).sub(0, 0, m, k);
  if (same_base) {
    // the reflectors live in Q's storage: copy them out before Q := I
    const long ldu = even_up(m);
    double* U = (double*)ws_get(WS_REPACK, sizeof(double) * (size_t)ldu * (size_t)std::max<long>(k, 1));
    if (!U) return FLA_FAILURE;
    if (copy_dev(u, dmat(U, ldu, m, k), st) != FLA_SUCCESS) return FLA_FAILURE;
    u = dmat(U, ldu, m, k);
    if (stage(Q, WS_STAGE_X, &sq, false, false) != FLA_SUCCESS) return FLA_FAILURE;
  } else {
    if (stage(Q, WS_STAGE_X, &sq, false, false) != FLA_SUCCESS) return FLA_FAILURE;
  }
  op_begin(st);
  DMat q = dm(sq);
  if (set_identity_dev(q, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (k > 0 && apply_q_dev(u, dm(stt).sub(0, 0, T.m, k), (int)T.m, q, false) != FLA_SUCCESS) return FLA_FAILURE;
  op_end(st);
  if (unstage(sq) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// FLA_Accum_T_UT(FLA_FORWARD, FLA_COLUMNWISE, A, t, T) as lapack2flame uses
// it (src/map/lapack2flamec/FLA_ormqr.c:66, FLA_orgqr.c:48): T (b x k)
// receives, block by block, striu(U^T U) + diag(t) for the reflectors
// stored below the diagonal of A (m x k) and libflame's t (1/tau of LAPACK).
FLA_Error FLA_Accum_T_UT(FLA_Direct direct, FLA_Store storev, FLA_Obj A, FLA_Obj t, FLA_Obj T) {
  ensure_init();
  FB_REQUIRE(direct == FLA_FORWARD && storev == FLA_COLUMNWISE, "FLA_Accum_T_UT",
             "only FLA_FORWARD / FLA_COLUMNWISE (QR_UT storage) is supported");
  FB_REQUIRE(A.base && t.base && T.base, "FLA_Accum_T_UT", "null object");
  FB_REQUIRE(A.base->datatype == FLA_DOUBLE && t.base->datatype == FLA_DOUBLE && T.base->datatype == FLA_DOUBLE,
             "FLA_Accum_T_UT", "objects must be FLA_DOUBLE");
  const long k = std::min<long>(A.m, A.n);
  FB_REQUIRE((long)(t.m * t.n) >= k && (long)T.n >= k && T.m >= 1, "FLA_Accum_T_UT", "nonconformal objects");
  if (k == 0) return FLA_SUCCESS;
  Staged sa, sv, stt;
  if (stage(A, WS_STAGE_A, &sa, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(t, WS_STAGE_X, &sv, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(T, WS_STAGE_B, &stt, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  const long inc = (t.n == 1) ? 1 : sv.ld;
  if (accum_t_dev(dm(sa), (const double*)sv.dev, inc, false, dm(stt), (int)T.m, ctx().stream) != FLA_SUCCESS)
    return FLA_FAILURE;
  if (unstage(stt) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

}  // extern "C"

namespace {

bool lsame1(const char* a, char c) { return a && (a[0] == c || a[0] == (char)(c + ('a' - 'A'))); }

int xerbla_ret(const char* name, int* info) {
  std::printf("lapack2flame: On entry to %6s, parameter number %2i had an illegal value\n", name, -*info);
  return FLA_FAILURE;
}

FLA_Obj raw(void* buf, long m, long n, long ld, FLA_Base_obj* base) {
  std::memset(base, 0, sizeof(*base));
  base->datatype = FLA_DOUBLE;
  base->elemtype = FLA_SCALAR;
  base->m = (dim_t)m;
  base->n = (dim_t)n;
  base->rs = 1;
  base->cs = (dim_t)(ld > 0 ? ld : 1);
  base->buffer = buf;
  FLA_Obj o;
  o.offm = o.offn = 0;
  o.m = (dim_t)m;
  o.n = (dim_t)n;
  o.m_inner = o.m;
  o.n_inner = o.n;
  o.base = base;
  return o;
}

// tau (host or device, k entries) on the device, and the T blocks of the
// k reflectors of U built from it (LAPACK tau, inverted on the fly).
int lapack_t_blocks(DMat U, const double* tau, long k, DMat* Tout, int* bout) {
  cudaStream_t st = ctx().stream;
  const int b = (int)std::min<long>(32, k);
  const double* dtau = tau;
  if (!is_device_ptr(tau)) {
    double* d = (double*)ws_get(WS_STAGE_P, sizeof(double) * (size_t)k);
    if (!d) return FLA_FAILURE;
    FB_CK(cudaMemcpyAsync(d, tau, sizeof(double) * k, cudaMemcpyHostToDevice, st));
    dtau = d;
  }
  const long ldt = even_up(b);
  double* Tb = (double*)ws_get(WS_LP4, sizeof(double) * (size_t)ldt * (size_t)k);
  if (!Tb) return FLA_FAILURE;
  DMat t = dmat(Tb, ldt, b, k);
  if (accum_t_dev(U, dtau, 1, true, t, b, st) != FLA_SUCCESS) return FLA_FAILURE;
  *Tout = t;
  *bout = b;
  return FLA_SUCCESS;
}

}  // namespace

extern "C" {

// src/map/lapack2flamec/FLA_ormqr.c:35-97 with dormqr_check
// (src/map/common/lapackcheck/dormqr_check.c): C := op(Q) C or C op(Q) for
// the Q of k reflectors from dgeqrf_ (A, LAPACK tau).  work only receives
// the workspace query answer; the library keeps its own workspace.
int dormqr_(char* side, char* trans, int* m, int* n, int* k, double* a, int* lda, double* tau, double* c,
            int* ldc, double* work, int* lwork, int* info) {
  *info = 0;
  const bool left = lsame1(side, 'L'), notran = lsame1(trans, 'N');
  const bool lquery = (*lwork == -1);
  const int nq = left ? *m : *n, nw = left ? *n : *m;
  if (!left && !lsame1(side, 'R')) *info = -1;
  else if (!notran && !lsame1(trans, 'T')) *info = -2;
  else if (*m < 0) *info = -3;
  else if (*n < 0) *info = -4;
  else if (*k < 0 || *k > nq) *info = -5;
  else if (*lda < std::max(1, nq)) *info = -7;
  else if (*ldc < std::max(1, *m)) *info = -10;
  else if (*lwork < std::max(1, nw) && !lquery) *info = -12;
  if (*info == 0 && work) work[0] = (double)(std::max(1, nw) * 32);
  if (*info != 0) return xerbla_ret("DORMQR", info);
  if (lquery) return 0;
  if (*m == 0 || *n == 0 || *k == 0) {
    if (work) work[0] = 1.0;
    return 0;
  }
  ensure_init();
  FLA_Base_obj ba, bc;
  FLA_Obj A = raw(a, nq, *k, *lda, &ba), C = raw(c, *m, *n, *ldc, &bc);
  Staged sa, sc;
  if (stage(A, WS_STAGE_A, &sa, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (stage(C, WS_STAGE_B, &sc) != FLA_SUCCESS) return FLA_FAILURE;
  cudaStream_t st = ctx().stream;
  op_begin(st);
  DMat T;
  int b = 0;
  if (lapack_t_blocks(dm(sa), tau, *k, &T, &b) != FLA_SUCCESS) return FLA_FAILURE;
  if (apply_q_side_dev(left, !notran, dm(sa), T, b, dm(sc), st) != FLA_SUCCESS) return FLA_FAILURE;
  op_end(st);
  if (unstage(sc) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return 0;
}

// src/map/lapack2flamec/FLA_orgqr.c:30-80 with dorgqr_check
// (src/map/common/lapackcheck/dorgqr_check.c): A (m x n) := the first n
// columns of H(1) ... H(k), the reflectors being A's first k columns as
// dgeqrf_ left them, with LAPACK's tau.
int dorgqr_(int* m, int* n, int* k, double* a, int* lda, double* tau, double* work, int* lwork, int* info) {
  *info = 0;
  if (work) work[0] = (double)(std::max(1, *n) * 32);
  const bool lquery = (*lwork == -1);
  if (*m < 0) *info = -1;
  else if (*n < 0 || *n > *m) *info = -2;
  else if (*k < 0 || *k > *n) *info = -3;
  else if (*lda < std::max(1, *m)) *info = -5;
  else if (*lwork < std::max(1, *n) && !lquery) *info = -8;
  if (*info != 0) return xerbla_ret("DORGQR", info);
  if (lquery) return 0;
  if (*n <= 0) {
    if (work) work[0] = 1.0;
    return 0;
  }
  ensure_init();
  FLA_Base_obj ba;
  FLA_Obj A = raw(a, *m, *n, *lda, &ba);
  Staged sa;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS) return FLA_FAILURE;
  cudaStream_t st = ctx().stream;
  op_begin(st);
  DMat ad = dm(sa);
  if (*k > 0) {
    const long ldu = even_up(*m);
    double* U = (double*)ws_get(WS_REPACK, sizeof(double) * (size_t)ldu * (size_t)(*k));
    if (!U) return FLA_FAILURE;
    DMat u = dmat(U, ldu, *m, *k);
    if (copy_dev(ad.sub(0, 0, *m, *k), u, st) != FLA_SUCCESS) return FLA_FAILURE;
    DMat T;
    int b = 0;
    if (lapack_t_blocks(u, tau, *k, &T, &b) != FLA_SUCCESS) return FLA_FAILURE;
    if (set_identity_dev(ad, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (apply_q_dev(u, T, b, ad, false) != FLA_SUCCESS) return FLA_FAILURE;
  } else {
    if (set_identity_dev(ad, st) != FLA_SUCCESS) return FLA_FAILURE;
  }
  op_end(st);
  if (unstage(sa) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return 0;
}

}  // extern "C"
