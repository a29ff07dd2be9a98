// FLA_Obj front ends (FLA_Chol, FLA_LU_piv, FLA_Apply_pivots, solves) and
// the lapack2flame LAPACK entry points, over the device drivers.
#include <algorithm>
#include <climits>
#include <cstring>
#include <vector>

#include "common.h"
#include "mixed.h"

namespace fb {

int trsm_left_dev(DMat T, DMat B, bool lower, bool trans, bool unit, cudaStream_t st);
int laswp_dev(double* A, long ld, int row0, const int* d_piv, int npiv, int c0, int n0, int c1,
              int n1, bool reverse, cudaStream_t st);

// dst := src^T for an m x n src (dst is n x m).  tri = 1: only the upper
// triangle of dst (i <= j) is written.
__global__ void transpose_kernel(const double* __restrict__ src, long lds, double* __restrict__ dst,
                                 long ldd, int m, int n, int tri) {
  __shared__ double tile[32][33];
  const int bx = blockIdx.x * 32, by = blockIdx.y * 32;  // bx over src rows, by over src cols
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = bx + threadIdx.x, c = by + j;
    if (r < m && c < n) tile[j][threadIdx.x] = src[r + (long)c * lds];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int r = by + threadIdx.x, c = bx + j;  // dst(r, c) = src(c, r)
    if (r < n && c < m && (!tri || r <= c)) dst[r + (long)c * ldd] = tile[threadIdx.x][j];
  }
}

int transpose_dev(const double* src, long lds, double* dst, long ldd, long m, long n, bool upper_only,
                  cudaStream_t st) {
  if (m <= 0 || n <= 0) return FLA_SUCCESS;
  dim3 grid((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32)), block(32, 8);
  transpose_kernel<<<grid, block, 0, st>>>(src, lds, dst, ldd, (int)m, (int)n, upper_only ? 1 : 0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

namespace {

__global__ void shift_pivots_kernel(int* p, int n, int delta_sign) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] += delta_sign * (i + 1);
}

bool is_float_type(FLA_Datatype dt) { return dt == FLA_FLOAT || dt == FLA_DOUBLE; }

void ensure_init() {
  if (!ctx().initialized) FLA_Init();
}

DMat to_dmat(const Staged& s) {
  DMat d;
  d.p = (double*)s.dev;
  d.ld = s.ld;
  d.m = s.m;
  d.n = s.n;
  return d;
}

// Pivot vector of an FLA_INT object: device pointer (staged when host).
struct PivStage {
  int* dev = nullptr;
  int* orig = nullptr;
  long n = 0;
  bool host = false;
};
int piv_stage(const FLA_Obj& p, long n, bool copy_in, PivStage* ps) {
  ps->n = n;
  ps->orig = (int*)FLA_Obj_buffer_at_view(p);
  ps->host = !is_device_ptr(p.base->buffer);
  long inc = (long)(p.base->rs);  // column vector: row stride
  if (!ps->host && inc == 1) {
    ps->dev = ps->orig;
    return FLA_SUCCESS;
  }
  int* d = (int*)ws_get(WS_STAGE_P, sizeof(int) * (size_t)(n > 0 ? n : 1));
  if (!d) return FLA_FAILURE;
  ps->dev = d;
  if (copy_in && n > 0) {
    if (inc == 1) {
      FB_CK(cudaMemcpyAsync(d, ps->orig, sizeof(int) * n, cudaMemcpyDefault, ctx().stream));
    } else {
      FB_CK(cudaMemcpy2DAsync(d, sizeof(int), ps->orig, sizeof(int) * inc, sizeof(int), n,
                              cudaMemcpyDefault, ctx().stream));
    }
  }
  return FLA_SUCCESS;
}
int piv_unstage(const FLA_Obj& p, const PivStage& ps) {
  if (ps.dev == ps.orig || ps.n == 0) return FLA_SUCCESS;
  long inc = (long)(p.base->rs);
  if (inc == 1) {
    FB_CK(cudaMemcpyAsync(ps.orig, ps.dev, sizeof(int) * ps.n, cudaMemcpyDefault, ctx().stream));
  } else {
    FB_CK(cudaMemcpy2DAsync(ps.orig, sizeof(int) * inc, ps.dev, sizeof(int), sizeof(int), ps.n,
                            cudaMemcpyDefault, ctx().stream));
  }
  return FLA_SUCCESS;
}

}  // namespace

// Upper Cholesky A = U^T U through the lower factorization of A^T: the
// upper triangle of A is transposed into a workspace, factored there, and
// U = L^T is written back to the upper triangle (the strictly lower part
// of A is left untouched, as FLA_Chol_u_blk_var3 leaves it).
int chol_lower_enqueue(DMat A, cudaStream_t st);
int chol_upper_dev(DMat A, int* info) {
  const long n = A.m;
  *info = -1;
  if (n == 0) return FLA_SUCCESS;
  long ldw = (n + 1) & ~1L;
  double* W = (double*)ws_get(WS_REPACK, sizeof(double) * (size_t)ldw * n);
  if (!W) return FLA_FAILURE;
  cudaStream_t st = ctx().stream;
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;
  if (transpose_dev(A.p, A.ld, W, ldw, n, n, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  DMat Wm;
  Wm.p = W;
  Wm.ld = ldw;
  Wm.m = Wm.n = n;
  if (chol_lower_enqueue(Wm, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (transpose_dev(W, ldw, A.p, A.ld, n, n, true, st) != FLA_SUCCESS) return FLA_FAILURE;
  return status_read(info);
}

}  // namespace fb

using namespace fb;

extern "C" {

// ---------------------------------------------------------------------------
// src/lapack/dec/chol/front/flamec/FLA_Chol.c:16-29 (+ FLA_Chol_check).
// ---------------------------------------------------------------------------
FLA_Error FLA_Chol(FLA_Uplo uplo, FLA_Obj A) {
  ensure_init();
  FB_REQUIRE(uplo == FLA_LOWER_TRIANGULAR || uplo == FLA_UPPER_TRIANGULAR, "FLA_Chol",
             "invalid uplo value");
  FB_REQUIRE(A.base != nullptr && is_float_type(A.base->datatype), "FLA_Chol",
             "object must be a real floating-point matrix");
  FB_REQUIRE(A.m == A.n, "FLA_Chol", "object must be square");
  FB_REQUIRE(A.base->datatype == FLA_DOUBLE, "FLA_Chol",
             "this build factors FLA_DOUBLE objects (FLA_FLOAT goes through the mixed-precision solvers)");
  Staged s;
  if (stage(A, WS_STAGE_A, &s) != FLA_SUCCESS) return FLA_FAILURE;
  int info = -1;
  int r = (uplo == FLA_LOWER_TRIANGULAR) ? chol_lower_dev(to_dmat(s), &info)
                                         : chol_upper_dev(to_dmat(s), &info);
  if (r != FLA_SUCCESS) return FLA_FAILURE;
  if (unstage(s) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return info >= 0 ? info : FLA_SUCCESS;
}

// ---------------------------------------------------------------------------
// src/lapack/dec/lu/piv/front/flamec/FLA_LU_piv.c:16-33 (+ FLA_LU_piv_check:
// p is an integer column vector of length >= min(m,n)).
// ---------------------------------------------------------------------------
FLA_Error FLA_LU_piv(FLA_Obj A, FLA_Obj p) {
  ensure_init();
  FB_REQUIRE(A.base != nullptr && A.base->datatype == FLA_DOUBLE, "FLA_LU_piv",
             "object must be an FLA_DOUBLE matrix");
  FB_REQUIRE(p.base != nullptr && p.base->datatype == FLA_INT, "FLA_LU_piv",
             "pivot object must be FLA_INT");
  const long mn = std::min<long>(A.m, A.n);
  FB_REQUIRE(p.n == 1 && (long)p.m >= mn, "FLA_LU_piv",
             "pivot object must be a column vector of length >= min(m,n)");
  Staged s;
  if (stage(A, WS_STAGE_A, &s) != FLA_SUCCESS) return FLA_FAILURE;
  PivStage ps;
  if (piv_stage(p, mn, false, &ps) != FLA_SUCCESS) return FLA_FAILURE;
  int info = -1;
  if (lu_piv_dev(to_dmat(s), ps.dev, &info) != FLA_SUCCESS) return FLA_FAILURE;
  if (unstage(s) != FLA_SUCCESS || piv_unstage(p, ps) != FLA_SUCCESS || sync_all() != FLA_SUCCESS)
    return FLA_FAILURE;
  return info >= 0 ? info : FLA_SUCCESS;
}

// ---------------------------------------------------------------------------
// src/lapack/util/app/piv/front/flamec/FLA_Apply_pivots.c
// ---------------------------------------------------------------------------
FLA_Error FLA_Apply_pivots(FLA_Side side, FLA_Trans trans, FLA_Obj p, FLA_Obj A) {
  ensure_init();
  FB_REQUIRE(side == FLA_LEFT, "FLA_Apply_pivots", "only side = FLA_LEFT is supported");
  FB_REQUIRE(trans == FLA_NO_TRANSPOSE || trans == FLA_TRANSPOSE, "FLA_Apply_pivots",
             "invalid trans value");
  FB_REQUIRE(p.base != nullptr && p.base->datatype == FLA_INT, "FLA_Apply_pivots",
             "pivot object must be FLA_INT");
  FB_REQUIRE(A.base != nullptr && A.base->datatype == FLA_DOUBLE, "FLA_Apply_pivots",
             "object must be an FLA_DOUBLE matrix");
  const long np = (long)p.m;
  if (np == 0 || A.n == 0) return FLA_SUCCESS;
  Staged s;
  if (stage(A, WS_STAGE_A, &s, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  PivStage ps;
  if (piv_stage(p, np, true, &ps) != FLA_SUCCESS) return FLA_FAILURE;
  if (apply_pivots_dev(to_dmat(s), ps.dev, 0, (int)np - 1, trans == FLA_TRANSPOSE, ctx().stream) !=
      FLA_SUCCESS)
    return FLA_FAILURE;
  if (unstage(s) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// ---------------------------------------------------------------------------
// src/base/flamec/util/lapack/FLA_Shift_pivots_to.c:13-42
// ---------------------------------------------------------------------------
FLA_Error FLA_Shift_pivots_to(FLA_Pivot_type ptype, FLA_Obj p) {
  ensure_init();
  FB_REQUIRE(ptype == FLA_NATIVE_PIVOTS || ptype == FLA_LAPACK_PIVOTS, "FLA_Shift_pivots_to",
             "invalid pivot type");
  FB_REQUIRE(p.base != nullptr && p.base->datatype == FLA_INT, "FLA_Shift_pivots_to",
             "pivot object must be FLA_INT");
  const int sgn = (ptype == FLA_LAPACK_PIVOTS) ? 1 : -1;
  const long n = (long)p.m * (long)p.n;
  int* buf = (int*)FLA_Obj_buffer_at_view(p);
  if (n == 0) return FLA_SUCCESS;
  if (!is_device_ptr(p.base->buffer)) {
    long inc = (long)p.base->rs;
    for (long i = 0; i < (long)p.m; ++i) buf[i * inc] += sgn * (int)(i + 1);
    return FLA_SUCCESS;
  }
  FB_REQUIRE(p.base->rs == 1, "FLA_Shift_pivots_to", "device pivot vector must be contiguous");
  shift_pivots_kernel<<<(unsigned)((p.m + 255) / 256), 256, 0, ctx().stream>>>(buf, (int)p.m, sgn);
  count_launch();
  return sync_all();
}

// ---------------------------------------------------------------------------
// Solves.
// ---------------------------------------------------------------------------
static int copy_into(const FLA_Obj& B, const Staged& X) {
  // X (device, staged or not) := B (host or device view)
  const void* src = FLA_Obj_buffer_at_view(B);
  FB_CK(cudaMemcpy2DAsync(X.dev, (size_t)X.ld * 8, src, (size_t)B.base->cs * 8, (size_t)B.m * 8,
                          (size_t)B.n, cudaMemcpyDefault, ctx().stream));
  return FLA_SUCCESS;
}

static bool same_view(const FLA_Obj& a, const FLA_Obj& b) {
  return a.base == b.base && a.offm == b.offm && a.offn == b.offn && a.m == b.m && a.n == b.n;
}

// src/lapack/dec/chol/front/flamec/FLA_Chol_solve.c:13-35
FLA_Error FLA_Chol_solve(FLA_Uplo uplo, FLA_Obj A, FLA_Obj B, FLA_Obj X) {
  ensure_init();
  FB_REQUIRE(uplo == FLA_LOWER_TRIANGULAR || uplo == FLA_UPPER_TRIANGULAR, "FLA_Chol_solve",
             "invalid uplo value");
  FB_REQUIRE(A.base && B.base && X.base, "FLA_Chol_solve", "null object");
  FB_REQUIRE(A.base->datatype == FLA_DOUBLE && B.base->datatype == FLA_DOUBLE &&
                 X.base->datatype == FLA_DOUBLE,
             "FLA_Chol_solve", "objects must be FLA_DOUBLE");
  FB_REQUIRE(A.m == A.n && B.m == A.m && X.m == B.m && X.n == B.n, "FLA_Chol_solve",
             "nonconformal objects");
  if (B.n == 0 || A.m == 0) return FLA_SUCCESS;
  Staged sa, sx;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS) return FLA_FAILURE;
  bool ident = same_view(B, X);
  if (stage(X, WS_STAGE_B, &sx, ident) != FLA_SUCCESS) return FLA_FAILURE;
  cudaStream_t st = ctx().stream;
  op_begin(st);
  if (!ident && copy_into(B, sx) != FLA_SUCCESS) return FLA_FAILURE;
  DMat a = to_dmat(sa), x = to_dmat(sx);
  int r;
  if (uplo == FLA_LOWER_TRIANGULAR) {
    r = trsm_left_dev(a, x, true, false, false, st);
    if (r == FLA_SUCCESS) r = trsm_left_dev(a, x, true, true, false, st);
  } else {
    r = trsm_left_dev(a, x, false, true, false, st);
    if (r == FLA_SUCCESS) r = trsm_left_dev(a, x, false, false, false, st);
  }
  if (r != FLA_SUCCESS) return FLA_FAILURE;
  op_end(st);
  if (unstage(sx) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// src/lapack/dec/lu/piv/front/flamec/FLA_LU_piv_solve.c:13-29
FLA_Error FLA_LU_piv_solve(FLA_Obj A, FLA_Obj p, FLA_Obj B, FLA_Obj X) {
  ensure_init();
  FB_REQUIRE(A.base && p.base && B.base && X.base, "FLA_LU_piv_solve", "null object");
  FB_REQUIRE(A.base->datatype == FLA_DOUBLE && B.base->datatype == FLA_DOUBLE &&
                 X.base->datatype == FLA_DOUBLE && p.base->datatype == FLA_INT,
             "FLA_LU_piv_solve", "objects must be FLA_DOUBLE (p FLA_INT)");
  FB_REQUIRE(A.m == A.n && B.m == A.m && X.m == B.m && X.n == B.n && (long)p.m >= (long)A.m,
             "FLA_LU_piv_solve", "nonconformal objects");
  if (B.n == 0 || A.m == 0) return FLA_SUCCESS;
  Staged sa, sx;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS) return FLA_FAILURE;
  bool ident = same_view(B, X);
  if (stage(X, WS_STAGE_B, &sx, ident) != FLA_SUCCESS) return FLA_FAILURE;
  PivStage ps;
  if (piv_stage(p, (long)A.m, true, &ps) != FLA_SUCCESS) return FLA_FAILURE;
  cudaStream_t st = ctx().stream;
  op_begin(st);
  if (!ident && copy_into(B, sx) != FLA_SUCCESS) return FLA_FAILURE;
  DMat a = to_dmat(sa), x = to_dmat(sx);
  if (apply_pivots_dev(x, ps.dev, 0, (int)A.m - 1, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (trsm_left_dev(a, x, true, false, true, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (trsm_left_dev(a, x, false, false, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  op_end(st);
  if (unstage(sx) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return FLA_SUCCESS;
}

// ===========================================================================
// LAPACK ABI (src/map/lapack2flamec, src/map/common/lapacksrc/f2c).
// Arguments are checked first like the reference's *_check routines
// (src/map/common/lapackcheck): a bad argument prints the xerbla message,
// sets info = -position and returns FLA_FAILURE.
// ===========================================================================
static bool lsame1(const char* a, char c) {
  return a && (a[0] == c || a[0] == (char)(c + ('a' - 'A')));
}
static int xerbla(const char* name, int pos, int* info) {
  *info = -pos;
  std::printf("lapack2flame: On entry to %6s, parameter number %2i had an illegal value\n", name, pos);
  return FLA_FAILURE;
}

// A raw column-major operand (host or device pointer) as an FLA_Obj view.
static FLA_Obj raw_obj(FLA_Datatype dt, void* buf, long m, long n, long ld, FLA_Base_obj* base) {
  std::memset(base, 0, sizeof(*base));
  base->datatype = dt;
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

// src/map/lapack2flamec/FLA_potrf.c:31-83 with dpotrf_check
int dpotrf_(char* uplo, int* n, double* a, int* lda, int* info) {
  *info = 0;
  bool up = lsame1(uplo, 'U');
  if (!up && !lsame1(uplo, 'L')) return xerbla("DPOTRF", 1, info);
  if (*n < 0) return xerbla("DPOTRF", 2, info);
  if (*lda < std::max(1, *n)) return xerbla("DPOTRF", 4, info);
  if (*n == 0) return 0;
  FLA_Base_obj b;
  FLA_Obj A = raw_obj(FLA_DOUBLE, a, *n, *n, *lda, &b);
  FLA_Error e = FLA_Chol(up ? FLA_UPPER_TRIANGULAR : FLA_LOWER_TRIANGULAR, A);
  if (e == FLA_FAILURE) return FLA_FAILURE;
  *info = (e != FLA_SUCCESS) ? e + 1 : 0;
  return 0;
}

// src/map/lapack2flamec/FLA_getrf.c:32-92 with dgetrf_check: pivots come
// back 1-based (FLA_Shift_pivots_to(FLA_LAPACK_PIVOTS)).
int dgetrf_(int* m, int* n, double* a, int* lda, int* ipiv, int* info) {
  *info = 0;
  if (*m < 0) return xerbla("DGETRF", 1, info);
  if (*n < 0) return xerbla("DGETRF", 2, info);
  if (*lda < std::max(1, *m)) return xerbla("DGETRF", 4, info);
  if (*m == 0 || *n == 0) return 0;
  ensure_init();
  const long mn = std::min(*m, *n);
  FLA_Base_obj b;
  FLA_Obj A = raw_obj(FLA_DOUBLE, a, *m, *n, *lda, &b);
  Staged s;
  if (stage(A, WS_STAGE_A, &s) != FLA_SUCCESS) return FLA_FAILURE;
  bool host = !is_device_ptr(ipiv);
  int* dp = host ? (int*)ws_get(WS_STAGE_P, sizeof(int) * mn) : ipiv;
  if (!dp) return FLA_FAILURE;
  int e = -1;
  if (lu_piv_dev(to_dmat(s), dp, &e) != FLA_SUCCESS) return FLA_FAILURE;
  shift_pivots_kernel<<<(unsigned)((mn + 255) / 256), 256, 0, ctx().stream>>>(dp, (int)mn, 1);
  count_launch();
  if (unstage(s) != FLA_SUCCESS) return FLA_FAILURE;
  if (host) FB_CK(cudaMemcpyAsync(ipiv, dp, sizeof(int) * mn, cudaMemcpyDeviceToHost, ctx().stream));
  if (sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  *info = (e >= 0) ? e + 1 : 0;
  return 0;
}

// Device-side solves shared by dpotrs_/dposv_ and dgetrs_/dgesv_.
static int potrs_dev(bool up, DMat a, DMat x) {
  cudaStream_t st = ctx().stream;
  if (!up) {
    if (trsm_left_dev(a, x, true, false, false, st) != FLA_SUCCESS) return FLA_FAILURE;
    return trsm_left_dev(a, x, true, true, false, st);
  }
  if (trsm_left_dev(a, x, false, true, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  return trsm_left_dev(a, x, false, false, false, st);
}

// LAPACK 1-based pivots -> relative zero-based (device, in workspace).
__global__ void lapack_to_rel_kernel(const int* ip, int* rel, int n) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rel[i] = ip[i] - (i + 1);
}

static int getrs_dev(bool trans, DMat a, const int* d_rel, DMat x) {
  cudaStream_t st = ctx().stream;
  const int n = (int)a.m;
  if (!trans) {
    if (apply_pivots_dev(x, d_rel, 0, n - 1, false, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (trsm_left_dev(a, x, true, false, true, st) != FLA_SUCCESS) return FLA_FAILURE;
    return trsm_left_dev(a, x, false, false, false, st);
  }
  // A^T X = B:  U^T (L^T (P X)) = B  ->  X = P^T inv(L^T) inv(U^T) B
  if (trsm_left_dev(a, x, false, true, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (trsm_left_dev(a, x, true, true, true, st) != FLA_SUCCESS) return FLA_FAILURE;
  return apply_pivots_dev(x, d_rel, 0, n - 1, true, st);
}

// src/map/common/lapacksrc/f2c/dpotrs.c (argument checks :150-175)
int dpotrs_(char* uplo, int* n, int* nrhs, double* a, int* lda, double* b, int* ldb, int* info) {
  *info = 0;
  bool up = lsame1(uplo, 'U');
  if (!up && !lsame1(uplo, 'L')) return xerbla("DPOTRS", 1, info);
  if (*n < 0) return xerbla("DPOTRS", 2, info);
  if (*nrhs < 0) return xerbla("DPOTRS", 3, info);
  if (*lda < std::max(1, *n)) return xerbla("DPOTRS", 5, info);
  if (*ldb < std::max(1, *n)) return xerbla("DPOTRS", 7, info);
  if (*n == 0 || *nrhs == 0) return 0;
  ensure_init();
  FLA_Base_obj ba, bb;
  FLA_Obj A = raw_obj(FLA_DOUBLE, a, *n, *n, *lda, &ba);
  FLA_Obj B = raw_obj(FLA_DOUBLE, b, *n, *nrhs, *ldb, &bb);
  Staged sa, sb;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS || stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS)
    return FLA_FAILURE;
  if (potrs_dev(up, to_dmat(sa), to_dmat(sb)) != FLA_SUCCESS) return FLA_FAILURE;
  if (unstage(sb) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return 0;
}

// src/map/common/lapacksrc/f2c/dgetrs.c (argument checks, dlaswp + 2 dtrsm)
int dgetrs_(char* trans, int* n, int* nrhs, double* a, int* lda, int* ipiv, double* b, int* ldb,
            int* info) {
  *info = 0;
  bool notran = lsame1(trans, 'N');
  if (!notran && !lsame1(trans, 'T') && !lsame1(trans, 'C')) return xerbla("DGETRS", 1, info);
  if (*n < 0) return xerbla("DGETRS", 2, info);
  if (*nrhs < 0) return xerbla("DGETRS", 3, info);
  if (*lda < std::max(1, *n)) return xerbla("DGETRS", 5, info);
  if (*ldb < std::max(1, *n)) return xerbla("DGETRS", 8, info);
  if (*n == 0 || *nrhs == 0) return 0;
  ensure_init();
  FLA_Base_obj ba, bb;
  FLA_Obj A = raw_obj(FLA_DOUBLE, a, *n, *n, *lda, &ba);
  FLA_Obj B = raw_obj(FLA_DOUBLE, b, *n, *nrhs, *ldb, &bb);
  Staged sa, sb;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS || stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS)
    return FLA_FAILURE;
  int* dip = (int*)ws_get(WS_STAGE_P, sizeof(int) * 2 * (size_t)*n);
  if (!dip) return FLA_FAILURE;
  FB_CK(cudaMemcpyAsync(dip, ipiv, sizeof(int) * *n, cudaMemcpyDefault, ctx().stream));
  lapack_to_rel_kernel<<<(*n + 255) / 256, 256, 0, ctx().stream>>>(dip, dip + *n, *n);
  count_launch();
  if (getrs_dev(!notran, to_dmat(sa), dip + *n, to_dmat(sb)) != FLA_SUCCESS) return FLA_FAILURE;
  if (unstage(sb) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  return 0;
}

// src/map/common/lapacksrc/f2c/dposv.c:120-190: dpotrf_ then dpotrs_, with
// both operands staged once.
int dposv_(char* uplo, int* n, int* nrhs, double* a, int* lda, double* b, int* ldb, int* info) {
  *info = 0;
  bool up = lsame1(uplo, 'U');
  if (!up && !lsame1(uplo, 'L')) return xerbla("DPOSV ", 1, info);
  if (*n < 0) return xerbla("DPOSV ", 2, info);
  if (*nrhs < 0) return xerbla("DPOSV ", 3, info);
  if (*lda < std::max(1, *n)) return xerbla("DPOSV ", 5, info);
  if (*ldb < std::max(1, *n)) return xerbla("DPOSV ", 7, info);
  if (*n == 0) return 0;
  ensure_init();
  FLA_Base_obj ba, bb;
  FLA_Obj A = raw_obj(FLA_DOUBLE, a, *n, *n, *lda, &ba);
  FLA_Obj B = raw_obj(FLA_DOUBLE, b, *n, *nrhs, *ldb, &bb);
  Staged sa, sb;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS) return FLA_FAILURE;
  int e = -1;
  DMat da = to_dmat(sa);
  int r = up ? chol_upper_dev(da, &e) : chol_lower_dev(da, &e);
  if (r != FLA_SUCCESS) return FLA_FAILURE;
  if (e < 0 && *nrhs > 0) {
    if (stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS) return FLA_FAILURE;
    if (potrs_dev(up, da, to_dmat(sb)) != FLA_SUCCESS) return FLA_FAILURE;
    if (unstage(sb) != FLA_SUCCESS) return FLA_FAILURE;
  }
  if (unstage(sa) != FLA_SUCCESS || sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  *info = (e >= 0) ? e + 1 : 0;
  return 0;
}

// src/map/common/lapacksrc/f2c/dgesv.c:113-175: dgetrf_ then dgetrs_.
int dgesv_(int* n, int* nrhs, double* a, int* lda, int* ipiv, double* b, int* ldb, int* info) {
  *info = 0;
  if (*n < 0) return xerbla("DGESV ", 1, info);
  if (*nrhs < 0) return xerbla("DGESV ", 2, info);
  if (*lda < std::max(1, *n)) return xerbla("DGESV ", 4, info);
  if (*ldb < std::max(1, *n)) return xerbla("DGESV ", 7, info);
  if (*n == 0) return 0;
  ensure_init();
  FLA_Base_obj ba, bb;
  FLA_Obj A = raw_obj(FLA_DOUBLE, a, *n, *n, *lda, &ba);
  FLA_Obj B = raw_obj(FLA_DOUBLE, b, *n, *nrhs, *ldb, &bb);
  Staged sa, sb;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS) return FLA_FAILURE;
  const int nn = *n;
  bool host = !is_device_ptr(ipiv);
  int* dp = (int*)ws_get(WS_STAGE_P, sizeof(int) * (size_t)nn);
  if (!dp) return FLA_FAILURE;
  int e = -1;
  DMat da = to_dmat(sa);
  if (lu_piv_dev(da, dp, &e) != FLA_SUCCESS) return FLA_FAILURE;
  // dgetrs_ runs only when dgetrf_ reported no zero pivot (dgesv.c:170-175)
  if (e < 0 && *nrhs > 0) {
    if (stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS) return FLA_FAILURE;
    if (getrs_dev(false, da, dp, to_dmat(sb)) != FLA_SUCCESS) return FLA_FAILURE;
    if (unstage(sb) != FLA_SUCCESS) return FLA_FAILURE;
  }
  shift_pivots_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, ctx().stream>>>(dp, nn, 1);
  count_launch();
  if (unstage(sa) != FLA_SUCCESS) return FLA_FAILURE;
  if (host) {
    FB_CK(cudaMemcpyAsync(ipiv, dp, sizeof(int) * nn, cudaMemcpyDeviceToHost, ctx().stream));
  } else {
    FB_CK(cudaMemcpyAsync(ipiv, dp, sizeof(int) * nn, cudaMemcpyDeviceToDevice, ctx().stream));
  }
  if (sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  *info = (e >= 0) ? e + 1 : 0;
  return 0;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Mixed-precision solvers.
// ---------------------------------------------------------------------------
namespace {

// Solve A X = B by low-precision LU/Cholesky + refinement, with the FP64
// factorization as the fallback.  A, B, X: device views (X aligned).  On
// success with refinement A is untouched; `fact` (if not null) receives the
// FP64 factors on fallback.  iter: refinement steps (>= 0) or the dsgesv_
// code of the fallback (-3 low-precision factorization failed, -31 no
// convergence).  d_piv receives the pivots used (relative, device).
int mixed_solve_dev(bool chol, bool upper, DMat A, DMat B, DMat X, int* d_piv, const IrConfig& cfg, bool overwrite_a,
                    int* iter, int* inner, int* info) {
  cudaStream_t st = ctx().stream;
  const long n = A.m;
  *iter = 0;
  *inner = 0;
  *info = 0;
  DMat Ares = A;
  if (chol) {
    // the refinement's residual needs the whole symmetric matrix
    const long ld = (n + 1) & ~1L;
    double* S = (double*)ws_get(WS_FB, sizeof(double) * (size_t)ld * (size_t)std::max<long>(1, n));
    if (!S) return FLA_FAILURE;
    if (symmetrize(A, upper, S, ld, st) != FLA_SUCCESS) return FLA_FAILURE;
    Ares.p = S;
    Ares.ld = ld;
  }
  // Escalation: the requested format first; if its factorization breaks
  // down or the refinement stalls, an FP32-accurate tensor-core format (the
  // FP16 hi/lo split after a 16-bit format; 3xTF32 for classic and GMRES-IR
  // refinement as well); then the FP64 factorization.
  int steps = 0, code = -31;
  std::vector<LowPrec> ladder{cfg.prec};
  if (cfg.prec == LP_FP16 || cfg.prec == LP_BF16) ladder.push_back(LP_FP16X3);
  if (cfg.prec != LP_TF32X3 && cfg.solver != IR_AUTO) ladder.push_back(LP_TF32X3);
  static const bool trace = std::getenv("FLA_B200_IR_TRACE") != nullptr;
  for (LowPrec p : ladder) {
    LpFactor f;
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (trace) {
      cudaEventCreate(&t0);
      cudaEventCreate(&t1);
      cudaEventRecord(t0, st);
    }
    int r = chol ? lp_chol_factor(A, upper, p, cfg.scale, &f) : lp_lu_factor(A, p, cfg.scale, &f);
    if (r != FLA_SUCCESS) return FLA_FAILURE;
    if (trace) {
      cudaEventRecord(t1, st);
      cudaEventSynchronize(t1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, t0, t1);
      std::fprintf(stderr, "libflame_b200 ir: %s factorization in format %d: %.3f ms (info %d)\n",
                   chol ? "Cholesky" : "LU", (int)p, ms, f.info);
      cudaEventDestroy(t0);
      cudaEventDestroy(t1);
    }
    if (f.info >= 0) {
      code = -3;
      continue;
    }
    IrConfig c2 = cfg;
    c2.prec = p;
    IrResult res;
    if (ir_refine(Ares, B, X.p, X.ld, f, c2, &res) != FLA_SUCCESS) return FLA_FAILURE;
    *inner += res.inner;
    if (res.iter >= 0) {
      *iter = steps + res.iter;
      if (!chol) FB_CK(cudaMemcpyAsync(d_piv, f.piv, sizeof(int) * n, cudaMemcpyDeviceToDevice, st));
      return sync_all();
    }
    steps += cfg.itermax;
    code = -(cfg.itermax + 1);
  }
  *iter = code;
  // FP64 factorization (in place, or on a copy when A must stay unchanged)
  DMat Af = A;
  if (!overwrite_a) {
    const long ld = (n + 1) & ~1L;
    double* Cp = (double*)ws_get(WS_FB, sizeof(double) * (size_t)ld * (size_t)std::max<long>(1, n));
    if (!Cp) return FLA_FAILURE;
    FB_CK(cudaMemcpy2DAsync(Cp, sizeof(double) * ld, A.p, sizeof(double) * A.ld, sizeof(double) * n, n,
                            cudaMemcpyDeviceToDevice, st));
    Af.p = Cp;
    Af.ld = ld;
  }
  int e = -1;
  if (chol) {
    if ((upper ? chol_upper_dev(Af, &e) : chol_lower_dev(Af, &e)) != FLA_SUCCESS) return FLA_FAILURE;
  } else {
    if (lu_piv_dev(Af, d_piv, &e) != FLA_SUCCESS) return FLA_FAILURE;
  }
  if (e >= 0) {
    *info = e + 1;
    return sync_all();
  }
  FB_CK(cudaMemcpy2DAsync(X.p, sizeof(double) * X.ld, B.p, sizeof(double) * B.ld, sizeof(double) * n, X.n,
                          cudaMemcpyDeviceToDevice, st));
  if ((chol ? potrs_dev(upper, Af, X) : getrs_dev(false, Af, d_piv, X)) != FLA_SUCCESS) return FLA_FAILURE;
  return sync_all();
}

IrConfig config_from(int prec, int solver) {
  IrConfig c = ir_default_config();
  if (prec == 0) c.prec = LP_BF16;
  if (prec == 1) c.prec = LP_FP16;
  if (prec == 2) c.prec = LP_TF32X3;
  if (prec == 3) c.prec = LP_FP16X3;
  if (solver == 0) c.solver = IR_CLASSIC;
  if (solver == 1) c.solver = IR_GMRES;
  if (solver == 2) c.solver = IR_AUTO;
  return c;
}

}  // namespace

extern "C" {

// src/map/common/lapacksrc/f2c/dsgesv.c:189-412: same arguments, checks and
// ITER/INFO conventions; the single-precision factorization is the 16-bit
// tensor-core LU (format and refinement from FLA_B200_IR_PREC /
// FLA_B200_IR_SOLVER; by default the FP16 hi/lo split with equilibration
// and the adaptive refinement of FLA_B200_LU_piv_solve_mixed).  work and swork are not
// referenced (the library keeps its own workspace).
int dsgesv_(int* n, int* nrhs, double* a, int* lda, int* ipiv, double* b, int* ldb, double* x, int* ldx,
            double* work, float* swork, int* iter, int* info) {
  (void)work;
  (void)swork;
  *info = 0;
  *iter = 0;
  if (*n < 0) return xerbla("DSGESV", 1, info);
  if (*nrhs < 0) return xerbla("DSGESV", 2, info);
  if (*lda < std::max(1, *n)) return xerbla("DSGESV", 4, info);
  if (*ldb < std::max(1, *n)) return xerbla("DSGESV", 7, info);
  if (*ldx < std::max(1, *n)) return xerbla("DSGESV", 9, info);
  if (*n == 0) return 0;
  ensure_init();
  FLA_Base_obj ba, bb, bx;
  FLA_Obj A = raw_obj(FLA_DOUBLE, a, *n, *n, *lda, &ba);
  FLA_Obj B = raw_obj(FLA_DOUBLE, b, *n, *nrhs, *ldb, &bb);
  FLA_Obj X = raw_obj(FLA_DOUBLE, x, *n, *nrhs, *ldx, &bx);
  Staged sa, sb, sx;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS || stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS ||
      stage(X, WS_STAGE_X, &sx, false) != FLA_SUCCESS)
    return FLA_FAILURE;
  const int nn = *n;
  int* dp = (int*)ws_get(WS_STAGE_P, sizeof(int) * (size_t)nn);
  if (!dp) return FLA_FAILURE;
  int it = 0, inner = 0, inf = 0;
  if (mixed_solve_dev(false, false, to_dmat(sa), to_dmat(sb), to_dmat(sx), dp, config_from(-1, -1), true, &it,
                      &inner, &inf) != FLA_SUCCESS)
    return FLA_FAILURE;
  shift_pivots_kernel<<<(unsigned)((nn + 255) / 256), 256, 0, ctx().stream>>>(dp, nn, 1);
  count_launch();
  if (it < 0 && unstage(sa) != FLA_SUCCESS) return FLA_FAILURE;  // FP64 factors on fallback
  if (inf == 0 && unstage(sx) != FLA_SUCCESS) return FLA_FAILURE;
  FB_CK(cudaMemcpyAsync(ipiv, dp, sizeof(int) * nn, cudaMemcpyDefault, ctx().stream));
  if (sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  *iter = it;
  *info = inf;
  return 0;
}

// src/map/common/lapacksrc/f2c/dsposv.c:250-413, as dsgesv_ with the
// Cholesky factorization of the uplo triangle.
int dsposv_(char* uplo, int* n, int* nrhs, double* a, int* lda, double* b, int* ldb, double* x, int* ldx,
            double* work, float* swork, int* iter, int* info) {
  (void)work;
  (void)swork;
  *info = 0;
  *iter = 0;
  const bool up = lsame1(uplo, 'U');
  if (!up && !lsame1(uplo, 'L')) return xerbla("DSPOSV", 1, info);
  if (*n < 0) return xerbla("DSPOSV", 2, info);
  if (*nrhs < 0) return xerbla("DSPOSV", 3, info);
  if (*lda < std::max(1, *n)) return xerbla("DSPOSV", 5, info);
  if (*ldb < std::max(1, *n)) return xerbla("DSPOSV", 7, info);
  if (*ldx < std::max(1, *n)) return xerbla("DSPOSV", 9, info);
  if (*n == 0) return 0;
  ensure_init();
  FLA_Base_obj ba, bb, bx;
  FLA_Obj A = raw_obj(FLA_DOUBLE, a, *n, *n, *lda, &ba);
  FLA_Obj B = raw_obj(FLA_DOUBLE, b, *n, *nrhs, *ldb, &bb);
  FLA_Obj X = raw_obj(FLA_DOUBLE, x, *n, *nrhs, *ldx, &bx);
  Staged sa, sb, sx;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS || stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS ||
      stage(X, WS_STAGE_X, &sx, false) != FLA_SUCCESS)
    return FLA_FAILURE;
  int it = 0, inner = 0, inf = 0;
  if (mixed_solve_dev(true, up, to_dmat(sa), to_dmat(sb), to_dmat(sx), nullptr, config_from(-1, -1), true, &it,
                      &inner, &inf) != FLA_SUCCESS)
    return FLA_FAILURE;
  if (it < 0 && unstage(sa) != FLA_SUCCESS) return FLA_FAILURE;
  if (inf == 0 && unstage(sx) != FLA_SUCCESS) return FLA_FAILURE;
  if (sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  *iter = it;
  *info = inf;
  return 0;
}

// X := A^-1 B by the mixed-precision LU solver; A is left unchanged.
// prec: 0 BF16, 1 FP16 (equilibrated), -1 library default; solver: 0
// classic refinement, 1 GMRES-IR, -1 default.  iter / inner (optional):
// refinement steps (or -3 / -31 when the FP64 fallback ran) and GMRES
// iterations.  Returns FLA_SUCCESS, the zero-based index of a zero pivot of
// the fallback factorization, or FLA_FAILURE.
FLA_Error FLA_B200_LU_piv_solve_mixed(FLA_Obj A, FLA_Obj B, FLA_Obj X, int prec, int solver, int* iter,
                                      int* inner) {
  ensure_init();
  FB_REQUIRE(A.base && A.base->datatype == FLA_DOUBLE && A.m == A.n, "FLA_B200_LU_piv_solve_mixed",
             "A must be a square FLA_DOUBLE matrix");
  FB_REQUIRE(B.base && X.base && B.m == A.m && X.m == A.m && X.n == B.n, "FLA_B200_LU_piv_solve_mixed",
             "B and X must be n x nrhs");
  if (A.m == 0 || B.n == 0) return FLA_SUCCESS;
  Staged sa, sb, sx;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS || stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS ||
      stage(X, WS_STAGE_X, &sx, false) != FLA_SUCCESS)
    return FLA_FAILURE;
  int* dp = (int*)ws_get(WS_STAGE_P, sizeof(int) * (size_t)A.m);
  if (!dp) return FLA_FAILURE;
  int it = 0, inn = 0, inf = 0;
  op_begin(ctx().stream);
  op_hold(true);
  const int r = mixed_solve_dev(false, false, to_dmat(sa), to_dmat(sb), to_dmat(sx), dp, config_from(prec, solver),
                                false, &it, &inn, &inf);
  op_hold(false);
  if (r != FLA_SUCCESS) return FLA_FAILURE;
  if (unstage(sx) != FLA_SUCCESS) return FLA_FAILURE;
  op_end(ctx().stream);
  if (sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  if (iter) *iter = it;
  if (inner) *inner = inn;
  return inf > 0 ? inf - 1 : FLA_SUCCESS;
}

// X := A^-1 B by the mixed-precision Cholesky solver (the uplo triangle of
// the SPD A is read; A is left unchanged).  Arguments and results as
// FLA_B200_LU_piv_solve_mixed; a non-positive pivot of the fallback
// factorization returns its zero-based column.
FLA_Error FLA_B200_Chol_solve_mixed(FLA_Uplo uplo, FLA_Obj A, FLA_Obj B, FLA_Obj X, int prec, int solver, int* iter,
                                    int* inner) {
  ensure_init();
  FB_REQUIRE(uplo == FLA_LOWER_TRIANGULAR || uplo == FLA_UPPER_TRIANGULAR, "FLA_B200_Chol_solve_mixed",
             "invalid uplo value");
  FB_REQUIRE(A.base && A.base->datatype == FLA_DOUBLE && A.m == A.n, "FLA_B200_Chol_solve_mixed",
             "A must be a square FLA_DOUBLE matrix");
  FB_REQUIRE(B.base && X.base && B.m == A.m && X.m == A.m && X.n == B.n, "FLA_B200_Chol_solve_mixed",
             "B and X must be n x nrhs");
  if (A.m == 0 || B.n == 0) return FLA_SUCCESS;
  Staged sa, sb, sx;
  if (stage(A, WS_STAGE_A, &sa) != FLA_SUCCESS || stage(B, WS_STAGE_B, &sb) != FLA_SUCCESS ||
      stage(X, WS_STAGE_X, &sx, false) != FLA_SUCCESS)
    return FLA_FAILURE;
  int it = 0, inn = 0, inf = 0;
  op_begin(ctx().stream);
  op_hold(true);
  const int r = mixed_solve_dev(true, uplo == FLA_UPPER_TRIANGULAR, to_dmat(sa), to_dmat(sb), to_dmat(sx), nullptr,
                                config_from(prec, solver), false, &it, &inn, &inf);
  op_hold(false);
  if (r != FLA_SUCCESS) return FLA_FAILURE;
  if (unstage(sx) != FLA_SUCCESS) return FLA_FAILURE;
  op_end(ctx().stream);
  if (sync_all() != FLA_SUCCESS) return FLA_FAILURE;
  if (iter) *iter = it;
  if (inner) *inner = inn;
  return inf > 0 ? inf - 1 : FLA_SUCCESS;
}

}  // extern "C"
