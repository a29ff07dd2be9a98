// Internal declarations shared by the libflame_b200 translation units.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "FLAME.h"

namespace fb {

// ---------------------------------------------------------------------------
// Library context (one per process, bound to the device current at FLA_Init).
// ---------------------------------------------------------------------------
struct Context {
  bool initialized = false;
  int device = 0;
  int num_sms = 148;
  size_t smem_optin = 0;
  cudaStream_t stream = nullptr;     // main stream: trailing updates
  cudaStream_t side = nullptr;       // lookahead stream: panels
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  int* d_status = nullptr;           // device status words (see Status below)
  int* h_status = nullptr;           // pinned mirror
  unsigned long long launches = 0;   // kernels launched by this library
};

Context& ctx();

// Device status block (reset per operation by status_reset()):
//   [ST_ERROR] nonzero when a kernel's bounded wait expired (code of the wait)
//   [ST_INFO]  numerical info: zero-based index of the first failing column,
//              INT_MAX when none; kernels atomicMin into it
//   [ST_BAR..] counters of the grid barriers of cooperative kernels
enum : int { ST_ERROR = 0, ST_INFO = 1, ST_BAR = 2, ST_WORDS = 64 };

// Record one kernel launch issued by this library (for the launch count
// reported by FLA_B200_kernel_launches()).
inline void count_launch(unsigned n = 1) { ctx().launches += n; }

// Device-side timing (CUDA events on the launching stream).
//   op_begin/op_end bracket the device work of one driver call; the elapsed
//   time is FLA_B200_last_op_ms().  When profiling is on, prof_begin/
//   prof_end bracket individual launches of a kernel class and accumulate
//   their durations and algorithmic flops (FLA_B200_profile_read()).
enum ProfClass : int { PROF_GEMM = 0, PROF_PANEL, PROF_TRSM, PROF_SWAP, PROF_DIAG, PROF_OTHER, PROF_NCLASS };
void op_begin(cudaStream_t st);
void op_end(cudaStream_t st);
void op_hold(bool on);      // keep the current op window open across nested drivers
void order_after_caller();  // main stream waits for the caller's default-stream work
bool prof_on();
int prof_begin(cudaStream_t st);                       // returns a slot or -1
void prof_end(int slot, cudaStream_t st, int cls, double flops);

// CUDA error handling: every runtime call on the op path goes through CK();
// a failure prints the call and returns FLA_FAILURE from the enclosing op.
void set_last_error(const std::string& msg);
#define FB_CK(call)                                                              \
  do {                                                                           \
    cudaError_t e_ = (call);                                                     \
    if (e_ != cudaSuccess) {                                                     \
      ::fb::set_last_error(std::string(#call) + ": " + cudaGetErrorString(e_)); \
      return FLA_FAILURE;                                                        \
    }                                                                            \
  } while (0)

// Argument-check failure: the reference prints a message and aborts
// (src/base/flamec/main/FLA_Check.c:38-56, FLA_Error.c:248-252).
[[noreturn]] void check_fail(const char* func, const char* what);
#define FB_REQUIRE(cond, func, what)                                             \
  do {                                                                           \
    if (FLA_Check_error_level() >= FLA_MIN_ERROR_CHECKING && !(cond))            \
      ::fb::check_fail(func, what);                                              \
  } while (0)

// ---------------------------------------------------------------------------
// Device workspace: persistent, grown on demand, one buffer per slot.
// ---------------------------------------------------------------------------
enum WsSlot : int {
  WS_STAGE_A = 0,   // host-buffer staging of the main operand
  WS_STAGE_B,       // staging of a second operand (B / X / T)
  WS_STAGE_P,       // staging of pivots
  WS_PANEL,         // panel scratch (candidates, rows, inverse blocks)
  WS_REPACK,        // aligned repack of an operand
  WS_MISC,
  WS_MISC2,
  WS_LP0,           // mixed-precision solvers: low-precision factor
  WS_LP1,           //   packed 16-bit operands
  WS_LP2,
  WS_LP3,           //   FP64 panel / inverses
  WS_LP4,           //   inverse blocks kept for the correction solves
  WS_LP5,           //   coupling blocks of the correction sweeps
  WS_IR0,           //   refinement vectors (FP64 / FP32)
  WS_IR1,
  WS_IR2,
  WS_STAGE_X,       // staging of a third operand (solution X)
  WS_FB,            // FP64 copy for the fallback factorization / symmetric residual
  WS_PERM,          // composed row orders of long pivot sequences
  WS_PERM_T,        // gathered rows
  WS_TRINV,         // inverted diagonal blocks of the solves
  WS_SOLVE_W,       // block of solved unknowns
  WS_SPLITK,        // partial products of split-K GEMMs (main stream)
  WS_SPLITK_SIDE,   //   (side stream: the two streams' GEMMs may overlap)
  WS_QR_T,          // FLA_QR_UT: the T factors of two panels (ping-pong)
  WS_QR_U,          //   unit lower trapezoids of the panel recursion
  WS_QR_W,          //   its W products
  WS_ADJ,           // per-stream scratch of the batched Cholesky adjoint
  WS_FLASH0,        // column-major copies of hierarchical (FLASH) operands
  WS_FLASH1,
  WS_FLASH2,
  WS_FLASH3,
  WS_PANEL_T,       // transposed copies of Cholesky panels (two, ping-pong)
  WS_SWEEP,         // ready flags of the one-launch triangular sweeps
  WS_NSLOTS
};
void* ws_get(int slot, size_t bytes);  // nullptr on allocation failure
void ws_release_all();

// A column-major matrix operand in device memory.
struct DMat {
  double* p = nullptr;
  long ld = 0;
  long m = 0, n = 0;
  DMat sub(long i, long j, long mm, long nn) const {
    DMat r;
    r.p = p + i + j * ld;
    r.ld = ld;
    r.m = mm;
    r.n = nn;
    return r;
  }
};
struct FMat {
  float* p = nullptr;
  long ld = 0;
  long m = 0, n = 0;
  FMat sub(long i, long j, long mm, long nn) const {
    FMat r;
    r.p = p + i + j * ld;
    r.ld = ld;
    r.m = mm;
    r.n = nn;
    return r;
  }
};

// Is ptr a device (or managed) address usable by kernels?
bool is_device_ptr(const void* ptr);

// Operand staging for an FLA_Obj view: yields a device pointer + ld.  Host
// views are copied into workspace slot `slot` (and copied back by
// finish()); device views are used in place.  Also repacks device views
// whose base or ld breaks the 16-byte alignment the TMA path needs.
struct Staged {
  void* dev = nullptr;       // device pointer of the (possibly staged) view
  long ld = 0;               // its leading dimension (elements)
  long m = 0, n = 0;
  size_t esize = 8;
  bool staged = false;       // copied from host or repacked
  void* orig = nullptr;      // original buffer at view
  long orig_ld = 0;
  bool orig_is_host = false;
};
// stage(): copy in (if needed).  `copy_in` false skips the H2D copy (pure
// outputs).  Returns FLA_SUCCESS or FLA_FAILURE.
int stage(const FLA_Obj& A, int slot, Staged* out, bool copy_in = true, bool need_align = true);
// unstage(): copy back to the original buffer when staged.
int unstage(const Staged& s, bool copy_out = true);

// Library-wide synchronisation of the main + side streams with error check.
int sync_all();

// Reset the device status block (error + info) on the main stream.
int status_reset();
// Read back the status block (after sync).  Returns FLA_FAILURE on a kernel
// timeout; writes the numerical info (first failing index or -1) to *info.
int status_read(int* info);

// ---------------------------------------------------------------------------
// FP64 GEMM engine (gemm_f64.cu).
//   C := alpha * op(A) * op(B) + beta * C, column-major, DMMA tiles fed by TMA.
//   ta/tb: false = no transpose, true = transpose.
//   mode LOWER: only C(i,j) with i - j >= diag_off are written (SYRK-style),
//   tiles entirely above are skipped.
// ---------------------------------------------------------------------------
enum GemmMode : int { GEMM_FULL = 0, GEMM_LOWER = 1 };
int gemm_f64(cudaStream_t st, bool ta, bool tb, long m, long n, long k, double alpha,
             const double* A, long lda, const double* B, long ldb, double beta, double* C,
             long ldc, GemmMode mode = GEMM_FULL, long diag_off = 0,
             const int* guard = nullptr, int guard_limit = 0x7fffffff, long kmax = 0);
// kmax > 0 (full mode only): split k so that no CTA runs more than about
// kmax of it, for GEMMs whose long-running tiles would keep SMs from a
// cluster kernel waiting on the other stream.
// The guard pointer is the status block's info word (INT_MAX, or the first
// failing column): the kernel returns at once when it holds a column below
// guard_limit, i.e. when a factorization step this update follows has failed.
inline const int* info_guard() { return ctx().d_status + ST_INFO; }

// TMA needs 16-byte aligned base and ld*8 % 16 == 0.
inline bool tma_ok(const void* p, long ld) {
  return ((reinterpret_cast<uintptr_t>(p) & 15u) == 0) && ((ld * 8) % 16 == 0);
}

// ---------------------------------------------------------------------------
// Factorization drivers on device operands (used by the FLA_* front ends
// and by the LAPACK entry points).  info: -1 or the zero-based index of the
// first failing column.  All enqueue on ctx().stream and read the status
// block back before returning.
// ---------------------------------------------------------------------------
int chol_lower_dev(DMat A, int* info);
int chol_upper_dev(DMat A, int* info);
int chol_lower_enqueue(DMat A, cudaStream_t st);
int lu_piv_dev(DMat A, int* d_piv, int* info);       // d_piv: device, relative
int apply_pivots_dev(DMat A, const int* d_piv, int k1, int k2, bool reverse, cudaStream_t st);
int laswp_dev(double* A, long ld, int row0, const int* d_piv, int npiv, int c0, int n0, int c1,
              int n1, bool reverse, cudaStream_t st);
// B := inv(op(T)) B, T n x n triangular (lower/upper, transposed, unit).
int trsm_left_dev(DMat T, DMat B, bool lower, bool trans, bool unit, cudaStream_t st);
int trsm_block(const double* T, long ldt, double* B, long ldb, int b, long n, bool lower,
               bool trans, bool unit, cudaStream_t st);
// X := inv(L), L b x b lower triangular (unit diagonal if unit), X ld ldx.
int tri_inverse_lower(const double* L, long ldl, int b, bool unit, double* X, long ldx, cudaStream_t st);
// Inverses of the 128 x 128 diagonal blocks of an n x n triangle, one
// launch: block q into X + q*128*128 (ld 128).
int tri_inverse_blocks(const double* T, long ldt, long n, bool lower, bool unit, double* X, cudaStream_t st);
// Inverses of the bs x bs (bs <= 128) diagonal blocks, block q into
// X + q*bs*bs (ld bs), one launch.
int tri_inverse_blocks_bs(const double* T, long ldt, long n, int bs, bool lower, bool unit, double* X,
                          cudaStream_t st);
// X := inv(T), T b x b triangular (lower or upper; unit diagonal if unit).
int tri_inverse(const double* T, long ldt, int b, bool lower, bool unit, double* X, long ldx, cudaStream_t st);
// X := X inv(op(T)) ^T row by row: every row x of the m x b block X is
// replaced by the solution of op(T) y = x (b <= 128).
int trsm_right_block(const double* T, long ldt, double* X, long ldx, long m, int b, bool lower, bool trans,
                     bool unit, cudaStream_t st);
// dst := src^T for an m x n src (dst n x m); upper_only writes i <= j only.
int transpose_dev(const double* src, long lds, double* dst, long ldd, long m, long n, bool upper_only,
                  cudaStream_t st);
// Row interchanges on a matrix stored transposed (AT = A^T, column-major):
// rows row0+i and row0+i+piv[i] of A (columns of AT) are exchanged, in
// order, over the A-columns [c0, c0+n0) and [c1, c1+n1) (rows of AT).
// U12 := inv(L11) A12 (unit lower L11 of order b) on transposed storage:
// L11(i, j) at Ls[j + i ld], A12(i, c) at X[c + i ld] (c < ncols), overwritten.
int u12_subst(const double* Ls, double* X, long ld, int b, long ncols, cudaStream_t st);
// X := X inv(L)^T (X ncols x b, L non-unit lower of order b <= 128, both
// column-major with leading dimension ld), by forward substitution.
int trsm_rlt_subst(const double* L, double* X, long ld, int b, long ncols, const int* guard, int guard_limit,
                   cudaStream_t st);
// The same with an FP32 X (ld ldx) and an FP64 L (ld ldl), solved in FP64.
int trsm_rlt_subst_f32(const double* L, long ldl, float* X, long ldx, int b, long ncols, const int* guard,
                       int guard_limit, cudaStream_t st);
int laswp_t_dev(double* AT, long ldt, int row0, const int* d_piv, int npiv, int c0, int n0, int c1, int n1,
                cudaStream_t st);
int laswp_t_f32(float* AT, long ldt, int row0, const int* d_piv, int npiv, int c0, int n0, int c1, int n1,
                cudaStream_t st);
// Cholesky of one b x b (b <= 128) lower diagonal block in place (FP64).
int potrf_diag_dev(double* A, long ld, int b, int gcol, cudaStream_t st);
// LU panel on the transposed matrix: the M x w panel of A whose element
// (i, j) is at P[i * ld + j] (rows of A are the columns of AT).
int lu_panel_factor_t(double* P, long ld, long M, int w, int* d_piv, int gcol, cudaStream_t st);
// LU panel: factor the M x w panel at P with partial pivoting (M >= w);
// d_piv gets w relative pivots; gcol = global index of the first column.
int lu_panel_factor(double* P, long ld, long M, int w, int* d_piv, int gcol, cudaStream_t st);
// X := X inv(L)^T for an m x b block (b <= 128); no-op once *guard != INT_MAX.
int trsm_right_lt_block(const double* L, long ldl, double* X, long ldx, long m, int b, const int* guard,
                        cudaStream_t st);

}  // namespace fb
