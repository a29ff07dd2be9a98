// Mixed-precision solvers (mixed.cu): low-precision factors and refinement.
#pragma once
#include "common.h"
#include "lowprec.h"

namespace fb {

// IR_AUTO: classic refinement while every step reduces the backward error at
// least fourfold; otherwise the caller escalates (a 16-bit format to the
// FP32-accurate FP16 hi/lo split, that one to the FP64 factorization).
enum IrSolver : int { IR_CLASSIC = 0, IR_GMRES = 1, IR_AUTO = 2 };

struct IrConfig {
  LowPrec prec = LP_FP16X3;  // format of the tensor-core updates: the FP16 hi/lo split (FP32-accurate)
  bool scale = true;        // power-of-two equilibration before rounding
  IrSolver solver = IR_AUTO;
  int itermax = 30;         // ITERMAX of dsgesv_/dsposv_
  int gmres_m = 30;         // GMRES restart length (inner iterations per step)
  double gmres_tol = 1e-8;  // inner relative residual target
  bool polish = true;       // refine on while the backward error still halves
};

struct IrResult {
  int iter = 0;      // refinement steps (>= 0), or -31 when not converged
  int inner = 0;     // GMRES iterations in total
  double anorm = 0;  // ||A||_inf
  bool stalled = false;  // stopped early: the backward error stopped decreasing
};

// Factors of diag(sr) A diag(sc) (LU, transposed layout) or of
// diag(sr) A diag(sr) (Cholesky, lower) held in FP32.
struct LpFactor {
  bool chol = false;
  bool scaled = false;
  LowPrec prec = LP_FP16;
  long n = 0;
  float* F = nullptr;   // LU: (P D_r A D_c)^T = (L U)^T; Cholesky: L (lower)
  long ldf = 0;
  int* piv = nullptr;   // LU: relative pivots
  int* perm = nullptr;  // LU: row order of P b (perm[i] = source row of row i)
  float* inv1 = nullptr;  // per 128-block: LU inv(L11^T); Cholesky inv(L11)
  float* inv2 = nullptr;  // per 128-block: LU inv(U11^T)
  float* wf = nullptr;    // per 128-block: coupling blocks of the forward sweep
  float* wb = nullptr;    //   and of the backward sweep (solve_sweep_kernel)
  bool coupled = false;   // wf / wb formed for the current factors
  double* sr = nullptr;   // row scaling (or the symmetric scaling)
  double* sc = nullptr;   // column scaling
  int info = -1;          // first failing column of the low-precision factorization
  double shift = 0.0;     // Cholesky: diagonal shift of the factored matrix
};

int lp_lu_factor(DMat A, LowPrec prec, bool scale, LpFactor* f);
int lp_chol_factor(DMat A, bool upper, LowPrec prec, bool scale, LpFactor* f);
// D := M^-1 R with the low-precision factors (FP64 in and out).
int lp_solve(const LpFactor& f, const double* R, long ldr, double* D, long ldd, long nrhs, float* T, float* Tb,
             cudaStream_t st);
int ir_refine(const DMat& A, const DMat& B, double* X, long ldx, const LpFactor& f, const IrConfig& cfg,
              IrResult* res);
int symmetrize(const DMat& A, bool upper, double* S, long lds, cudaStream_t st);
IrConfig ir_default_config();

}  // namespace fb
