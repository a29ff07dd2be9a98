// Batched factorizations (batched.cu).
#pragma once
#include "common.h"

namespace fb {

template <typename T>
struct BatchArgs {
  int count = 0;
  const int* order = nullptr;   // schedule (matrix indices)
  int* counter = nullptr;       // next schedule slot
  const int* n = nullptr;       // orders
  const long* ld = nullptr;     // leading dimensions
  T** A = nullptr;              // matrices (column-major)
  int** piv = nullptr;          // LU: relative pivots per matrix
  int nrhs = 0;                 // right-hand sides (0: factor only)
  T** B = nullptr;
  const long* ldb = nullptr;
  int* info = nullptr;          // per matrix: -1 or the failing / first zero-pivot column
  const int* nb_of_size = nullptr;  // panel width by order
  T* logdet = nullptr;          // optional: per matrix sum_i log L(i, i) (FP64 Cholesky)
  int* err = nullptr;           // status word for wait timeouts (FP64 Cholesky)
};

template <typename T>
int batched_factor(bool lu, int count, const int* h_n, T** d_A, const long* d_ld, const int* d_n, int** d_piv,
                   int nrhs, T** d_B, const long* d_ldb, int* d_info, cudaStream_t st, T* d_logdet = nullptr);
int batched_tune(bool lu, bool f64, int samples_per_bin, double* times_out);
int batched_nb(bool lu, bool f64, int n);
int batched_fill_dominant(bool f64, int count, void** dA, const int* dn, const long* dld, cudaStream_t st);

}  // namespace fb
