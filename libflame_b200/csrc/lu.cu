// LU factorization with partial pivoting (FLA_LU_piv) on the GPU, plus the
// row-interchange kernels behind FLA_Apply_pivots and the blocked left
// triangular solve of the solves.
//
// Blocked right-looking algorithm with the reference's structure
// (src/lapack/dec/lu/piv/vars/flamec/FLA_LU_piv_blk_var5.c:13-114):
//   for each block of nb columns:
//     [A11;A21], p1 := LU_piv([A11;A21])   lu_panel_factor (lu_panel.cu)
//     pivot [A10;A20] and [A12;A22]         laswp_compose/apply kernels
//     A12 := inv(tril_unit(A11)) A12         forward substitution, one launch
//                                            (u12_subst_kernel)
//     A22 -= A21 A12                         DMMA GEMM engine
// run on the transposed matrix, with the next panel factored on a second
// stream while the trailing update runs (lu_piv_dev below).  Pivot choice is the reference's: the entry of
// largest magnitude in the current column, the first (smallest row) among
// equals (idamax, src/flablas/f2c/idamax.c:41,60 via bl1_damax).  A zero
// pivot column is not swapped or scaled and its index is reported (the first
// one), and the factorization continues (FLA_LU_piv_opt_var4.c:272-331).
//
// lu_panel_kernel (below) is the grid-wide form of the panel: the
// (m-k) x nb panel is split in row slabs, one per CTA of a cooperative
// launch, held in shared memory for the whole panel.  Per column: each CTA
// finds its local pivot candidate and publishes it (value, row, the full
// panel row) in global memory; one grid barrier; every CTA then picks the
// same winner, the owners of rows j and p(j) exchange them, and every CTA
// scales its part of column j and applies the rank-1 update to its slab.
// It serves the allocation-free single-panel entry point.
#include <climits>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <string>
#include <vector>

#include "common.h"
#include "dev_util.cuh"

namespace fb {

namespace {

constexpr int PANEL_THREADS = 256;
constexpr int NBMAX = 128;
constexpr size_t PANEL_SMEM_CAP = 200 * 1024;

struct PanelArgs {
  double* P;         // panel (row k, col k), column-major
  long ld;
  int M;             // panel rows (m - k)
  int nb;            // panel columns
  int R;             // rows per CTA
  int lds;           // SMEM leading dimension
  int G;             // CTAs
  int gcol;          // global column of panel column 0
  int* piv;          // out: nb relative pivots
  double* cand_row;  // [2][G][nb]
  double* cand_val;  // [2][G]
  int* cand_idx;     // [2][G]
  double* diag_row;  // [2][nb]
  unsigned* bar;     // barrier counter (zeroed before launch)
  int* err;
  int* info;
};

__global__ void __launch_bounds__(PANEL_THREADS) lu_panel_kernel(PanelArgs a) {
  extern __shared__ double S[];  // slab: S[i + col*lds], then u row
  __shared__ double s_rv[PANEL_THREADS / 32];
  __shared__ int s_ri[PANEL_THREADS / 32];
  __shared__ int s_ci, s_w, s_r;
  double* su = S + (size_t)a.lds * a.nb;  // nb doubles

  const int c = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r0 = c * a.R;
  const int rows = min(a.R, a.M - r0);
  const int nb = a.nb, lds = a.lds, G = a.G;

  for (int col = 0; col < nb; ++col)
    for (int i = tid; i < rows; i += PANEL_THREADS) S[i + col * lds] = a.P[(long)(r0 + i) + (long)col * a.ld];
  __syncthreads();

  int first_null = -1;
  for (int j = 0; j < nb; ++j) {
    const int par = j & 1;
    // ---- 1. local candidate: max |a(i,j)|, smallest row on ties, rows >= j
    double bv = -1.0;
    int bi = INT_MAX;
    for (int i = tid; i < rows; i += PANEL_THREADS) {
      const int gi = r0 + i;
      if (gi >= j) {
        const double v = fabs(S[i + j * lds]);
        if (v > bv || (v == bv && gi < bi)) { bv = v; bi = gi; }
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { s_rv[warp] = bv; s_ri[warp] = bi; }
    __syncthreads();
    if (tid == 0) {
      double v = s_rv[0];
      int i0 = s_ri[0];
      for (int w = 1; w < PANEL_THREADS / 32; ++w)
        if (s_rv[w] > v || (s_rv[w] == v && s_ri[w] < i0)) { v = s_rv[w]; i0 = s_ri[w]; }
      __stcg(a.cand_val + par * G + c, v);
      __stcg(a.cand_idx + par * G + c, i0);
      s_ci = i0;
    }
    __syncthreads();
    // ---- 2. publish the candidate row and (owner of row j) the row j
    if (s_ci != INT_MAX) {
      const int li = s_ci - r0;
      for (int col = tid; col < nb; col += PANEL_THREADS)
        __stcg(a.cand_row + ((size_t)par * G + c) * nb + col, S[li + col * lds]);
    }
    if (j >= r0 && j < r0 + rows)
      for (int col = tid; col < nb; col += PANEL_THREADS) __stcg(a.diag_row + par * nb + col, S[(j - r0) + col * lds]);
    // ---- 3. grid barrier
    if (!grid_barrier(a.bar, (unsigned)G, (unsigned)(j + 1), a.err, 21)) return;
    // ---- 4. winner (same on every CTA)
    if (warp == 0) {
      double v = -2.0;
      int i0 = INT_MAX, w0 = 0;
      for (int w = lane; w < G; w += 32) {
        const double cv = __ldcg(a.cand_val + par * G + w);
        const int ci = __ldcg(a.cand_idx + par * G + w);
        if (ci != INT_MAX && (cv > v || (cv == v && ci < i0))) { v = cv; i0 = ci; w0 = w; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i0, off);
        const int ow = __shfl_xor_sync(0xffffffffu, w0, off);
        if (ov > v || (ov == v && oi < i0)) { v = ov; i0 = oi; w0 = ow; }
      }
      if (lane == 0) { s_w = w0; s_r = i0; }
    }
    __syncthreads();
    const int w = s_w;
    int r = s_r;
    const double* wrow = a.cand_row + ((size_t)par * G + w) * nb;
    if (r == INT_MAX) {
      // no orderable candidate (every magnitude NaN): keep row j, as idamax
      // does when no later entry compares greater than the first; row j was
      // published by its owner before the barrier
      r = j;
      wrow = a.diag_row + par * nb;
    }
    for (int col = tid; col < nb; col += PANEL_THREADS) su[col] = __ldcg(wrow + col);
    __syncthreads();
    const double piv = su[j];
    if (c == 0 && tid == 0) a.piv[j] = r - j;
    if (piv == 0.0) {
      if (first_null < 0) first_null = j;
    } else if (r != j) {
      // ---- 5. interchange rows j and r (whole panel row)
      if (j >= r0 && j < r0 + rows)
        for (int col = tid; col < nb; col += PANEL_THREADS) S[(j - r0) + col * lds] = su[col];
      if (r >= r0 && r < r0 + rows)
        for (int col = tid; col < nb; col += PANEL_THREADS)
          S[(r - r0) + col * lds] = __ldcg(a.diag_row + par * nb + col);
    }
    __syncthreads();
    // ---- 6. scale column j below the pivot and update the slab
    if (piv != 0.0) {
      const double rinv = 1.0 / piv;  // reciprocal multiply, as bl1_dinvscalv
      for (int i = tid; i < rows; i += PANEL_THREADS) {
        if (r0 + i > j) {
          const double l = S[i + j * lds] * rinv;
          S[i + j * lds] = l;
          for (int col = j + 1; col < nb; ++col) S[i + col * lds] -= l * su[col];
        }
      }
    }
    __syncthreads();
  }
  for (int col = 0; col < nb; ++col)
    for (int i = tid; i < rows; i += PANEL_THREADS) a.P[(long)(r0 + i) + (long)col * a.ld] = S[i + col * lds];
  if (c == 0 && tid == 0 && first_null >= 0) atomicMin(a.info, a.gcol + first_null);
}

// Row interchanges on a set of columns: for each column, rows row0+i and
// row0+i+piv[i] are swapped for i = 0..npiv-1 in order (or in reverse when
// `reverse`, which applies P^T).  Columns: [c0, c0+n0) and [c1, c1+n1).
//
// Blocked form (npiv <= LASWP_MAXP): the interchanges touch at most 2*npiv
// rows ("slots": rows row0..row0+npiv-1, then each distinct target below
// them).  Each CTA of laswp_apply_kernel composes the whole sequence of
// interchanges into one permutation of the slots (in shared memory) and
// then moves its columns' slot values with independent, coalesced loads
// and stores, LASWP_NC columns per CTA.
// TR: the matrix is stored transposed (element (row, col) of A at
// A[col + row * ld]); consecutive threads then take consecutive columns of
// one slot row, which are contiguous.
constexpr int LASWP_MAXP = 128;
constexpr int LASWP_NC = 16;  // columns per CTA (static SMEM < 48 KB)

// Composition of the interchange sequence into slot rows and sources, in
// shared memory (every CTA of the apply kernel forms it itself: the sequence
// has at most LASWP_MAXP entries, and a separate launch would cost more).
__device__ void laswp_compose(const int* __restrict__ piv, int npiv, int reverse, int* s_piv, int* s_tgt,
                              int* s_row, int* s_src) {
  const int tid = threadIdx.x;
  const int nslot = 2 * npiv;
  for (int s = tid; s < nslot; s += blockDim.x) s_row[s] = (s < npiv) ? s : -1;
  for (int i = tid; i < npiv; i += blockDim.x) s_piv[i] = piv[i];
  __syncthreads();
  for (int i = tid; i < npiv; i += blockDim.x) {
    const int t = i + s_piv[i];  // target row offset
    int slot;
    if (t < npiv) {
      slot = t;
    } else {
      // the first interchange with the same far target owns the slot
      // (branch-free scan: the loads of the unrolled loop overlap)
      int first = i;
#pragma unroll 8
      for (int i2 = i - 1; i2 >= 0; --i2) first = (i2 + s_piv[i2] == t) ? i2 : first;
      slot = npiv + first;
      if (first == i) s_row[slot] = t;
    }
    s_tgt[i] = slot;
  }
  __syncthreads();
  if (tid == 0) {
    for (int s = 0; s < nslot; ++s) s_src[s] = s;
    for (int q = 0; q < npiv; ++q) {
      const int i = reverse ? npiv - 1 - q : q;
      const int a = i, b = s_tgt[i];
      const int x = s_src[a];
      s_src[a] = s_src[b];
      s_src[b] = x;
    }
  }
  __syncthreads();
}

template <typename T, bool TR>
__global__ void __launch_bounds__(256) laswp_apply_kernel(T* A, long ld, int row0, const int* __restrict__ piv,
                                                          int npiv, int reverse, int c0, int n0, int c1, int n1) {
  __shared__ int s_piv[LASWP_MAXP];
  __shared__ int s_tgt[LASWP_MAXP];
  __shared__ int s_row[2 * LASWP_MAXP];
  __shared__ int s_src[2 * LASWP_MAXP];
  __shared__ T s_val[LASWP_NC][2 * LASWP_MAXP + 1];
  const int tid = threadIdx.x;
  laswp_compose(piv, npiv, reverse, s_piv, s_tgt, s_row, s_src);
  const int nslot = 2 * npiv;
  const int ncols = n0 + n1;
  const int cbase = blockIdx.x * LASWP_NC;
  // load: consecutive threads take consecutive slots of one column
  // (consecutive columns of one slot when TR)
  for (int e = tid; e < LASWP_NC * nslot; e += blockDim.x) {
    const int cl = TR ? e % LASWP_NC : e / nslot, s = TR ? e / LASWP_NC : e % nslot;
    const int t = cbase + cl;
    if (t >= ncols || s_row[s] < 0) continue;
    const long col = t < n0 ? c0 + t : c1 + (t - n0);
    const long row = (long)row0 + s_row[s];
    s_val[cl][s] = TR ? A[col + row * ld] : A[row + col * ld];
  }
  __syncthreads();
  for (int e = tid; e < LASWP_NC * nslot; e += blockDim.x) {
    const int cl = TR ? e % LASWP_NC : e / nslot, s = TR ? e / LASWP_NC : e % nslot;
    const int t = cbase + cl;
    if (t >= ncols || s_row[s] < 0 || s_src[s] == s) continue;
    const long col = t < n0 ? c0 + t : c1 + (t - n0);
    const long row = (long)row0 + s_row[s];
    (TR ? A[col + row * ld] : A[row + col * ld]) = s_val[cl][s_src[s]];
  }
}

__global__ void laswp_kernel(double* A, long ld, int row0, const int* __restrict__ piv, int npiv,
                             int c0, int n0, int c1, int n1, int reverse) {
  extern __shared__ int sp[];
  for (int i = threadIdx.x; i < npiv; i += blockDim.x) sp[i] = piv[i];
  __syncthreads();
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n0 + n1) return;
  const int col = t < n0 ? c0 + t : c1 + (t - n0);
  double* a = A + (long)col * ld;
  if (!reverse) {
    for (int i = 0; i < npiv; ++i) {
      const int p = sp[i];
      if (p != 0) {
        const long r1 = row0 + i, r2 = r1 + p;
        const double x = a[r1];
        a[r1] = a[r2];
        a[r2] = x;
      }
    }
  } else {
    for (int i = npiv - 1; i >= 0; --i) {
      const int p = sp[i];
      if (p != 0) {
        const long r1 = row0 + i, r2 = r1 + p;
        const double x = a[r1];
        a[r1] = a[r2];
        a[r2] = x;
      }
    }
  }
}

bool g_attrs = false;
void set_attrs() {
  if (g_attrs) return;
  cudaFuncSetAttribute(lu_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(220 * 1024));
  g_attrs = true;
}


}  // namespace

template <typename T>
int laswp_blocked(T* A, long ld, int row0, const int* d_piv, int npiv, int c0, int n0, int c1, int n1,
                  bool reverse, bool tr, cudaStream_t st) {
  const int ncols = n0 + n1;
  const int ps = prof_begin(st);
  const unsigned grid = (unsigned)((ncols + LASWP_NC - 1) / LASWP_NC);
  if (tr)
    laswp_apply_kernel<T, true><<<grid, 256, 0, st>>>(A, ld, row0, d_piv, npiv, reverse ? 1 : 0, c0, n0, c1, n1);
  else
    laswp_apply_kernel<T, false><<<grid, 256, 0, st>>>(A, ld, row0, d_piv, npiv, reverse ? 1 : 0, c0, n0, c1, n1);
  prof_end(ps, st, PROF_SWAP, 0.0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

int laswp_dev(double* A, long ld, int row0, const int* d_piv, int npiv, int c0, int n0, int c1,
              int n1, bool reverse, cudaStream_t st) {
  const int ncols = n0 + n1;
  if (ncols <= 0 || npiv <= 0) return FLA_SUCCESS;
  if (npiv <= LASWP_MAXP) return laswp_blocked<double>(A, ld, row0, d_piv, npiv, c0, n0, c1, n1, reverse, false, st);
  const int threads = 128;
  const int ps = prof_begin(st);
  laswp_kernel<<<(ncols + threads - 1) / threads, threads, npiv * sizeof(int), st>>>(
      A, ld, row0, d_piv, npiv, c0, n0, c1, n1, reverse ? 1 : 0);
  prof_end(ps, st, PROF_SWAP, 0.0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// Row interchanges on a transposed matrix (see laswp_apply_kernel<T, true>),
// in chunks of at most LASWP_MAXP interchanges.
template <typename T>
int laswp_t_any(T* AT, long ldt, int row0, const int* d_piv, int npiv, int c0, int n0, int c1, int n1,
                cudaStream_t st) {
  const int ncols = n0 + n1;
  if (ncols <= 0 || npiv <= 0) return FLA_SUCCESS;
  for (int i0 = 0; i0 < npiv; i0 += LASWP_MAXP) {
    const int cnt = std::min(LASWP_MAXP, npiv - i0);
    if (laswp_blocked<T>(AT, ldt, row0 + i0, d_piv + i0, cnt, c0, n0, c1, n1, false, true, st) != FLA_SUCCESS)
      return FLA_FAILURE;
  }
  return FLA_SUCCESS;
}
int laswp_t_dev(double* AT, long ldt, int row0, const int* d_piv, int npiv, int c0, int n0, int c1, int n1,
                cudaStream_t st) {
  return laswp_t_any<double>(AT, ldt, row0, d_piv, npiv, c0, n0, c1, n1, st);
}
int laswp_t_f32(float* AT, long ldt, int row0, const int* d_piv, int npiv, int c0, int n0, int c1, int n1,
                cudaStream_t st) {
  return laswp_t_any<float>(AT, ldt, row0, d_piv, npiv, c0, n0, c1, n1, st);
}

// Row order produced by the interchanges i <-> i + p[i], i = 0..npiv-1 (in
// reverse order when `reverse`), on rows 0..mrows-1 of a block: src[r] is
// the original row that ends in row r.  One thread applies the sequence to
// the identity, in shared memory when it fits.
__global__ void pivot_perm_kernel(const int* __restrict__ piv, int npiv, int mrows, int reverse,
                                  int* __restrict__ src, int use_smem) {
  extern __shared__ int sv[];
  int* v = use_smem ? sv : src;
  for (int i = threadIdx.x; i < mrows; i += blockDim.x) v[i] = i;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < npiv; ++q) {
      const int i = reverse ? npiv - 1 - q : q;
      const int t = i + piv[i];
      const int x = v[i];
      v[i] = v[t];
      v[t] = x;
    }
  }
  __syncthreads();
  if (use_smem)
    for (int i = threadIdx.x; i < mrows; i += blockDim.x) src[i] = v[i];
}
// T(r, c) = A(src[r], c) for the mrows x ncols block; then copied back
__global__ void gather_rows_f64_kernel(const double* __restrict__ A, long lda, const int* __restrict__ src,
                                       double* __restrict__ T, long ldt, int mrows, int ncols) {
  const long total = (long)mrows * ncols;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long r = e % mrows, c = e / mrows;
    T[r + c * ldt] = A[src[r] + c * lda];
  }
}

int apply_pivots_dev(DMat A, const int* d_piv, int k1, int k2, bool reverse, cudaStream_t st) {
  // FLA_Apply_pivots_ln_opd_var1 (src/lapack/util/app/piv/ln/flamec/
  // FLA_Apply_pivots_ln_opt_var1.c:274-340): swap rows i and i + p[i].
  const int npiv = k2 - k1 + 1;
  if (npiv <= 0 || A.n <= 0) return FLA_SUCCESS;
  const long mrows = A.m - k1;
  if (A.n <= 64 && npiv > LASWP_MAXP && mrows <= INT_MAX) {
    // few columns, many interchanges (the solves): compose the whole
    // sequence into one row order, gather the block, copy it back
    int* src = (int*)ws_get(WS_PERM, sizeof(int) * ((size_t)mrows + 64));
    double* T = (double*)ws_get(WS_PERM_T, sizeof(double) * (size_t)mrows * (size_t)A.n);
    if (!src || !T) return FLA_FAILURE;
    const size_t sb = sizeof(int) * (size_t)mrows;
    const bool smem = sb <= 200 * 1024;
    if (smem) cudaFuncSetAttribute(pivot_perm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    pivot_perm_kernel<<<1, 1024, smem ? sb : 0, st>>>(d_piv + k1, npiv, (int)mrows, reverse ? 1 : 0, src,
                                                       smem ? 1 : 0);
    const long total = mrows * A.n;
    gather_rows_f64_kernel<<<(unsigned)std::min<long>(8192, (total + 255) / 256), 256, 0, st>>>(
        A.p + k1, A.ld, src, T, mrows, (int)mrows, (int)A.n);
    count_launch(2);
    FB_CK(cudaGetLastError());
    FB_CK(cudaMemcpy2DAsync(A.p + k1, sizeof(double) * A.ld, T, sizeof(double) * mrows, sizeof(double) * mrows,
                            A.n, cudaMemcpyDeviceToDevice, st));
    return FLA_SUCCESS;
  }
  // otherwise blocks of LASWP_MAXP interchanges (composed per block)
  const int chunk = LASWP_MAXP;
  if (!reverse) {
    for (int i0 = k1; i0 <= k2; i0 += chunk) {
      int cnt = std::min(chunk, k2 - i0 + 1);
      if (laswp_dev(A.p, A.ld, i0, d_piv + i0, cnt, 0, (int)A.n, 0, 0, false, st) != FLA_SUCCESS)
        return FLA_FAILURE;
    }
  } else {
    int nchunks = (k2 - k1 + chunk) / chunk;
    for (int cidx = nchunks - 1; cidx >= 0; --cidx) {
      int i0 = k1 + cidx * chunk;
      int cnt = std::min(chunk, k2 - i0 + 1);
      if (laswp_dev(A.p, A.ld, i0, d_piv + i0, cnt, 0, (int)A.n, 0, 0, true, st) != FLA_SUCCESS)
        return FLA_FAILURE;
    }
  }
  return FLA_SUCCESS;
}

// Blocked left triangular solve  B := inv(op(T)) B  for an n x n triangular
// T and an n x nrhs block B: 128-row diagonal solves (trsm_block) and GEMM
// updates of the rows not yet solved.  Replaces the dtrsm_ calls of
// FLA_Chol_solve / FLA_LU_piv_solve (FLA_Chol_solve.c:24-33,
// FLA_LU_piv_solve.c:22-27).
int trsm_left_dev(DMat T, DMat B, bool lower, bool trans, bool unit, cudaStream_t st) {
  const long n = T.m, nr = B.n;
  if (n == 0 || nr == 0) return FLA_SUCCESS;
  const bool fwd = (lower != trans);
  const long nblk = (n + NBMAX - 1) / NBMAX;
  if (nr <= 256 && n > NBMAX && tma_ok(T.p, T.ld) && tma_ok(B.p, B.ld)) {
    // Few right-hand sides: every diagonal block's inverse in one launch,
    // then per block X_b := op(inv(T_bb)) B_b and the update of the rows
    // still to solve, both DMMA GEMMs (no 128-step substitution chain).
    double* Inv = (double*)ws_get(WS_TRINV, sizeof(double) * (size_t)nblk * NBMAX * NBMAX);
    const long ldw = NBMAX;
    double* W = (double*)ws_get(WS_SOLVE_W, sizeof(double) * (size_t)ldw * (size_t)nr);
    if (!Inv || !W) return FLA_FAILURE;
    if (tri_inverse_blocks(T.p, T.ld, n, lower, unit, Inv, st) != FLA_SUCCESS) return FLA_FAILURE;
    for (long bi = 0; bi < nblk; ++bi) {
      const long jb = fwd ? bi * NBMAX : (nblk - 1 - bi) * NBMAX;
      const int b = (int)std::min<long>(NBMAX, n - jb);
      double* Bj = B.p + jb;
      const double* Ij = Inv + (jb / NBMAX) * NBMAX * NBMAX;
      // op(inv(T_bb)) = inv(op(T_bb))
      if (gemm_f64(st, trans, false, b, nr, b, 1.0, Ij, NBMAX, Bj, B.ld, 0.0, W, ldw) != FLA_SUCCESS)
        return FLA_FAILURE;
      FB_CK(cudaMemcpy2DAsync(Bj, sizeof(double) * B.ld, W, sizeof(double) * ldw, sizeof(double) * b, nr,
                              cudaMemcpyDeviceToDevice, st));
      if (fwd) {
        const long rest = n - jb - b;
        if (rest <= 0) continue;
        const double* Tblk = trans ? (T.p + jb + (jb + b) * T.ld) : (T.p + (jb + b) + jb * T.ld);
        if (gemm_f64(st, trans, false, rest, nr, b, -1.0, Tblk, T.ld, W, ldw, 1.0, B.p + jb + b, B.ld) !=
            FLA_SUCCESS)
          return FLA_FAILURE;
      } else {
        if (jb == 0) continue;
        const double* Tblk = trans ? (T.p + jb) : (T.p + jb * T.ld);
        if (gemm_f64(st, trans, false, jb, nr, b, -1.0, Tblk, T.ld, W, ldw, 1.0, B.p, B.ld) != FLA_SUCCESS)
          return FLA_FAILURE;
      }
    }
    return FLA_SUCCESS;
  }
  for (long bi = 0; bi < nblk; ++bi) {
    const long jb = fwd ? bi * NBMAX : (nblk - 1 - bi) * NBMAX;
    const int b = (int)std::min<long>(NBMAX, n - jb);
    const double* Tjj = T.p + jb + jb * T.ld;
    double* Bj = B.p + jb;
    if (trsm_block(Tjj, T.ld, Bj, B.ld, b, nr, lower, trans, unit, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (fwd) {
      const long rest = n - jb - b;
      if (rest <= 0) continue;
      // rows below: B2 -= op(T)(jb+b:, jb:jb+b) Bj
      const double* Tblk = trans ? (T.p + jb + (jb + b) * T.ld)   // stored b x rest (upper, transposed)
                                 : (T.p + (jb + b) + jb * T.ld);  // stored rest x b (lower)
      if (gemm_f64(st, trans, false, rest, nr, b, -1.0, Tblk, T.ld, Bj, B.ld, 1.0, B.p + jb + b, B.ld) !=
          FLA_SUCCESS)
        return FLA_FAILURE;
    } else {
      if (jb == 0) continue;
      // rows above: B0 -= op(T)(0:jb, jb:jb+b) Bj
      const double* Tblk = trans ? (T.p + jb)               // stored b x jb (lower, transposed)
                                 : (T.p + jb * T.ld);       // stored jb x b (upper)
      if (gemm_f64(st, trans, false, jb, nr, b, -1.0, Tblk, T.ld, Bj, B.ld, 1.0, B.p, B.ld) != FLA_SUCCESS)
        return FLA_FAILURE;
    }
  }
  return FLA_SUCCESS;
}

// Outer blocksize of FLA_LU_piv (the reference's 128,
// FLA_LU_piv_cntl_init.c:29-74); FLA_B200_LU_BLOCKSIZE (a multiple of 16,
// 16..256) overrides it for tuning.
int lu_blocksize() {
  static int nb = 0;
  if (nb == 0) {
    nb = NBMAX;
    if (const char* e = std::getenv("FLA_B200_LU_BLOCKSIZE")) {
      const int v = std::atoi(e);
      if (v >= 16 && v <= 256 && v % 16 == 0) nb = v;
    }
  }
  return nb;
}

// Blocked right-looking LU with a lookahead of one panel, run on A^T.
//
// Row interchanges are the costly part of partial pivoting in column-major
// storage: every interchange touches one element per column, 8-byte pieces
// scattered over HBM.  The factorization therefore works on AT = A^T (a
// workspace, n x m column-major), where a row of A is a contiguous column
// of AT and every interchange moves contiguous pieces; A is transposed in
// at the start and back at the end (two streaming passes).
//
//   main stream, step k:  the next panel's columns only: row interchanges
//                         of panel k, U12 (substitution), lookahead update
//                         A22^T(next panel rows) -= U12^T(next) A21^T;
//   side stream:          factor the next panel (cluster leaves, recursive
//                         split);
//   main stream:          concurrently, the other columns: interchanges
//                         left of panel k and right of the next panel,
//                         their U12 and A22^T(rest) -= U12^T(rest) A21^T;
//                         then wait for the side stream.
// Only three launches stand between the end of one panel and the start of
// the next.  The side stream has the higher priority, so the panel's CTAs
// are placed as soon as trailing-update CTAs retire.
// U12 := inv(L11) A12 on the transposed storage by forward substitution,
// the order of dtrsm's left, lower, no-transpose, unit case
// (src/flablas/f2c/dtrsm.c): for j = 0..b-1, rows i > j of every column c
// lose L11(i, j) U12(j, c).  L11(i, j) is at Ls[j + i ld] (row i of L11 is
// a contiguous column of A^T), A12(i, c) at X[c + i ld], overwritten.
// The triangle (b <= 128) sits in shared memory; one warp per RV columns c
// keeps rows lane, lane+32, lane+64, lane+96 of them in registers, and at
// step j the owner lane broadcasts U12(j, c): no block barrier inside the
// sweep, so a step costs one shuffle and a few FMAs of latency.
constexpr int U12_WARPS = 16;
constexpr int U12_LDS = NBMAX + 1;  // odd stride: a half-warp reads 16 banks
// shared memory for a triangle of order b: whole 32-row groups (the sweep
// reads the rows of every group it touches)
// (and, after it, the reciprocals of the diagonal for the non-unit form)
inline size_t u12_smem(int b) { return sizeof(double) * ((size_t)((b + 31) & ~31) * U12_LDS + NBMAX); }

// NU = false: unit lower L11 with L11(i, j) at Ls[j + i ld] (the LU on A^T).
// NU = true:  non-unit lower L11 with L11(i, j) at Ls[i + j ld] (column-
//             major, the Cholesky's A21 := A21 inv(L11)^T, rows of A21 as
//             the right-hand sides); each solved entry is first multiplied
//             by the reciprocal of its pivot (dtrsm's R,L,T,N case).
// Returns at once when *guard holds a failing column below guard_limit.
// TX: the element type of X (float for the low-precision Cholesky's
// factors: loaded into FP64, solved in FP64, rounded back); X has its own
// leading dimension ldx.
template <int RV, bool NU, typename TX = double>
__global__ void __launch_bounds__(U12_WARPS * 32) u12_subst_kernel(const double* __restrict__ Ls,
                                                                    TX* __restrict__ X, long ld, int b,
                                                                    int ncols, const int* guard, int guard_limit,
                                                                    long ldx) {
  extern __shared__ double sL[];  // sL[i * U12_LDS + j] = L11(i, j), rows i < 32 ceil(b / 32)
  double* sR = sL + ((b + 31) & ~31) * U12_LDS;
  if (guard && *((volatile const int*)guard) < guard_limit) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // The triangle: lanes run along its contiguous index e (a column of L11
  // for NU, a row for the transposed storage), each warp takes every
  // sixteenth line o; sixteen loads per lane are in flight before they are
  // stored (one memory round trip per batch, not per entry).
  for (int o0 = warp; o0 < b; o0 += U12_WARPS * 4) {
    double v[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int o = o0 + a * U12_WARPS, e = lane + 32 * q;
        v[a][q] = (o < b && e < b) ? Ls[e + (long)o * ld] : 0.0;
      }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int o = o0 + a * U12_WARPS, e = lane + 32 * q;
        if (o < b && e < b) {
          if (NU) {
            sL[e * U12_LDS + o] = v[a][q];  // L11(e, o)
            if (e == o) sR[o] = 1.0 / v[a][q];
          } else {
            sL[o * U12_LDS + e] = v[a][q];  // L11(o, e)
          }
        }
      }
  }
  __syncthreads();
  const int c0 = (blockIdx.x * U12_WARPS + warp) * RV;
  if (c0 >= ncols) return;
  double r[4][RV];
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int v = 0; v < RV; ++v) {
      const int i = lane + 32 * m, c = c0 + v;
      r[m][v] = (i < b && c < ncols) ? (double)X[c + (long)i * ldx] : 0.0;
    }
  // rows at or beyond b hold zeros and read unset shared memory of their
  // group: they are never written back; groups at or beyond b are skipped
  const int groups = (b + 31) >> 5;
#pragma unroll
  for (int slot = 0; slot < 4; ++slot) {
    if (slot >= groups) break;
    const int jend = min(32, b - 32 * slot);
    for (int jj = 0; jj < jend; ++jj) {
      const int j = 32 * slot + jj;
      double y[RV];
#pragma unroll
      for (int v = 0; v < RV; ++v) y[v] = __shfl_sync(0xffffffffu, r[slot][v], jj);
      if (NU) {
        const double rc = sR[j];
#pragma unroll
        for (int v = 0; v < RV; ++v) {
          y[v] *= rc;
          if (lane == jj) r[slot][v] = y[v];
        }
      }
      const double l0 = sL[(lane + 32 * slot) * U12_LDS + j];
      if (lane > jj) {
#pragma unroll
        for (int v = 0; v < RV; ++v) r[slot][v] = fma(-l0, y[v], r[slot][v]);
      }
#pragma unroll
      for (int m = slot + 1; m < 4; ++m) {
        if (m < groups) {
          const double l = sL[(lane + 32 * m) * U12_LDS + j];
#pragma unroll
          for (int v = 0; v < RV; ++v) r[m][v] = fma(-l, y[v], r[m][v]);
        }
      }
    }
  }
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int v = 0; v < RV; ++v) {
      const int i = lane + 32 * m, c = c0 + v;
      if (i < b && c < ncols) X[c + (long)i * ldx] = (TX)r[m][v];
    }
}

template <int RV, bool NU = false, typename TX = double>
void u12_subst_launch(const double* Ls, TX* X, long ld, int b, int ncols, cudaStream_t st,
                      const int* guard = nullptr, int guard_limit = 0, long ldx = -1) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(u12_subst_kernel<RV, NU, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)u12_smem(NBMAX));
    attr = true;
  }
  const unsigned grid = (unsigned)((ncols + U12_WARPS * RV - 1) / (U12_WARPS * RV));
  u12_subst_kernel<RV, NU, TX><<<grid, U12_WARPS * 32, u12_smem(b), st>>>(Ls, X, ld, b, ncols, guard, guard_limit,
                                                                         ldx < 0 ? ld : ldx);
}

// X := X inv(L)^T for an ncols x b block X (column-major, ld ld) and a
// non-unit lower L of order b <= 128 (column-major, same ld): the
// Cholesky's A21 := A21 inv(L11)^T by forward substitution in one launch.
int trsm_rlt_subst(const double* L, double* X, long ld, int b, long ncols, const int* guard, int guard_limit,
                   cudaStream_t st) {
  if (ncols <= 0 || b <= 0) return FLA_SUCCESS;
  if (b > NBMAX) {
    set_last_error("trsm_rlt_subst: triangle wider than 128");
    return FLA_FAILURE;
  }
  const int sms = ctx().num_sms;
  const int ps = prof_begin(st);
  if (ncols <= (long)sms * U12_WARPS) u12_subst_launch<1, true>(L, X, ld, b, (int)ncols, st, guard, guard_limit);
  else if (ncols <= (long)sms * U12_WARPS * 2) u12_subst_launch<2, true>(L, X, ld, b, (int)ncols, st, guard, guard_limit);
  else if (ncols <= (long)sms * U12_WARPS * 4) u12_subst_launch<4, true>(L, X, ld, b, (int)ncols, st, guard, guard_limit);
  else u12_subst_launch<8, true>(L, X, ld, b, (int)ncols, st, guard, guard_limit);
  prof_end(ps, st, PROF_TRSM, (double)ncols * b * b);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// The same for an FP32 X (ld ldx) against an FP64 L (ld ldl): the
// low-precision Cholesky's A21 := A21 inv(L11)^T with L11 its FP64
// diagonal factor, solved in FP64 and rounded to FP32.
int trsm_rlt_subst_f32(const double* L, long ldl, float* X, long ldx, int b, long ncols, const int* guard,
                       int guard_limit, cudaStream_t st) {
  if (ncols <= 0 || b <= 0) return FLA_SUCCESS;
  if (b > NBMAX) {
    set_last_error("trsm_rlt_subst_f32: triangle wider than 128");
    return FLA_FAILURE;
  }
  const int sms = ctx().num_sms;
  const int ps = prof_begin(st);
  if (ncols <= (long)sms * U12_WARPS)
    u12_subst_launch<1, true, float>(L, X, ldl, b, (int)ncols, st, guard, guard_limit, ldx);
  else if (ncols <= (long)sms * U12_WARPS * 2)
    u12_subst_launch<2, true, float>(L, X, ldl, b, (int)ncols, st, guard, guard_limit, ldx);
  else if (ncols <= (long)sms * U12_WARPS * 4)
    u12_subst_launch<4, true, float>(L, X, ldl, b, (int)ncols, st, guard, guard_limit, ldx);
  else
    u12_subst_launch<8, true, float>(L, X, ldl, b, (int)ncols, st, guard, guard_limit, ldx);
  prof_end(ps, st, PROF_TRSM, (double)ncols * b * b);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// U12 := inv(L11) A12 for ncols columns (layout above), any b: blocks of
// 128 rows, each solved by the kernel, the rows below updated by a GEMM.
// Columns per warp grow with ncols so that the grid stays about one wave
// (a 128-row triangle's 132 KB of shared memory allow one CTA per SM).
int u12_subst(const double* Ls, double* X, long ld, int b, long ncols, cudaStream_t st) {
  if (ncols <= 0 || b <= 0) return FLA_SUCCESS;
  const int sms = ctx().num_sms;
  for (int r0 = 0; r0 < b; r0 += NBMAX) {
    const int bb = std::min(NBMAX, b - r0);
    const double* L = Ls + r0 + (long)r0 * ld;
    double* Y = X + (long)r0 * ld;
    const int ps = prof_begin(st);
    if (ncols <= (long)sms * U12_WARPS) u12_subst_launch<1>(L, Y, ld, bb, (int)ncols, st);
    else if (ncols <= (long)sms * U12_WARPS * 2) u12_subst_launch<2>(L, Y, ld, bb, (int)ncols, st);
    else if (ncols <= (long)sms * U12_WARPS * 4) u12_subst_launch<4>(L, Y, ld, bb, (int)ncols, st);
    else u12_subst_launch<8>(L, Y, ld, bb, (int)ncols, st);
    prof_end(ps, st, PROF_TRSM, (double)ncols * bb * bb);
    count_launch();
    FB_CK(cudaGetLastError());
    const int rest = b - r0 - bb;
    // U12^T[:, r0+bb:] -= U12^T[:, r0:r0+bb] L11^T[r0:r0+bb, r0+bb:]
    if (rest > 0 && gemm_f64(st, false, false, ncols, rest, bb, -1.0, Y, ld, Ls + r0 + (long)(r0 + bb) * ld, ld,
                             1.0, X + (long)(r0 + bb) * ld, ld) != FLA_SUCCESS)
      return FLA_FAILURE;
  }
  return FLA_SUCCESS;
}

int lu_piv_dev(DMat A, int* d_piv, int* info) {
  set_attrs();
  Context& cx = ctx();
  cudaStream_t st = cx.stream, sd = cx.side;
  const long m = A.m, n = A.n, mn = std::min(m, n);
  *info = -1;
  if (mn == 0) return FLA_SUCCESS;
  auto even = [](long x) { return (x + 1) & ~1L; };  // TMA: 16-byte leading dimensions
  const int NBL = (int)std::min<long>(lu_blocksize(), mn);
  // Width of the panel starting at column k: twice NBL while more than
  // wide_rows rows remain (the trailing updates dominate there, and K = 2 NBL
  // halves each update tile's fixed cost), NBL after (the panels dominate;
  // at n = 16384 that is the last ~8000 rows, and an n = 8192 factorization
  // is panel-bound from the start).  FLA_B200_LU_WIDE_ROWS overrides it.
  static const long wide_rows = [] {
    long v = 8192;
    if (const char* e = std::getenv("FLA_B200_LU_WIDE_ROWS")) v = std::atol(e);
    return v;
  }();
  auto width = [&](long k) -> int {
    const int w = (NBL <= 128 && m - k > wide_rows) ? 2 * NBL : NBL;
    return (int)std::min<long>(w, mn - k);
  };
  const long ldT = even(n);
  double* AT = (double*)ws_get(WS_REPACK, sizeof(double) * (size_t)ldT * (size_t)m);
  if (!AT) return FLA_FAILURE;
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;
  cudaEvent_t ev_look = cx.ev[0], ev_panel = cx.ev[1];
  // element (i, j) of A inside AT
  auto t_at = [&](long i, long j) { return AT + j + i * ldT; };
  if (transpose_dev(A.p, A.ld, AT, ldT, m, n, false, st) != FLA_SUCCESS) return FLA_FAILURE;

  // FLA_B200_LU_TRACE: per-step event timeline (main stream: step start,
  // lookahead done, trailing update done; side stream: panel done), summed
  // and printed to stderr after the factorization
  static const bool trace = std::getenv("FLA_B200_LU_TRACE") != nullptr;
  static const bool trace_all = trace && std::string(std::getenv("FLA_B200_LU_TRACE")) == "all";
  std::vector<cudaEvent_t> tev;
  auto tmark = [&](cudaStream_t s) {
    if (!trace) return;
    cudaEvent_t e;
    cudaEventCreate(&e);
    cudaEventRecord(e, s);
    tev.push_back(e);
  };
  auto tdrop = [&](size_t keep) {  // an incomplete step is not traced
    for (size_t q = keep; q < tev.size(); ++q) cudaEventDestroy(tev[q]);
    tev.resize(std::min(keep, tev.size()));
  };
  // first panel, on the main stream
  {
    const int b = width(0);
    if (lu_panel_factor_t(AT, ldT, m, b, d_piv, 0, st) != FLA_SUCCESS) return FLA_FAILURE;
  }
  for (long k = 0, b = 0; k < mn; k += b) {
    b = width(k);
    const long nr = n - k - b, m2 = m - k - b;
    const size_t tbase = tev.size();
    tmark(st);
    // next panel's width (0: none); its columns go first, the rest of the
    // step's work runs on this stream while the side stream factors it
    const int nb2 = (nr > 0 && m2 > 0 && k + b < mn) ? width(k + b) : 0;
    if (nb2 == 0) {
      if (laswp_t_dev(AT, ldT, (int)k, d_piv + k, b, 0, (int)k, (int)(k + b), (int)nr, st) != FLA_SUCCESS)
        return FLA_FAILURE;
      if (nr <= 0) {
        tdrop(tbase);
        continue;
      }
      if (u12_subst(t_at(k, k), t_at(k, k + b), ldT, b, nr, st) != FLA_SUCCESS) return FLA_FAILURE;
      tdrop(tbase);
      continue;
    }
    // the next panel's columns: interchanges, U12, lookahead update
    if (laswp_t_dev(AT, ldT, (int)k, d_piv + k, b, (int)(k + b), nb2, 0, 0, st) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (u12_subst(t_at(k, k), t_at(k, k + b), ldT, b, nb2, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (gemm_f64(st, false, false, nb2, m2, b, -1.0, t_at(k, k + b), ldT, t_at(k + b, k), ldT, 1.0,
                 t_at(k + b, k + b), ldT) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_look, st));
    tmark(st);
    FB_CK(cudaStreamWaitEvent(sd, ev_look, 0));
    if (lu_panel_factor_t(t_at(k + b, k + b), ldT, m2, nb2, d_piv + k + b, (int)(k + b), sd) != FLA_SUCCESS)
      return FLA_FAILURE;
    FB_CK(cudaEventRecord(ev_panel, sd));
    tmark(sd);
    // the rest, beside the panel: interchanges left of the panel and right of
    // the next one (disjoint from the columns the side stream works on),
    // U12 of the remaining columns, trailing update
    if (laswp_t_dev(AT, ldT, (int)k, d_piv + k, b, 0, (int)k, (int)(k + b + nb2), (int)(nr - nb2), st) !=
        FLA_SUCCESS)
      return FLA_FAILURE;
    if (u12_subst(t_at(k, k), t_at(k, k + b + nb2), ldT, b, nr - nb2, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (nr > nb2 &&
        gemm_f64(st, false, false, nr - nb2, m2, b, -1.0, t_at(k, k + b + nb2), ldT, t_at(k + b, k), ldT, 1.0,
                 t_at(k + b, k + b + nb2), ldT) != FLA_SUCCESS)
      return FLA_FAILURE;
    tmark(st);
    if (tev.size() != tbase + 4) tdrop(tbase);
    FB_CK(cudaStreamWaitEvent(st, ev_panel, 0));
  }
  if (transpose_dev(AT, ldT, A.p, A.ld, n, m, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  const int rs = status_read(info);
  if (trace && !tev.empty()) {
    // per step: [0] start, [1] lookahead done, [2] panel done, [3] trailing done
    double serial = 0, panel = 0, trail = 0, crit = 0;
    int panel_bound = 0;
    const size_t steps = tev.size() / 4;
    for (size_t q = 0; q < steps; ++q) {
      float a = 0, p = 0, t = 0;
      cudaEventElapsedTime(&a, tev[4 * q], tev[4 * q + 1]);
      cudaEventElapsedTime(&p, tev[4 * q + 1], tev[4 * q + 2]);
      cudaEventElapsedTime(&t, tev[4 * q + 1], tev[4 * q + 3]);
      serial += a;
      panel += p;
      trail += t;
      crit += a + std::max(p, t);
      if (p > t) ++panel_bound;
      if (trace_all || q % 16 == 0 || q + 1 == steps)
        std::fprintf(stderr, "libflame_b200 lu: step %4zu  lookahead %.3f ms  panel %.3f ms  trailing %.3f ms\n", q, a, p,
                     t);
    }
    std::fprintf(stderr,
                 "libflame_b200 lu: %zu steps: lookahead part %.2f ms, panels %.2f ms, trailing %.2f ms, "
                 "critical %.2f ms, %d steps panel-bound\n",
                 steps, serial, panel, trail, crit, panel_bound);
    for (cudaEvent_t e : tev) cudaEventDestroy(e);
  }
  return rs;
}

}  // namespace fb

namespace fb {

// ===========================================================================
// Allocation-free LU panel factorization.
//
// Some callers cannot let a library call cudaMalloc: a caller whose own
// memory manager has reserved the device memory up front (an allocator
// that owns the HBM pool, a service with a fixed memory budget) sees a
// stray cudaMalloc fail or break its accounting, and a latency-bound caller
// cannot afford cudaMalloc/cudaFree, which may synchronize the device.
// FLA_B200_LU_piv_panel_noalloc gives them the LU panel factorization (the
// kernel above) with its scratch (pivot candidates, exchanged rows, the
// grid-barrier counter and the status words) in a fixed array in device
// memory that is part of the loaded library, so the call allocates nothing.
//
// Limits: panels of at most kNaMaxCols columns, m >= n, and a panel
// geometry of at most kNaMaxCtas CTAs whose row slab fits in shared memory
// (m up to about 29,000 rows on a 148-SM B200 for 128 columns).  The array
// (about 334 KB) is held by every GPU that loads the library until the
// process exits.  Every call on a device uses the same array and finds the
// previous call's contents there; the barrier counter and status words are
// cleared at the start of each call.  Calls whose work overlaps on the GPU
// (concurrent streams, or several host threads) race on the array and must
// be serialized by the caller.
// ===========================================================================
namespace {

constexpr int kNaMaxCtas = 160;
constexpr int kNaMaxCols = 128;

struct NoAllocScratch {
  double cand_row[2 * kNaMaxCtas * kNaMaxCols];
  double cand_val[2 * kNaMaxCtas];
  double diag_row[2 * kNaMaxCols];
  int cand_idx[2 * kNaMaxCtas];
  unsigned bar;
  int status[2];  // [0] wait-timeout flag, [1] first null pivot (INT_MAX: none)
};

// The scratch itself: a file-scope device array of fixed size.
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Device address of g_noalloc_scratch, looked up once per device.  In host
// code the array's name is only a host-side stand-in, so the address must
// come from cudaGetSymbolAddress with that device current.
constexpr int kNaMaxDevices = 64;
NoAllocScratch* g_na_ptr[kNaMaxDevices] = {};
std::mutex g_na_mutex;

__global__ void noalloc_reset_kernel(NoAllocScratch* s) {
  s->bar = 0u;
  s->status[0] = 0;
  s->status[1] = INT_MAX;
}

}  // namespace

}  // namespace fb

// No counterpart in the reference libflame (see include/FLAME_b200.h).
extern "C" int FLA_B200_LU_piv_panel_noalloc(int m, int n, double* A, int lda, int* piv,
                                             void* stream) {
  using namespace fb;
  if (m < 0 || n < 0 || n > kNaMaxCols || m < n) {
    set_last_error("FLA_B200_LU_piv_panel_noalloc: need 0 <= n <= 128 and m >= n (got m=" +
                   std::to_string(m) + ", n=" + std::to_string(n) + ")");
    return FLA_FAILURE;
  }
  if (lda < (m > 1 ? m : 1)) {
    set_last_error("FLA_B200_LU_piv_panel_noalloc: lda < max(1, m)");
    return FLA_FAILURE;
  }
  if (n == 0) return FLA_SUCCESS;
  if (!A || !piv || !is_device_ptr(A) || !is_device_ptr(piv)) {
    set_last_error("FLA_B200_LU_piv_panel_noalloc: A and piv must be device pointers");
    return FLA_FAILURE;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNaMaxDevices) {
    cudaGetLastError();
    set_last_error("FLA_B200_LU_piv_panel_noalloc: no usable current device");
    return FLA_FAILURE;
  }
  NoAllocScratch* s = nullptr;
  {
    // Set-up, once per device, with that device current.  The first call on
    // a device does it, so that first call should come before any stream
    // capture.
    std::lock_guard<std::mutex> lk(g_na_mutex);
    if (!g_na_ptr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || p == nullptr) {
        cudaGetLastError();
        set_last_error(std::string("FLA_B200_LU_piv_panel_noalloc: cudaGetSymbolAddress failed: ") +
                       cudaGetErrorString(e));
        return FLA_FAILURE;
      }
      cudaFuncSetAttribute(lu_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(220 * 1024));
      g_na_ptr[dev] = reinterpret_cast<NoAllocScratch*>(p);
    }
    s = g_na_ptr[dev];
  }
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    set_last_error("FLA_B200_LU_piv_panel_noalloc: cannot query the SM count");
    return FLA_FAILURE;
  }
  // Panel geometry: the same rule as the library's LU driver.
  const long M = m;
  const int R = (int)std::max<long>(std::min<long>(M, 32), (M + sms - 1) / sms);
  const int G = (int)((M + R - 1) / R);
  const int lds = R | 1;
  const size_t smem = (size_t)lds * n * 8 + (size_t)n * 8;
  if (G > kNaMaxCtas || smem > PANEL_SMEM_CAP) {
    set_last_error("FLA_B200_LU_piv_panel_noalloc: panel of " + std::to_string(m) + " x " +
                   std::to_string(n) + " exceeds the fixed scratch / shared-memory limits");
    return FLA_FAILURE;
  }
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
  noalloc_reset_kernel<<<1, 1, 0, st>>>(s);
  {
    const cudaError_t re = cudaGetLastError();
    if (re != cudaSuccess) {
      set_last_error(std::string("FLA_B200_LU_piv_panel_noalloc: reset launch failed: ") +
                     cudaGetErrorString(re));
      return FLA_FAILURE;
    }
  }
  count_launch();
  PanelArgs pa;
  pa.P = A;
  pa.ld = lda;
  pa.M = m;
  pa.nb = n;
  pa.R = R;
  pa.lds = lds;
  pa.G = G;
  pa.gcol = 0;
  pa.piv = piv;
  pa.cand_row = s->cand_row;
  pa.cand_val = s->cand_val;
  pa.cand_idx = s->cand_idx;
  pa.diag_row = s->diag_row;
  pa.bar = &s->bar;
  pa.err = &s->status[0];
  pa.info = &s->status[1];
  void* args[] = {&pa};
  cudaError_t e = cudaLaunchCooperativeKernel((void*)lu_panel_kernel, dim3(G), dim3(PANEL_THREADS), args,
                                              smem, st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_error(std::string("FLA_B200_LU_piv_panel_noalloc: launch failed: ") + cudaGetErrorString(e));
    return FLA_FAILURE;
  }
  count_launch();
  int h[2] = {0, 0};
  e = cudaMemcpyAsync(h, s->status, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_last_error(std::string("FLA_B200_LU_piv_panel_noalloc: ") + cudaGetErrorString(e));
    return FLA_FAILURE;
  }
  if (h[0] != 0) {
    set_last_error("FLA_B200_LU_piv_panel_noalloc: a grid barrier exceeded its wait limit");
    return FLA_FAILURE;
  }
  return h[1] == INT_MAX ? FLA_SUCCESS : h[1];
}
