// LU panel factorization with partial pivoting for the blocked FLA_LU_piv,
// B200 form: a recursive split of the panel whose leaves run inside one
// thread-block cluster.
//
// Reference: the panel step of FLA_LU_piv_blk_var5
// (src/lapack/dec/lu/piv/vars/flamec/FLA_LU_piv_blk_var5.c:52-60), whose leaf
// is the Crout kernel FLA_LU_piv_opt_var4.c:218-331.  Pivot choice is the
// reference's: largest magnitude in the column, the smallest row among
// equals (idamax, src/flablas/f2c/idamax.c:41,60); a column whose largest
// magnitude is zero is neither swapped nor scaled, its index is reported
// (the first one), and the factorization goes on.
//
// Leaf (lu_leaf_cluster_kernel): the M x w leaf is split in row slabs, one
// per CTA of a cluster of up to 16 CTAs, each slab held in shared memory for
// the whole leaf.  Per column: every CTA finds its best candidate row and
// pushes the candidate (magnitude, row, the whole w-wide row) and, if it owns
// it, the current row j into every CTA's shared memory (DSMEM stores); one
// hardware cluster barrier; then every CTA picks the same winner from its
// local copy, the owners of rows j and p(j) exchange them, and each CTA
// scales its part of column j and applies the rank-1 update to its slab.
// Exchange buffers alternate between two halves by column parity, so one
// barrier per column suffices.  Cluster CTAs are co-scheduled by the
// hardware, so the leaf can run on a second stream beside the trailing
// update without any co-residency assumption, and the barrier is not a spin.
//
// Recursion (lu_panel_factor): a panel too wide for the cluster's shared
// memory is split in two halves: factor the left half, swap the right half's
// rows, solve its top block, update the rest with the DMMA GEMM engine,
// factor the lower right half, and swap the left half's lower rows.  The
// relative pivot convention (row i exchanges with row i + p[i]) makes the
// right half's pivot vector a plain suffix of the panel's.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

#include "common.h"
#include "dev_util.cuh"

namespace cg = cooperative_groups;

namespace fb {

namespace {

constexpr int LEAF_THREADS = 1024;
constexpr int LEAF_ROWS_TARGET = 256;  // rows per CTA the cluster size aims at
constexpr int LEAF_MAXC = 16;     // largest cluster
constexpr int LEAF_MAXW = 128;    // widest leaf

struct LeafArgs {
  double* P;   // leaf (row 0, col 0), column-major
  long ld;
  int M;       // rows
  int w;       // columns
  int R;       // rows per CTA
  int lds;     // SMEM leading dimension of the slab
  int gcol;    // global column of leaf column 0 (for info)
  int* piv;    // out: w relative pivots
  int* info;   // atomicMin of the first zero-pivot column
  int* err;    // wait-timeout flag (register-resident leaf)
};

// Shared-memory layout of one CTA (doubles unless noted):
//   slab   [lds * w]
//   xrow   [2][C][w]   candidate rows pushed by each CTA
//   xval   [2][C]      candidate magnitudes
//   rowj   [2][w]      row j pushed by its owner
//   xidx   [2][C] int  candidate global rows (INT_MAX: none)
__host__ __device__ inline size_t leaf_smem_bytes(int lds, int w, int C) {
  return sizeof(double) * ((size_t)lds * w + 2 * (size_t)C * w + 2 * C + 2 * w) + sizeof(int) * 2 * C + 64;
}

// RM: the panel is stored transposed (element (i, col) at P[i * ld + col],
// rows of A being columns of A^T); otherwise column-major.
template <bool RM>
__global__ void __launch_bounds__(LEAF_THREADS, 1) lu_leaf_cluster_kernel(LeafArgs a) {
  extern __shared__ double S[];
  __shared__ double s_rv[LEAF_THREADS / 32];
  __shared__ int s_ri[LEAF_THREADS / 32];
  __shared__ double s_bv;
  __shared__ int s_bi, s_wc, s_r;
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int c = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int w = a.w, lds = a.lds;
  double* slab = S;
  double* xrow = slab + (size_t)lds * w;
  double* xval = xrow + 2 * (size_t)C * w;
  double* rowj = xval + 2 * C;
  int* xidx = reinterpret_cast<int*>(rowj + 2 * w);

  const int r0 = c * a.R;
  const int rows = max(0, min(a.R, a.M - r0));
  if (RM) {
    // eight independent loads in flight per thread
    const int tot = rows * w;
    for (int e0 = tid; e0 < tot; e0 += 8 * LEAF_THREADS) {
      double v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int e = e0 + k * LEAF_THREADS;
        if (e < tot) {
          const int i = e / w, col = e - i * w;
          v[k] = a.P[(long)(r0 + i) * a.ld + col];
        }
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int e = e0 + k * LEAF_THREADS;
        if (e < tot) {
          const int i = e / w, col = e - i * w;
          slab[i + col * lds] = v[k];
        }
      }
    }
  } else {
    for (int col = 0; col < w; ++col)
      for (int i = tid; i < rows; i += LEAF_THREADS) slab[i + col * lds] = a.P[(long)(r0 + i) + (long)col * a.ld];
  }
  __syncthreads();

  // Thread -> (row i = tid mod RT, column group g = tid / RT), RT the slab
  // height rounded up to a power of two (32 .. 1024); with G = 1024 / RT
  // groups, group g updates columns j+1+g, j+1+g+G, ... of its rows, so
  // within a column only the candidate reduction needs a CTA barrier and
  // the exchange one cluster barrier.  Slabs taller than 1024 rows give each
  // thread rows i, i + 1024, ... (G = 1).  Group 0 owns column j + 1 and
  // tracks the next candidate.
  int rt_log = 5;
  while ((1 << rt_log) < rows && rt_log < 10) ++rt_log;
  const int RT = 1 << rt_log, G = LEAF_THREADS >> rt_log;
  const int my_i = tid & (RT - 1), my_g = tid >> rt_log;
  int first_null = -1;
  double bv = -1.0;  // this thread's candidate for the current column
  int bi = INT_MAX;
  if (my_g == 0)
    for (int i = my_i; i < rows; i += RT) {
      const double v = fabs(slab[i]);
      const int gi = r0 + i;
      if (v > bv || (v == bv && gi < bi)) { bv = v; bi = gi; }
    }
  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    // ---- 1. CTA candidate: max |a(i,j)| over rows i >= j, smallest row on
    // ties (warp shuffles, then warp 0 over the warps' results)
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { s_rv[warp] = bv; s_ri[warp] = bi; }
    __syncthreads();
    if (warp == 0) {
      double v = s_rv[lane];  // LEAF_THREADS / 32 == 32 partial results
      int i0 = s_ri[lane];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i0, off);
        if (ov > v || (ov == v && oi < i0)) { v = ov; i0 = oi; }
      }
      if (lane == 0) { s_bv = v; s_bi = i0; }
    }
    __syncthreads();
    bv = s_bv;
    bi = s_bi;
    // a thread's own a(i, j), read before group 0 overwrites it with l(i, j)
    // (one row per thread whenever G > 1)
    const double vj = (G > 1 && my_i < rows) ? slab[my_i + j * lds] : 0.0;
    // ---- 2. push the candidate (and row j, by its owner) to every CTA
    {
      const int li = bi - r0;  // local row of the candidate (if any)
      const bool have = bi != INT_MAX;
      const bool own_j = (j >= r0) && (j < r0 + rows);
      const int per = w + 1;
      for (int e = tid; e < C * per; e += LEAF_THREADS) {
        const int d = e / per, q = e - d * per;
        if (q < w) {
          double* dst = cluster.map_shared_rank(xrow + ((size_t)par * C + c) * w + q, d);
          *dst = have ? slab[li + q * lds] : 0.0;
        } else {
          *cluster.map_shared_rank(xval + par * C + c, d) = bv;
          *cluster.map_shared_rank(xidx + par * C + c, d) = bi;
        }
      }
      if (own_j)
        for (int e = tid; e < C * w; e += LEAF_THREADS) {
          const int d = e / w, q = e - d * w;
          *cluster.map_shared_rank(rowj + par * w + q, d) = slab[(j - r0) + q * lds];
        }
    }
    cluster.sync();
    // ---- 3. winner (identical on every CTA: same data, same order)
    if (warp == 0) {
      double v = -2.0;
      int i0 = INT_MAX, q0 = 0;
      for (int q = lane; q < C; q += 32) {
        const double cv = xval[par * C + q];
        const int ci = xidx[par * C + q];
        if (ci != INT_MAX && (cv > v || (cv == v && ci < i0))) { v = cv; i0 = ci; q0 = q; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i0, off);
        const int oq = __shfl_xor_sync(0xffffffffu, q0, off);
        if (ov > v || (ov == v && oi < i0)) { v = ov; i0 = oi; q0 = oq; }
      }
      if (lane == 0) { s_wc = q0; s_r = i0; }
    }
    __syncthreads();
    int r = s_r;
    const int w0 = s_wc;
    const double* u = xrow + ((size_t)par * C + w0) * w;  // the pivot row
    if (r == INT_MAX) {
      // no orderable candidate (every magnitude NaN): keep row j, as idamax
      // does when no later entry compares greater than the first
      r = j;
      u = rowj + par * w;
    }
    const double* oldj = rowj + par * w;
    const double piv = u[j];
    if (c == 0 && tid == 0) a.piv[j] = r - j;
    bv = -1.0;
    bi = INT_MAX;
    if (piv == 0.0) {
      // null column: no exchange, no scaling, no update
      if (first_null < 0) first_null = j;
      if (j + 1 < w && my_g == 0)
        for (int i = my_i; i < rows; i += RT) {
          const int gi = r0 + i;
          if (gi > j) {
            const double t = fabs(slab[i + (j + 1) * lds]);
            if (t > bv || (t == bv && gi < bi)) { bv = t; bi = gi; }
          }
        }
      continue;
    }
    // ---- 4. exchange rows j and r: warp 0 writes the pivot row into row j,
    // warp 1 the old row j's first j entries into row r; row r's update
    // reads the old row j directly.  Then per row: scale column j below the
    // pivot (reciprocal multiply, as bl1_dinvscalv), rank-1 update of the
    // rest of the row, and (group 0) the row's candidate for column j + 1.
    const double rinv = 1.0 / piv;
    if (r != j) {
      if (warp == 0 && j >= r0 && j < r0 + rows)
        for (int q = lane; q < w; q += 32) slab[(j - r0) + q * lds] = u[q];
      if (warp == 1 && r >= r0 && r < r0 + rows)
        for (int q = lane; q < j; q += 32) slab[(r - r0) + q * lds] = oldj[q];
    }
    for (int i = my_i; i < rows; i += RT) {
      const int gi = r0 + i;
      if (gi <= j) continue;
      const double* src = (gi == r) ? oldj : nullptr;
      const double l = (src ? src[j] : (G > 1 ? vj : slab[i + j * lds])) * rinv;
      int q = j + 1 + my_g;
      if (my_g == 0) {
        slab[i + j * lds] = l;
        if (q < w) {
          const double t = fma(-l, u[q], src ? src[q] : slab[i + q * lds]);
          slab[i + q * lds] = t;
          const double at = fabs(t);
          if (at > bv || (at == bv && gi < bi)) { bv = at; bi = gi; }
          q += G;
        }
      }
      if (src) {
        for (; q < w; q += G) slab[i + q * lds] = fma(-l, u[q], src[q]);
      } else {
        for (; q + G < w; q += 2 * G) {
          const double x0 = slab[i + q * lds], x1 = slab[i + (q + G) * lds];
          slab[i + q * lds] = fma(-l, u[q], x0);
          slab[i + (q + G) * lds] = fma(-l, u[q + G], x1);
        }
        if (q < w) slab[i + q * lds] = fma(-l, u[q], slab[i + q * lds]);
      }
    }
  }
  __syncthreads();
  if (RM) {
    for (int e = tid; e < rows * w; e += LEAF_THREADS) {
      const int i = e / w, col = e - i * w;
      a.P[(long)(r0 + i) * a.ld + col] = slab[i + col * lds];
    }
  } else {
    for (int col = 0; col < w; ++col)
      for (int i = tid; i < rows; i += LEAF_THREADS) a.P[(long)(r0 + i) + (long)col * a.ld] = slab[i + col * lds];
  }
  if (c == 0 && tid == 0 && first_null >= 0) atomicMin(a.info, a.gcol + first_null);
}

// Register-resident leaf for a panel stored transposed (element (i, col) at
// P[i * ld + col]), w == W columns: thread t of each CTA owns the slab rows
// i = t + k * 512 (k < RPT) and keeps their W entries in registers, so the
// rank-1 updates never touch memory.  Per column: warp shuffles and warp 0
// find the CTA's candidate (two CTA barriers); the warp holding the
// candidate row gathers it by shuffles and pushes it, with the magnitude
// and row index, into every CTA's shared memory, and the warp holding row j
// does the same with row j; one cluster barrier; warp 0 picks the winner
// (one CTA barrier); then each thread exchanges, scales and updates its own
// rows and forms its candidate for the next column.  Same pivot order, tie
// rule, null-column and NaN handling as lu_leaf_cluster_kernel.
constexpr int RLEAF_THREADS = 512;

__host__ __device__ inline size_t rleaf_smem_bytes(int w, int C) {
  return sizeof(double) * (2 * (size_t)C * w + 2 * C + 2 * w) + sizeof(int) * 2 * C + 64;
}

template <int W, int RPT>
__device__ __forceinline__ double rleaf_pick(const double (&rv)[RPT][W], int k, int q) {
  double v = rv[0][q];
#pragma unroll
  for (int kk = 1; kk < RPT; ++kk)
    if (kk == k) v = rv[kk][q];
  return v;
}

// Lane `src` of the calling warp holds the row (slot k; have = false pushes
// zeros); every lane gets it by shuffles and lane d < C stores it into CTA
// d's buffer at local offset `dst` with st.async, completing bytes on CTA
// d's mbarrier `bar` (both shared::cta addresses of this CTA, mapped).
template <int W, int RPT>
__device__ __forceinline__ void rleaf_push_row(const double (&rv)[RPT][W], int k, int src, bool have, uint32_t dst,
                                               uint32_t bar, int C) {
  const int lane = threadIdx.x & 31;
  const uint32_t rank = (uint32_t)(lane < C ? lane : 0);
  const uint32_t rdst = mapa_shared(dst, rank), rbar = mapa_shared(bar, rank);
#pragma unroll
  for (int q0 = 0; q0 < W; q0 += 4) {
    double row[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) row[q] = __shfl_sync(0xffffffffu, rleaf_pick<W, RPT>(rv, k, q0 + q), src);
    if (lane < C)
#pragma unroll
      for (int q = 0; q < 4; ++q) st_async_f64(rdst + 8 * (q0 + q), have ? row[q] : 0.0, rbar);
  }
}

// Entry j (run-time) of a register row: a select chain over compile-time
// indices, so the row stays in registers.
template <int W>
__device__ __forceinline__ double rleaf_pick_col(const double (&row)[W], int j) {
  double v = row[0];
#pragma unroll
  for (int q = 1; q < W; ++q)
    if (q == j) v = row[q];
  return v;
}

// Column J of the leaf for the calling thread's rows, J a compile-time
// constant so every register of a row is addressed directly: exchange
// rows j and r, scale column J below the pivot (reciprocal multiply, as
// bl1_dinvscalv), rank-1 update, and the candidate for column J + 1.
template <int W, int RPT, int J>
__device__ __forceinline__ void rleaf_column(double (&rv)[RPT][W], int tid, int r0, int rows, int r,
                                             const double* u, const double* oldj, double rinv, double& bv,
                                             int& bi) {
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int i = tid + k * RLEAF_THREADS, gi = r0 + i;
    if (i >= rows || gi < J) continue;
    if (gi == J) {
      if (r != J)
#pragma unroll
        for (int q = 0; q < W; ++q) rv[k][q] = u[q];
      continue;
    }
    if (gi == r)
#pragma unroll
      for (int q = 0; q < W; ++q) rv[k][q] = oldj[q];
    const double l = rv[k][J] * rinv;
    rv[k][J] = l;
#pragma unroll
    for (int q = J + 1; q < W; ++q) rv[k][q] = fma(-l, u[q], rv[k][q]);
    if constexpr (J + 1 < W) {
      const double t = fabs(rv[k][J + 1]);
      if (t > bv) { bv = t; bi = gi; }
    }
  }
}

template <int W, int RPT, int J = 0>
__device__ __forceinline__ void rleaf_column_at(int j, double (&rv)[RPT][W], int tid, int r0, int rows, int r,
                                                const double* u, const double* oldj, double rinv, double& bv,
                                                int& bi) {
  if constexpr (J < W) {
    if (j == J) {
      rleaf_column<W, RPT, J>(rv, tid, r0, rows, r, u, oldj, rinv, bv, bi);
      return;
    }
    rleaf_column_at<W, RPT, J + 1>(j, rv, tid, r0, rows, r, u, oldj, rinv, bv, bi);
  }
}

template <int W, int RPT>
__global__ void __launch_bounds__(RLEAF_THREADS, 1) lu_leaf_reg_kernel(LeafArgs a) {
  extern __shared__ double S[];
  constexpr int NW = RLEAF_THREADS / 32;
  __shared__ double s_rv[2][NW];
  __shared__ int s_ri[2][NW];
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int c = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* xrow = S;                                  // [2][C][W] candidate rows
  double* xval = xrow + 2 * (size_t)C * W;           // [2][C] candidate magnitudes
  double* rowj = xval + 2 * C;                       // [2][W] row j
  int* xidx = reinterpret_cast<int*>(rowj + 2 * W);  // [2][C] candidate rows (INT_MAX: none)
  const int r0 = c * a.R;
  const int rows = max(0, min(a.R, a.M - r0));
  // full[p]: the exchange buffers of parity p are complete (armed by thread
  // 0 with the bytes expected per column, completed by the st.async pushes)
  __shared__ __align__(8) unsigned long long s_full[2];
  const uint32_t full0 = smem_u32(&s_full[0]);
  const uint32_t xrow_s = smem_u32(xrow), xval_s = smem_u32(xval), rowj_s = smem_u32(rowj), xidx_s = smem_u32(xidx);
  const uint32_t col_bytes = (uint32_t)(C * (8 * W + 8 + 4) + 8 * W);
  if (tid == 0) {
    mbar_init(full0, 1);
    mbar_init(full0 + 8, 1);
    fence_barrier_init();
  }
  cluster.sync();  // every CTA's barriers exist before the first push

  double rv[RPT][W];
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int i = tid + k * RLEAF_THREADS;
#pragma unroll
    for (int q = 0; q < W; ++q) rv[k][q] = (i < rows) ? a.P[(long)(r0 + i) * a.ld + q] : 0.0;
  }
  int first_null = -1;
  double bv = -1.0;
  int bi = INT_MAX;
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int i = tid + k * RLEAF_THREADS;
    if (i < rows) {
      const double v = fabs(rv[k][0]);
      if (v > bv) { bv = v; bi = r0 + i; }  // rows ascend with k
    }
  }
  // The column loop is not unrolled (the unrolled body would overflow the
  // instruction cache); the per-column update is dispatched to a
  // compile-time column.  Per column one CTA barrier (the warps' candidates)
  // and one cluster barrier (the pushed rows); every warp reduces the
  // warps' candidates and the CTAs' candidates itself.
#pragma unroll 1
  for (int j = 0; j < W; ++j) {
    const int par = j & 1;
    // ---- 1. CTA candidate
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double ov = __shfl_xor_sync(0xffffffffu, bv, off);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
      if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
    }
    if (lane == 0) { s_rv[par][warp] = bv; s_ri[par][warp] = bi; }
    __syncthreads();
    {
      double v = lane < NW ? s_rv[par][lane] : -1.0;
      int i0 = lane < NW ? s_ri[par][lane] : INT_MAX;
      // all 32 lanes take part (lanes >= NW hold the neutral element), so
      // every lane of every warp ends with the same candidate
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i0, off);
        if (ov > v || (ov == v && oi < i0)) { v = ov; i0 = oi; }
      }
      bv = v;
      bi = i0;
    }
    // ---- 2. push the candidate row (zeros when this CTA has none), its
    // magnitude and row, and row j (by its owner) into every CTA with
    // st.async; each CTA waits for the column's bytes on its own mbarrier
    const uint32_t fullp = full0 + 8 * par;
    {
      const bool have = bi != INT_MAX && bi - r0 >= 0 && bi - r0 < rows;
      const int li = have ? bi - r0 : 0, ot = li & (RLEAF_THREADS - 1);
      if (warp == (ot >> 5))
        rleaf_push_row<W, RPT>(rv, li / RLEAF_THREADS, ot & 31, have,
                               xrow_s + 8u * (uint32_t)((par * C + c) * W), fullp, C);
    }
    if (warp == NW - 1 && lane < C) {
      const uint32_t rbar = mapa_shared(fullp, (uint32_t)lane);
      st_async_f64(mapa_shared(xval_s + 8u * (uint32_t)(par * C + c), (uint32_t)lane), bv, rbar);
      st_async_b32(mapa_shared(xidx_s + 4u * (uint32_t)(par * C + c), (uint32_t)lane), (uint32_t)bi, rbar);
    }
    if (j >= r0 && j < r0 + rows) {
      const int lj = j - r0, jt = lj & (RLEAF_THREADS - 1);
      if (warp == (jt >> 5))
        rleaf_push_row<W, RPT>(rv, lj / RLEAF_THREADS, jt & 31, true, rowj_s + 8u * (uint32_t)(par * W), fullp, C);
    }
    if (tid == 0) mbar_arrive_expect_tx(fullp, col_bytes);
    // every thread waits with cluster-scope acquire; the CTA leaves the loop
    // together if the (bounded) wait ran out
    const bool got = mbar_wait_cluster(fullp, (uint32_t)((j >> 1) & 1), a.err, 21);
    if (!__syncthreads_and(got ? 1 : 0)) break;
    // ---- 3. winner (identical in every warp of every CTA: same data, same
    // order)
    int r, w0;
    {
      double v = -2.0;
      int i0 = INT_MAX, q0 = 0;
      for (int q = lane; q < C; q += 32) {
        const double cv = xval[par * C + q];
        const int ci = xidx[par * C + q];
        if (ci != INT_MAX && (cv > v || (cv == v && ci < i0))) { v = cv; i0 = ci; q0 = q; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i0, off);
        const int oq = __shfl_xor_sync(0xffffffffu, q0, off);
        if (ov > v || (ov == v && oi < i0)) { v = ov; i0 = oi; q0 = oq; }
      }
      r = i0;
      w0 = q0;
    }
    const double* u = xrow + ((size_t)par * C + w0) * W;  // the pivot row
    if (r == INT_MAX) {
      // no orderable candidate (every magnitude NaN): keep row j, as idamax
      // does when no later entry compares greater than the first
      r = j;
      u = rowj + par * W;
    }
    const double* oldj = rowj + par * W;
    const double piv = u[j];
    if (c == 0 && tid == 0) a.piv[j] = r - j;
    bv = -1.0;
    bi = INT_MAX;
    if (piv == 0.0) {
      // null column: no exchange, no scaling, no update
      if (first_null < 0) first_null = j;
      if (j + 1 < W)
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          const int i = tid + k * RLEAF_THREADS, gi = r0 + i;
          if (i < rows && gi > j) {
            const double t = fabs(rleaf_pick_col<W>(rv[k], j + 1));
            if (t > bv) { bv = t; bi = gi; }
          }
        }
      continue;
    }
    // ---- 4. exchange, scale, update, next candidate
    rleaf_column_at<W, RPT>(j, rv, tid, r0, rows, r, u, oldj, 1.0 / piv, bv, bi);
  }
  // no CTA leaves while another may still push into its shared memory
  cluster.sync();
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int i = tid + k * RLEAF_THREADS;
    if (i < rows)
#pragma unroll
      for (int q = 0; q < W; ++q) a.P[(long)(r0 + i) * a.ld + q] = rv[k][q];
  }
  if (c == 0 && tid == 0 && first_null >= 0) atomicMin(a.info, a.gcol + first_null);
}

struct LeafConfig {
  bool ready = false;
  int max_cluster = 8;
  int max_cluster_reg = 8;  // register-resident leaf
  size_t smem_cap = 0;  // usable dynamic SMEM per CTA
};
LeafConfig g_leaf;

int leaf_setup() {
  if (g_leaf.ready) return FLA_SUCCESS;
  Context& cx = ctx();
  g_leaf.smem_cap = std::min<size_t>(cx.smem_optin, 227 * 1024) - 1024;
  for (auto kern : {lu_leaf_cluster_kernel<false>, lu_leaf_cluster_kernel<true>}) {
    FB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)g_leaf.smem_cap));
    FB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  }
  // Largest cluster (16, else 8, 4 ...) that can be resident with a full
  // shared-memory slab per CTA.
  g_leaf.max_cluster = 1;
  for (int cs = LEAF_MAXC; cs >= 2; cs >>= 1) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(LEAF_THREADS);
    cfg.dynamicSmemBytes = g_leaf.smem_cap;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, lu_leaf_cluster_kernel<false>, &cfg) == cudaSuccess &&
        nclusters > 0) {
      g_leaf.max_cluster = cs;
      break;
    }
    cudaGetLastError();
  }
  // the register-resident leaf: 512 threads, a few KB of SMEM
  for (auto kern : {lu_leaf_reg_kernel<8, 4>, lu_leaf_reg_kernel<16, 2>, lu_leaf_reg_kernel<32, 1>})
    FB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  g_leaf.max_cluster_reg = 1;
  for (int cs = LEAF_MAXC; cs >= 2; cs >>= 1) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(RLEAF_THREADS);
    cfg.dynamicSmemBytes = rleaf_smem_bytes(32, cs);
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    bool ok = true;
    for (auto kern : {lu_leaf_reg_kernel<8, 4>, lu_leaf_reg_kernel<16, 2>, lu_leaf_reg_kernel<32, 1>}) {
      nclusters = 0;
      if (cudaOccupancyMaxActiveClusters(&nclusters, kern, &cfg) != cudaSuccess || nclusters <= 0) ok = false;
      cudaGetLastError();
    }
    if (ok) {
      g_leaf.max_cluster_reg = cs;
      break;
    }
  }
  g_leaf.ready = true;
  return FLA_SUCCESS;
}

// Cluster geometry of the register-resident leaf for an M x w panel:
// w must be 8, 16 or 32 and the rows must fit 512 x RPT per CTA.
bool rleaf_geometry(long M, int w, int* C, int* R) {
  if (w != 8 && w != 16 && w != 32) return false;
  const long cap = (long)RLEAF_THREADS * (w == 8 ? 4 : w == 16 ? 2 : 1);
  int cs = 1;
  while (cs < g_leaf.max_cluster_reg && (M + cs - 1) / cs > cap) cs <<= 1;
  if ((M + cs - 1) / cs > cap) return false;
  *C = cs;
  *R = (int)((M + cs - 1) / cs);
  return true;
}

int rleaf_launch(double* P, long ld, long M, int w, int* d_piv, int gcol, cudaStream_t st) {
  int C = 0, R = 0;
  if (!rleaf_geometry(M, w, &C, &R)) {
    set_last_error("LU panel leaf does not fit in a cluster");
    return FLA_FAILURE;
  }
  LeafArgs la;
  la.P = P;
  la.ld = ld;
  la.M = (int)M;
  la.w = w;
  la.R = R;
  la.lds = 0;
  la.gcol = gcol;
  la.piv = d_piv;
  la.info = ctx().d_status + ST_INFO;
  la.err = ctx().d_status + ST_ERROR;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(RLEAF_THREADS);
  cfg.dynamicSmemBytes = rleaf_smem_bytes(w, C);
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const int ps = prof_begin(st);
  if (w == 8) FB_CK(cudaLaunchKernelEx(&cfg, lu_leaf_reg_kernel<8, 4>, la));
  else if (w == 16) FB_CK(cudaLaunchKernelEx(&cfg, lu_leaf_reg_kernel<16, 2>, la));
  else FB_CK(cudaLaunchKernelEx(&cfg, lu_leaf_reg_kernel<32, 1>, la));
  prof_end(ps, st, PROF_PANEL, 0.0);
  count_launch();
  return FLA_SUCCESS;
}

// Cluster size and slab geometry for an M x w leaf; false if it does not fit.
// Widest leaf: the leaf's rank-1 updates re-read the whole slab every
// column, so wide leaves are split and their halves joined by DMMA GEMMs;
// FLA_B200_LU_LEAF_MAXW (8..128) overrides the default for tuning.
int leaf_maxw() {
  static int mw = 0;
  if (mw == 0) {
    mw = 32;
    if (const char* e = std::getenv("FLA_B200_LU_LEAF_MAXW")) {
      const int v = std::atoi(e);
      if (v >= 8 && v <= LEAF_MAXW) mw = v;
    }
  }
  return mw;
}

bool leaf_geometry(long M, int w, int* C, int* R, int* lds, size_t* smem) {
  if (w > leaf_maxw()) return false;
  // about LEAF_ROWS_TARGET rows per CTA when M is small, the largest cluster
  // otherwise
  int cs = 1;
  while (cs < g_leaf.max_cluster && (M + cs - 1) / cs > LEAF_ROWS_TARGET) cs <<= 1;
  for (; cs <= g_leaf.max_cluster; cs <<= 1) {
    const long r = (M + cs - 1) / cs;
    const int l = (int)(r | 1);
    const size_t need = leaf_smem_bytes(l, w, cs);
    if (need <= g_leaf.smem_cap) {
      *C = cs;
      *R = (int)r;
      *lds = l;
      *smem = need;
      return true;
    }
  }
  return false;
}

int leaf_launch(double* P, long ld, long M, int w, int* d_piv, int gcol, bool rm, cudaStream_t st) {
  int C = 0, R = 0, lds = 0;
  size_t smem = 0;
  if (!leaf_geometry(M, w, &C, &R, &lds, &smem)) {
    set_last_error("LU panel leaf does not fit in a cluster");
    return FLA_FAILURE;
  }
  LeafArgs la;
  la.P = P;
  la.ld = ld;
  la.M = (int)M;
  la.w = w;
  la.R = R;
  la.lds = lds;
  la.gcol = gcol;
  la.piv = d_piv;
  la.info = ctx().d_status + ST_INFO;
  la.err = ctx().d_status + ST_ERROR;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(LEAF_THREADS);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const int ps = prof_begin(st);
  if (rm)
    FB_CK(cudaLaunchKernelEx(&cfg, lu_leaf_cluster_kernel<true>, la));
  else
    FB_CK(cudaLaunchKernelEx(&cfg, lu_leaf_cluster_kernel<false>, la));
  prof_end(ps, st, PROF_PANEL, 0.0);
  count_launch();
  return FLA_SUCCESS;
}

}  // namespace

// Factor the M x w panel at P (ld) with partial pivoting; d_piv receives w
// relative pivots; gcol is the global index of the panel's first column.
int lu_panel_factor(double* P, long ld, long M, int w, int* d_piv, int gcol, cudaStream_t st) {
  if (leaf_setup() != FLA_SUCCESS) return FLA_FAILURE;
  if (w <= 0 || M <= 0) return FLA_SUCCESS;
  int C, R, lds;
  size_t smem;
  if (leaf_geometry(M, w, &C, &R, &lds, &smem) || w <= 2) return leaf_launch(P, ld, M, w, d_piv, gcol, false, st);
  // split: left half a multiple of 2 columns (keeps 16-byte alignment)
  const int w1 = std::max(2, (w / 2) & ~1);
  const int w2 = w - w1;
  if (lu_panel_factor(P, ld, M, w1, d_piv, gcol, st) != FLA_SUCCESS) return FLA_FAILURE;
  double* P12 = P + (long)w1 * ld;
  if (laswp_dev(P, ld, 0, d_piv, w1, w1, w2, 0, 0, false, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (trsm_block(P, ld, P12, ld, w1, w2, true, false, true, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (M > w1) {
    if (gemm_f64(st, false, false, M - w1, w2, w1, -1.0, P + w1, ld, P12, ld, 1.0, P12 + w1, ld) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (lu_panel_factor(P12 + w1, ld, M - w1, w2, d_piv + w1, gcol + w1, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (laswp_dev(P, ld, w1, d_piv + w1, (int)std::min<long>(w2, M - w1), 0, w1, 0, 0, false, st) != FLA_SUCCESS)
      return FLA_FAILURE;
  }
  return FLA_SUCCESS;
}


// The same recursion on a panel stored transposed (element (i, j) of the
// panel at P[i * ld + j]): row interchanges move contiguous pieces of
// columns of A^T, the top-right solve is a row-wise solve with L11 (held as
// the upper triangle L11^T), and the update is A22^T -= U12^T A21^T.
int lu_panel_factor_t(double* P, long ld, long M, int w, int* d_piv, int gcol, cudaStream_t st) {
  if (leaf_setup() != FLA_SUCCESS) return FLA_FAILURE;
  if (w <= 0 || M <= 0) return FLA_SUCCESS;
  int C, R, lds;
  size_t smem;
  if (rleaf_geometry(M, w, &C, &R)) return rleaf_launch(P, ld, M, w, d_piv, gcol, st);
  if (leaf_geometry(M, w, &C, &R, &lds, &smem) || w <= 2) return leaf_launch(P, ld, M, w, d_piv, gcol, true, st);
  const int w1 = std::max(2, (w / 2) & ~1);
  const int w2 = w - w1;
  if (lu_panel_factor_t(P, ld, M, w1, d_piv, gcol, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (laswp_t_dev(P, ld, 0, d_piv, w1, w1, w2, 0, 0, st) != FLA_SUCCESS) return FLA_FAILURE;
  // U12^T (w2 x w1 at P + w1): each row y solves L11 y = x
  if (trsm_right_block(P, ld, P + w1, ld, w2, w1, false, true, true, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (M > w1) {
    if (gemm_f64(st, false, false, w2, M - w1, w1, -1.0, P + w1, ld, P + (long)w1 * ld, ld, 1.0,
                 P + w1 + (long)w1 * ld, ld) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (lu_panel_factor_t(P + w1 + (long)w1 * ld, ld, M - w1, w2, d_piv + w1, gcol + w1, st) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (laswp_t_dev(P, ld, w1, d_piv + w1, (int)std::min<long>(w2, M - w1), 0, w1, 0, 0, st) != FLA_SUCCESS)
      return FLA_FAILURE;
  }
  return FLA_SUCCESS;
}

}  // namespace fb
