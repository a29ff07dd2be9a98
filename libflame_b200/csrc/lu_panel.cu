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
  int pl, pr;  // register-resident leaf: columns of the enclosing panel left
               // of the leaf and right of it, which receive the leaf's row
               // interchanges at its end (0, 0: none)
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
// rank-1 updates never touch memory.  Per column:
//  1. each warp finds its candidate (largest magnitude, smallest row among
//     equals) with three redux.sync reductions over a 64-bit ordering key,
//     and the lane holding it writes the key and row index (16 bytes) into
//     the warp's header in shared memory; the owner of row j writes row j;
//  2. one CTA barrier; every warp reduces the 16 headers the same way, and
//     the one thread holding the CTA's candidate writes its row into the
//     CTA's exchange slot (sixteen warps each storing a whole row cost a
//     quarter of the column time);
//  3. (clusters only) once that thread has arrived on a local mbarrier, warp
//     0 bulk-copies the slot, and row j if this CTA owns it, into every
//     other CTA's shared memory, each copy completing bytes on the
//     receiver's mbarrier, and waits for the column's bytes; a second CTA
//     barrier releases the other warps, and every warp reduces the C slot
//     headers to the winner;
//  4. each thread exchanges, scales and updates its own rows and forms its
//     candidate for the next column.
// Same pivot order, tie rule, null-column and NaN handling as
// lu_leaf_cluster_kernel.  Exchange slots alternate between two halves by
// column parity: a CTA cannot receive column j + 2's copies before every
// CTA has finished reading column j's (it must first have passed column
// j + 1's exchange, which needs this CTA's column j + 1 copies, issued
// after its column j work).
constexpr int RLEAF_THREADS = 512;
constexpr int RLEAF_NW = RLEAF_THREADS / 32;

// One exchange slot: 16-byte header and the W entries of the row.
template <int W>
struct RSlot {
  unsigned long long key;  // ordering key: 0 no candidate, else bits(|x|) + 1
  int row;                 // global row of the candidate (INT_MAX: none)
  int pad;
  double v[W];
};

// A warp's candidate: ordering key and row.
struct RHdr {
  unsigned long long key;
  int row;
  int pad;
};

// Layout: hdr [2][16] (the warps' candidates), cslot [2][C] (the CTAs'
// candidates with their rows), rowj [2][W], four mbarriers (peers' copies
// and this CTA's slot written, by parity), then one 32 x (W + 1) staging
// tile per warp for the coalesced load and store of the slab.
__host__ __device__ inline size_t rleaf_tile_offset(int w, int C) {
  const size_t slot = 16 + 8 * (size_t)w;
  return 2 * RLEAF_NW * sizeof(RHdr) + 2 * (size_t)C * slot + 16 * (size_t)w + 32;
}
__host__ __device__ inline size_t rleaf_smem_bytes(int w, int C) {
  return rleaf_tile_offset(w, C) + sizeof(double) * RLEAF_NW * 32 * ((size_t)w + 1) + 128;
}

// Non-negative magnitudes order like their bit patterns, so the key orders
// candidates by magnitude; no candidate orders below every magnitude (and
// NaN never becomes a candidate: `t > best` is false for it).
__device__ __forceinline__ unsigned long long rleaf_key(double bv, int bi) {
  return bi == INT_MAX ? 0ull : (unsigned long long)__double_as_longlong(bv) + 1ull;
}

// Warp argmax of (key, row): the largest key, the smallest row among equal
// keys; every lane receives the result.  Rows are distinct, INT_MAX marks
// no candidate (key 0).
__device__ __forceinline__ void rleaf_argmax_warp(unsigned long long& key, int& row) {
  const unsigned hi = (unsigned)(key >> 32), lo = (unsigned)key;
  const unsigned mhi = __reduce_max_sync(0xffffffffu, hi);
  const unsigned mlo = __reduce_max_sync(0xffffffffu, hi == mhi ? lo : 0u);
  const bool top = hi == mhi && lo == mlo;
  row = (int)__reduce_min_sync(0xffffffffu, top ? (unsigned)row : 0xffffffffu);
  key = ((unsigned long long)mhi << 32) | mlo;
}

template <int W, int RPT>
__device__ __forceinline__ double rleaf_pick(const double (&rv)[RPT][W], int k, int q) {
  double v = rv[0][q];
#pragma unroll
  for (int kk = 1; kk < RPT; ++kk)
    if (kk == k) v = rv[kk][q];
  return v;
}

// Row slot k of the calling thread into shared memory (16-byte aligned).
template <int W, int RPT>
__device__ __forceinline__ void rleaf_store_row(const double (&rv)[RPT][W], int k, double* dst) {
#pragma unroll
  for (int q = 0; q < W; q += 2)
    *reinterpret_cast<double2*>(dst + q) = make_double2(rleaf_pick<W, RPT>(rv, k, q), rleaf_pick<W, RPT>(rv, k, q + 1));
}

// The warp's 32 rows of slot k (slab rows base .. base + 31) pass through
// its 32 x (W + 1) shared tile, so every global access of the warp reads or
// writes whole rows (W contiguous doubles) instead of one entry of 32 rows.
template <int W, int RPT>
__device__ __forceinline__ void rleaf_load(double (&rv)[RPT][W], const LeafArgs& a, int r0, int rows,
                                           double* tile, int warp, int lane) {
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int base = warp * 32 + k * RLEAF_THREADS;
#pragma unroll 8
    for (int e = lane; e < 32 * W; e += 32) {
      const int rr = e / W, q = e % W;
      tile[rr * (W + 1) + q] = (base + rr < rows) ? a.P[(long)(r0 + base + rr) * a.ld + q] : 0.0;
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < W; ++q) rv[k][q] = tile[lane * (W + 1) + q];
    __syncwarp();
  }
}

template <int W, int RPT>
__device__ __forceinline__ void rleaf_store(const double (&rv)[RPT][W], const LeafArgs& a, int r0, int rows,
                                            double* tile, int warp, int lane) {
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int base = warp * 32 + k * RLEAF_THREADS;
#pragma unroll
    for (int q = 0; q < W; ++q) tile[lane * (W + 1) + q] = rv[k][q];
    __syncwarp();
#pragma unroll 8
    for (int e = lane; e < 32 * W; e += 32) {
      const int rr = e / W, q = e % W;
      if (base + rr < rows) a.P[(long)(r0 + base + rr) * a.ld + q] = tile[rr * (W + 1) + q];
    }
    __syncwarp();
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
                                             int& bi, int& bk) {
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
      if (t > bv) { bv = t; bi = gi; bk = k; }
    }
  }
}

// Run-time column j to its compile-time body through one jump table.
template <int W, int RPT>
__device__ __forceinline__ void rleaf_column_at(int j, double (&rv)[RPT][W], int tid, int r0, int rows, int r,
                                                const double* u, const double* oldj, double rinv, double& bv,
                                                int& bi, int& bk) {
  static_assert(W <= 32, "leaf width");
  switch (j) {
#define FB_RLEAF_CASE(J)                                                              \
  case J:                                                                             \
    if constexpr (J < W) rleaf_column<W, RPT, J>(rv, tid, r0, rows, r, u, oldj, rinv, bv, bi, bk); \
    break;
    FB_RLEAF_CASE(0) FB_RLEAF_CASE(1) FB_RLEAF_CASE(2) FB_RLEAF_CASE(3) FB_RLEAF_CASE(4) FB_RLEAF_CASE(5)
    FB_RLEAF_CASE(6) FB_RLEAF_CASE(7) FB_RLEAF_CASE(8) FB_RLEAF_CASE(9) FB_RLEAF_CASE(10) FB_RLEAF_CASE(11)
    FB_RLEAF_CASE(12) FB_RLEAF_CASE(13) FB_RLEAF_CASE(14) FB_RLEAF_CASE(15) FB_RLEAF_CASE(16)
    FB_RLEAF_CASE(17) FB_RLEAF_CASE(18) FB_RLEAF_CASE(19) FB_RLEAF_CASE(20) FB_RLEAF_CASE(21)
    FB_RLEAF_CASE(22) FB_RLEAF_CASE(23) FB_RLEAF_CASE(24) FB_RLEAF_CASE(25) FB_RLEAF_CASE(26)
    FB_RLEAF_CASE(27) FB_RLEAF_CASE(28) FB_RLEAF_CASE(29) FB_RLEAF_CASE(30) FB_RLEAF_CASE(31)
#undef FB_RLEAF_CASE
    default:
      break;
  }
}

// The leaf's row interchanges (row j <-> row s_r[j], j = 0..W-1, in order)
// applied to the other columns of the enclosing panel: pl columns left of
// the leaf and pr right of it (FLA_Apply_pivots on A10/A12 of the panel
// recursion, done here instead of by separate launches).  The interchanges
// move at most 2W rows: the W leaf rows and the distinct far targets.  Their
// composition (the row that ends in each slot) is formed once; each CTA of
// the cluster then gathers its share of the columns for those rows into
// shared memory and writes them back permuted.  The leaf's own columns are
// not touched, so no CTA waits for another.
template <int W>
__device__ void rleaf_apply_pivots(const LeafArgs& a, const int* s_r, int c, int C, double* buf) {
  __shared__ int s_tgt[W];       // slot receiving row j's interchange partner
  __shared__ int s_row[2 * W];   // leaf-relative row of each slot (-1: unused)
  __shared__ int s_src[2 * W];   // slot whose original row ends in this slot
  const int tid = threadIdx.x;
  __syncthreads();  // s_r complete
  for (int q = tid; q < 2 * W; q += blockDim.x) s_row[q] = q < W ? q : -1;
  __syncthreads();
  if (tid < W) {
    const int t = s_r[tid];
    int slot = t;
    if (t >= W) {  // far target: the first interchange with it owns the slot
      int first = tid;
      for (int i2 = tid - 1; i2 >= 0; --i2) first = s_r[i2] == t ? i2 : first;
      slot = W + first;
      if (first == tid) s_row[slot] = t;
    }
    s_tgt[tid] = slot;
  }
  __syncthreads();
  if (tid == 0) {
    for (int q = 0; q < 2 * W; ++q) s_src[q] = q;
    for (int i = 0; i < W; ++i) {
      const int b = s_tgt[i];
      const int x = s_src[i];
      s_src[i] = s_src[b];
      s_src[b] = x;
    }
  }
  __syncthreads();
  const int tot = a.pl + a.pr;
  const int per = (tot + C - 1) / C;
  const int cb = c * per, ce = min(tot, cb + per);
  const int cap = (RLEAF_NW * 32 * (W + 1)) / (2 * W);  // columns per pass
  for (int c0 = cb; c0 < ce; c0 += cap) {
    const int n = min(cap, ce - c0);
    for (int e = tid; e < 2 * W * n; e += blockDim.x) {
      const int q = e / n, t = e - q * n;
      const int col = (c0 + t) < a.pl ? (c0 + t) - a.pl : W + (c0 + t - a.pl);
      if (s_row[q] >= 0) buf[e] = a.P[col + (long)s_row[q] * a.ld];
    }
    __syncthreads();
    for (int e = tid; e < 2 * W * n; e += blockDim.x) {
      const int q = e / n, t = e - q * n;
      const int col = (c0 + t) < a.pl ? (c0 + t) - a.pl : W + (c0 + t - a.pl);
      if (s_row[q] >= 0 && s_src[q] != q) a.P[col + (long)s_row[q] * a.ld] = buf[s_src[q] * n + t];
    }
    __syncthreads();
  }
}

template <int W, int RPT>
__global__ void __launch_bounds__(RLEAF_THREADS, 1) lu_leaf_reg_kernel(LeafArgs a) {
  using Slot = RSlot<W>;
  extern __shared__ __align__(128) unsigned char rleaf_smem[];
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int c = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  RHdr* hdr = reinterpret_cast<RHdr*>(rleaf_smem);                                 // [2][16]
  Slot* cslot = reinterpret_cast<Slot*>(rleaf_smem + 2 * RLEAF_NW * sizeof(RHdr));   // [2][C]
  double* rowj = reinterpret_cast<double*>(cslot + 2 * C);                         // [2][W]
  const uint32_t full0 = smem_u32(rowj + 2 * W);                                   // 2 mbarriers: peers' copies
  const uint32_t ready0 = full0 + 16;                                              // 2: own slot written
  const int r0 = c * a.R;
  const int rows = max(0, min(a.R, a.M - r0));
  if (C > 1) {
    if (tid == 0) {
      mbar_init(full0, 1);
      mbar_init(full0 + 8, 1);
      mbar_init(ready0, 1);
      mbar_init(ready0 + 8, 1);
      fence_barrier_init();
    }
    cluster.sync();  // every CTA's barriers exist before the first copy
  }

  double* tile = reinterpret_cast<double*>(rleaf_smem + rleaf_tile_offset(W, C)) + warp * 32 * (W + 1);
  __shared__ int s_r[W];  // pivot row of every column (leaf-relative)
  bool done = true;       // uniform in the CTA: false if a wait ran out
  double rv[RPT][W];
  rleaf_load<W, RPT>(rv, a, r0, rows, tile, warp, lane);
  int first_null = -1;
  double bv = -1.0;
  int bi = INT_MAX, bk = 0;
#pragma unroll
  for (int k = 0; k < RPT; ++k) {
    const int i = tid + k * RLEAF_THREADS;
    if (i < rows) {
      const double v = fabs(rv[k][0]);
      if (v > bv) { bv = v; bi = r0 + i; bk = k; }  // rows ascend with k
    }
  }
  // The column loop is not unrolled (the unrolled body would overflow the
  // instruction cache); the per-column update is dispatched to a
  // compile-time column.
#pragma unroll 1
  for (int j = 0; j < W; ++j) {
    const int par = j & 1;
    const bool own_j = j >= r0 && j < r0 + rows;  // uniform in the CTA
    // ---- 1. the warp's candidate header; row j by its owner
    {
      unsigned long long wk = rleaf_key(bv, bi);
      int wi = bi;
      rleaf_argmax_warp(wk, wi);
      if (wi == INT_MAX ? lane == 0 : wi == bi) {
        RHdr h;
        h.key = wk;
        h.row = wi;
        h.pad = 0;
        hdr[par * RLEAF_NW + warp] = h;
      }
      if (own_j && tid == ((j - r0) & (RLEAF_THREADS - 1))) {
        rleaf_store_row<W, RPT>(rv, (j - r0) / RLEAF_THREADS, rowj + par * W);
        if (C > 1) fence_proxy_async_smem();
      }
    }
    __syncthreads();
    // ---- 2. the CTA's candidate (every warp, same data, same result); its
    // holder writes it, with its row, into the CTA's slot
    Slot* mine = cslot + par * C + c;
    const Slot* best = mine;
    int r;
    {
      const RHdr* hs = hdr + par * RLEAF_NW + (lane < RLEAF_NW ? lane : 0);
      unsigned long long ck = lane < RLEAF_NW ? hs->key : 0ull;
      int ci = lane < RLEAF_NW ? hs->row : INT_MAX;
      rleaf_argmax_warp(ck, ci);
      if (ci == INT_MAX ? tid == 0 : ci == bi) {
        mine->key = ck;
        mine->row = ci;
        if (ci != INT_MAX) rleaf_store_row<W, RPT>(rv, bk, mine->v);
        if (C > 1) {
          fence_proxy_async_smem();
          mbar_arrive(ready0 + 8 * par);
        }
      }
      r = ci;
    }
    // ---- 3. exchange with the other CTAs of the cluster
    if (C > 1) {
      const uint32_t fullp = full0 + 8 * par;
      const uint32_t ph = (uint32_t)((j >> 1) & 1);
      bool ok = true;
      if (warp == 0) {
        ok = mbar_wait(ready0 + 8 * par, ph, a.err, 22);  // the slot is written
        if (ok) {
          if (lane < C && lane != c) {
            const uint32_t rbar = mapa_shared(fullp, (uint32_t)lane);
            bulk_copy_to_peer(mapa_shared(smem_u32(mine), (uint32_t)lane), smem_u32(mine), (uint32_t)sizeof(Slot),
                              rbar);
            if (own_j)
              bulk_copy_to_peer(mapa_shared(smem_u32(rowj + par * W), (uint32_t)lane), smem_u32(rowj + par * W),
                                (uint32_t)(8 * W), rbar);
          }
          if (lane == 0) mbar_arrive_expect_tx(fullp, (uint32_t)((C - 1) * sizeof(Slot) + (own_j ? 0 : 8 * W)));
          ok = mbar_wait_cluster(fullp, ph, a.err, 21);
        }
      }
      // the CTA leaves the loop together if a (bounded) wait ran out
      if (__syncthreads_or(ok ? 0 : 1)) {
        done = false;
        break;
      }
      if (warp != 0) (void)mbar_try_wait_cluster(fullp, ph);  // acquire of the completed phase
      const Slot* hs = cslot + par * C + (lane < C ? lane : c);
      unsigned long long gk = lane < C ? hs->key : 0ull;
      const int gm = lane < C ? hs->row : INT_MAX;
      int gi = gm;
      rleaf_argmax_warp(gk, gi);
      const unsigned m = __ballot_sync(0xffffffffu, lane < C && gm == gi);
      best = cslot + par * C + (m ? __ffs(m) - 1 : c);
      r = gi;
    } else {
      __syncthreads();  // the CTA's candidate row is visible to every warp
    }
    const double* u = best->v;  // the pivot row
    const double* oldj = rowj + par * W;
    if (r == INT_MAX) {
      // no orderable candidate (every magnitude NaN): keep row j, as idamax
      // does when no later entry compares greater than the first
      r = j;
      u = oldj;
    }
    const double piv = u[j];
    if (c == 0 && tid == 0) a.piv[j] = r - j;
    if (tid == 0) s_r[j] = r;
    bv = -1.0;
    bi = INT_MAX;
    bk = 0;
    if (piv == 0.0) {
      // null column: no exchange, no scaling, no update
      if (first_null < 0) first_null = j;
      if (j + 1 < W)
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
          const int i = tid + k * RLEAF_THREADS, gi = r0 + i;
          if (i < rows && gi > j) {
            const double t = fabs(rleaf_pick_col<W>(rv[k], j + 1));
            if (t > bv) { bv = t; bi = gi; bk = k; }
          }
        }
      continue;
    }
    // ---- 4. exchange, scale, update, next candidate
    rleaf_column_at<W, RPT>(j, rv, tid, r0, rows, r, u, oldj, 1.0 / piv, bv, bi, bk);
  }
  rleaf_store<W, RPT>(rv, a, r0, rows, tile, warp, lane);
  if (c == 0 && tid == 0 && first_null >= 0) atomicMin(a.info, a.gcol + first_null);
  if (done && a.pl + a.pr > 0) rleaf_apply_pivots<W>(a, s_r, c, C, reinterpret_cast<double*>(rleaf_smem + rleaf_tile_offset(W, C)));
  // no CTA leaves while another may still copy into its shared memory
  if (C > 1) cluster.sync();
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
  for (auto kern : {lu_leaf_reg_kernel<8, 4>, lu_leaf_reg_kernel<16, 2>, lu_leaf_reg_kernel<32, 1>}) {
    FB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    FB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)rleaf_smem_bytes(32, LEAF_MAXC)));
  }
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

int rleaf_launch(double* P, long ld, long M, int w, int* d_piv, int gcol, cudaStream_t st, int pl = 0, int pr = 0) {
  int C = 0, R = 0;
  if (!rleaf_geometry(M, w, &C, &R)) {
    set_last_error("LU panel leaf does not fit in a cluster");
    return FLA_FAILURE;
  }
  LeafArgs la = {};
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
  la.pl = pl;
  la.pr = pr;
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
  LeafArgs la = {};
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
// Panel recursion in which every leaf is register-resident and applies its
// row interchanges to the other columns of the panel itself (pl columns left
// of this sub-panel, pr right of it): the joins need no interchange launches.
int panel_rec_reg(double* P, long ld, long M, int w, int* d_piv, int gcol, int pl, int pr, cudaStream_t st) {
  int C, R;
  if (rleaf_geometry(M, w, &C, &R)) return rleaf_launch(P, ld, M, w, d_piv, gcol, st, pl, pr);
  const int w1 = std::max(8, (w / 2) & ~7);
  const int w2 = w - w1;
  if (panel_rec_reg(P, ld, M, w1, d_piv, gcol, pl, pr + w2, st) != FLA_SUCCESS) return FLA_FAILURE;
  // U12 := inv(L11) U12 (U12^T is the w2 x w1 block at P + w1)
  if (u12_subst(P, P + w1, ld, w1, w2, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (M > w1) {
    if (gemm_f64(st, false, false, w2, M - w1, w1, -1.0, P + w1, ld, P + (long)w1 * ld, ld, 1.0,
                 P + w1 + (long)w1 * ld, ld) != FLA_SUCCESS)
      return FLA_FAILURE;
    if (panel_rec_reg(P + w1 + (long)w1 * ld, ld, M - w1, w2, d_piv + w1, gcol + w1, pl + w1, pr, st) != FLA_SUCCESS)
      return FLA_FAILURE;
  }
  return FLA_SUCCESS;
}

// True when every leaf of the recursion below (halves rounded down to
// multiples of 8, leaves of 8, 16 or 32 columns) fits the register leaf:
// the rows only shrink down the recursion, so the top M decides.
bool panel_all_reg(long M, int w) {
  int C, R;
  if (w % 8 != 0) return false;
  if (rleaf_geometry(M, w, &C, &R)) return true;
  if (w <= 32) return false;
  const int w1 = std::max(8, (w / 2) & ~7);
  return panel_all_reg(M, w1) && panel_all_reg(M, w - w1);
}

int lu_panel_factor_t(double* P, long ld, long M, int w, int* d_piv, int gcol, cudaStream_t st) {
  if (leaf_setup() != FLA_SUCCESS) return FLA_FAILURE;
  if (w <= 0 || M <= 0) return FLA_SUCCESS;
  if (w > 32 && panel_all_reg(M, w)) return panel_rec_reg(P, ld, M, w, d_piv, gcol, 0, 0, st);
  int C, R, lds;
  size_t smem;
  if (rleaf_geometry(M, w, &C, &R)) return rleaf_launch(P, ld, M, w, d_piv, gcol, st);
  if (leaf_geometry(M, w, &C, &R, &lds, &smem) || w <= 2) return leaf_launch(P, ld, M, w, d_piv, gcol, true, st);
  const int w1 = std::max(2, (w / 2) & ~1);
  const int w2 = w - w1;
  if (lu_panel_factor_t(P, ld, M, w1, d_piv, gcol, st) != FLA_SUCCESS) return FLA_FAILURE;
  if (laswp_t_dev(P, ld, 0, d_piv, w1, w1, w2, 0, 0, st) != FLA_SUCCESS) return FLA_FAILURE;
  // U12 := inv(L11) U12 (U12^T is the w2 x w1 block at P + w1)
  if (u12_subst(P, P + w1, ld, w1, w2, st) != FLA_SUCCESS) return FLA_FAILURE;
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
