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
  int rt_log = 5;  // log2 of the slab height rounded up to a power of two (>= 32)
  while ((1 << rt_log) < rows && rt_log < 10) ++rt_log;
  const int rt_mask = (1 << rt_log) - 1;
  const int i_row0 = tid & rt_mask, cg = tid >> rt_log, cgs = LEAF_THREADS >> rt_log;
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

  int first_null = -1;
  for (int j = 0; j < w; ++j) {
    const int par = j & 1;
    // ---- 1. local candidate: max |a(i,j)| over rows i >= j, smallest row on ties
    double bv = -1.0;
    int bi = INT_MAX;
    for (int i = tid; i < rows; i += LEAF_THREADS) {
      const int gi = r0 + i;
      if (gi >= j) {
        const double v = fabs(slab[i + j * lds]);
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
    if (warp == 0) {
      double v = s_rv[lane];  // LEAF_THREADS / 32 == 32 partial results
      int i0 = s_ri[lane];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i0, off);
        if (ov > v || (ov == v && oi < i0)) { v = ov; i0 = oi; }
      }
      if (lane == 0) {
        s_bv = v;
        s_bi = i0;
      }
    }
    __syncthreads();
    // ---- 2. push the candidate (and row j, by its owner) to every CTA
    {
      const int li = s_bi - r0;  // local row of the candidate (if any)
      const bool have = s_bi != INT_MAX;
      const bool own_j = (j >= r0) && (j < r0 + rows);
      const int per = w + 1;
      for (int e = tid; e < C * per; e += LEAF_THREADS) {
        const int d = e / per, q = e - d * per;
        if (q < w) {
          double* dst = cluster.map_shared_rank(xrow + ((size_t)par * C + c) * w + q, d);
          *dst = have ? slab[li + q * lds] : 0.0;
        } else {
          *cluster.map_shared_rank(xval + par * C + c, d) = s_bv;
          *cluster.map_shared_rank(xidx + par * C + c, d) = s_bi;
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
      int i0 = INT_MAX, w0 = 0;
      for (int q = lane; q < C; q += 32) {
        const double cv = xval[par * C + q];
        const int ci = xidx[par * C + q];
        if (ci != INT_MAX && (cv > v || (cv == v && ci < i0))) { v = cv; i0 = ci; w0 = q; }
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, off);
        const int oi = __shfl_xor_sync(0xffffffffu, i0, off);
        const int ow = __shfl_xor_sync(0xffffffffu, w0, off);
        if (ov > v || (ov == v && oi < i0)) { v = ov; i0 = oi; w0 = ow; }
      }
      if (lane == 0) { s_wc = w0; s_r = i0; }
    }
    __syncthreads();
    int r = s_r;
    const double* u = xrow + ((size_t)par * C + s_wc) * w;  // the pivot row
    if (r == INT_MAX) {
      // no orderable candidate (every magnitude NaN): keep row j, as idamax
      // does when no later entry compares greater than the first
      r = j;
      u = rowj + par * w;
    }
    const double piv = u[j];
    if (c == 0 && tid == 0) a.piv[j] = r - j;
    if (piv == 0.0) {
      if (first_null < 0) first_null = j;
    } else {
      if (r != j) {
        // ---- 4. exchange rows j and r (whole leaf row)
        if (j >= r0 && j < r0 + rows)
          for (int q = tid; q < w; q += LEAF_THREADS) slab[(j - r0) + q * lds] = u[q];
        if (r >= r0 && r < r0 + rows)
          for (int q = tid; q < w; q += LEAF_THREADS) slab[(r - r0) + q * lds] = rowj[par * w + q];
      }
      __syncthreads();
      // ---- 5. scale column j below the pivot (reciprocal multiply, as
      // bl1_dinvscalv), then the rank-1 update of the slab, one element per
      // thread and pass (rows fastest), four independent elements in flight
      const double rinv = 1.0 / piv;
      const int i_lo = max(0, j + 1 - r0);  // first local row below the pivot
      for (int i = i_lo + tid; i < rows; i += LEAF_THREADS) slab[i + j * lds] *= rinv;
      __syncthreads();
      // thread -> (row i = tid mod RT, column group cg = tid / RT); RT is the
      // slab height rounded up to a power of two, so no divisions
      for (int i_row = i_row0 + max(0, ((i_lo - i_row0) + rt_mask) >> rt_log << rt_log); i_row < rows;
           i_row += rt_mask + 1) {
        const double l = slab[i_row + j * lds];
        int q = j + 1 + cg;
        for (; q + 3 * cgs < w; q += 4 * cgs) {
          double v[4], uq[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            v[k] = slab[i_row + (q + k * cgs) * lds];
            uq[k] = u[q + k * cgs];
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) slab[i_row + (q + k * cgs) * lds] = fma(-l, uq[k], v[k]);
        }
        for (; q < w; q += cgs) slab[i_row + q * lds] = fma(-l, u[q], slab[i_row + q * lds]);
      }
    }
    __syncthreads();
  }
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

struct LeafConfig {
  bool ready = false;
  int max_cluster = 8;
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
  g_leaf.ready = true;
  return FLA_SUCCESS;
}

// Cluster size and slab geometry for an M x w leaf; false if it does not fit.
// Widest leaf: the leaf's rank-1 updates re-read the whole slab every
// column, so wide leaves are split and their halves joined by DMMA GEMMs;
// FLA_B200_LU_LEAF_MAXW (8..128) overrides the default for tuning.
int leaf_maxw() {
  static int mw = 0;
  if (mw == 0) {
    mw = 64;
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
