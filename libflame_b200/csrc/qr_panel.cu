// Householder QR panel for FLA_QR_UT, B200 form: a recursive split of the
// panel whose leaves run inside one thread-block cluster with the panel in
// registers.
//
// Reference: the panel step of FLA_QR_UT_blk_var1
// (src/lapack/dec/q/qrut/vars/flamec/FLA_QR_UT_blk_var1.c:52-60), whose
// unblocked leaf FLA_QR_UT_opt_var2.c:161-226 forms, per column j,
//   the Householder vector of FLA_Househ2_UT.c:274-386
//     alpha = -sign(chi1) ||[chi1; x2]||,  u2 = x2 / (chi1 - alpha),
//     tau = 1/2 + 1/2 (||x2|| / |chi1 - alpha|)^2,  chi1 := alpha
//     (||x2|| = 0: tau = 1/2, chi1 := -chi1),
//   w = (a12 + A22^T u2) / tau, A12 -= w, A22 -= u2 w^T,
//   and column j of T: t01 = a10 + A20^T u2 above the diagonal tau.
//
// Leaf (qr_leaf_kernel<W>): an M x w panel (w <= W in {8, 16, 32}),
// column-major.  Lanes map to columns: lane (g, q) of a warp holds column q
// of 32 consecutive rows (row group g of the warp's 32 * (32 / W) rows), so
// every dot product of column j with the other columns accumulates in the
// lane that owns the other column and needs no shuffle reduction, and the
// rank-1 update of column q runs in its own lane.  Per column j:
//   1. the lanes holding column j broadcast it (rows <= j masked to zero)
//      through shared memory; every lane accumulates x^T a_q over its rows,
//      the row groups of a warp are summed and written to the warp's slot;
//      the owner of row j publishes row j;
//   2. one CTA barrier; the CTA's partial vector is the fixed-order sum of
//      the 16 warp slots (its entry q = j is ||x2||^2);
//   3. (clusters only) warp 0 bulk-copies the CTA's partial vector, and
//      CTA 0 row j, into every other CTA's shared memory, waits for the
//      column's bytes on its mbarrier, and a second CTA barrier releases
//      the CTA; every lane sums the C partial vectors in CTA order, so every
//      CTA holds the same bits;
//   4. every lane forms alpha, tau and the scale 1 / (chi1 - alpha); since
//      u2 = x2 * scale, u2^T a_q = scale * (x^T a_q), so one exchange per
//      column gives both ||x2|| and the update row w; the column-j lanes
//      scale their column into u2 and broadcast u (with u_j = 1), and the
//      lanes q > j apply a_q -= u w_q.  CTA 0 writes column j of T.
// One exchange per column where the reference's order needs two reductions
// (the norm, then the dot products): the sums are the same up to the
// rounding of scaling before or after the summation.
//
// Recursion (qr_panel_factor): a panel too wide for a leaf, or too tall for
// a cluster at that width, is split in halves: factor the left half,
// B := (I - U1 T11^-T U1^T) B on the right half with the GEMM engine, factor
// the right half's lower part, and form T12 = U1^T U2, so that the panel's
// whole T (striu(U^T U) + diag(tau), the UT transform's triangular factor)
// is available to the blocked trailing update.
#include <cooperative_groups.h>

#include <algorithm>
#include <climits>

#include "common.h"
#include "dev_util.cuh"

namespace cg = cooperative_groups;

namespace fb {

// Cooperative panel kernel of qr.cu, for pieces taller than any cluster.
int qr_coop_panel(double* P, long ld, long M, int nb, double* Tb, long ldtb, cudaStream_t st);
int unit_lower_copy(const double* P, long ldp, double* U, long ldu, long M, int b, cudaStream_t st);

namespace {

constexpr int QL_THREADS = 512;
constexpr int QL_NW = QL_THREADS / 32;
constexpr int QL_MAXC = 16;

struct QrLeafArgs {
  double* P;  // panel (row 0, col 0), column-major
  long ld;
  int M;      // rows
  int w;      // columns actually present (<= W)
  int R;      // rows per CTA
  double* T;  // out: w x w upper triangle with the diagonal (ld ldt)
  long ldt;
  double* U;  // out (optional): the unit lower trapezoid of the factored panel (ld ldu)
  long ldu;
  int* err;
};

// Shared memory, in doubles: per warp a 32G x (W + 1) staging tile (the
// column broadcast xs[32G] reuses its start during the column loop);
// wpart[2][16][W]; cslot[2][C][W]; rowj[2][W]; two mbarriers.
__host__ __device__ inline size_t qleaf_tile_doubles(int W) { return (size_t)(32 * 32 / W) * (W + 1); }
__host__ __device__ inline size_t qleaf_smem_bytes(int W, int C) {
  return sizeof(double) * (QL_NW * qleaf_tile_doubles(W) + 2 * QL_NW * (size_t)W + 2 * (size_t)C * W + 2 * W) +
         16 + 128;
}

template <int W>
__global__ void __launch_bounds__(QL_THREADS, 1) qr_leaf_kernel(QrLeafArgs a) {
  constexpr int G = 32 / W;   // row groups per warp
  constexpr int WR = 32 * G;  // rows per warp
  extern __shared__ __align__(128) unsigned char qleaf_smem[];
  cg::cluster_group cluster = cg::this_cluster();
  const int C = (int)cluster.num_blocks();
  const int c = (int)cluster.block_rank();
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = lane % W, g = lane / W;
  double* base = reinterpret_cast<double*>(qleaf_smem);
  double* tile = base + (size_t)warp * qleaf_tile_doubles(W);
  double* xs = tile;  // column j of the warp's rows (rows <= j zero)
  double* wpart = base + QL_NW * qleaf_tile_doubles(W);  // [2][16][W]
  double* cslot = wpart + 2 * QL_NW * W;                 // [2][C][W]
  double* rowj = cslot + 2 * (size_t)C * W;              // [2][W]
  const uint32_t full0 = smem_u32(rowj + 2 * W);
  const int r0 = c * a.R;
  const int rows = max(0, min(a.R, a.M - r0));
  const int wrow0 = warp * WR;  // first row of the warp within the CTA
  if (C > 1) {
    if (tid == 0) {
      mbar_init(full0, 1);
      mbar_init(full0 + 8, 1);
      fence_barrier_init();
    }
    cluster.sync();
  }

  // ---- load: the warp reads each column's 32G rows coalesced into its
  // tile, then lane (g, q) takes column q of rows g*32 .. g*32 + 31
  double v[32];
#pragma unroll 4
  for (int e = lane; e < WR * W; e += 32) {
    const int qq = e / WR, rr = e % WR;
    const int li = wrow0 + rr;
    tile[rr * (W + 1) + qq] = (qq < a.w && li < rows) ? a.P[(long)(r0 + li) + (long)qq * a.ld] : 0.0;
  }
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = tile[(g * 32 + i) * (W + 1) + q];
  __syncwarp();

  const int gfirst = r0 + wrow0 + g * 32;  // global row of v[0]
  const int ncols = min(a.w, a.M);
#pragma unroll 1
  for (int j = 0; j < ncols; ++j) {
    const int par = j & 1;
    // ---- 1. broadcast column j; row j; partial dot products
    const bool low = r0 + wrow0 <= j;  // this warp holds rows <= j (CTA 0, warp 0)
    if (q == j) {
      if (low) {
#pragma unroll
        for (int i = 0; i < 32; i += 2)
          *reinterpret_cast<double2*>(xs + g * 32 + i) =
              make_double2(gfirst + i > j ? v[i] : 0.0, gfirst + i + 1 > j ? v[i + 1] : 0.0);
      } else {
#pragma unroll
        for (int i = 0; i < 32; i += 2) *reinterpret_cast<double2*>(xs + g * 32 + i) = make_double2(v[i], v[i + 1]);
      }
    }
    if (low && j >= gfirst && j < gfirst + 32) {
      // row j lives in this lane group: publish it
      const int ij = j - gfirst;
      double r = v[0];
#pragma unroll
      for (int i = 1; i < 32; ++i)
        if (i == ij) r = v[i];
      rowj[par * W + q] = r;
      if (C > 1) fence_proxy_async_smem();
    }
    __syncwarp();
    double d = 0.0;
#pragma unroll
    for (int i = 0; i < 32; i += 2) {
      const double2 x = *reinterpret_cast<const double2*>(xs + g * 32 + i);
      d = fma(x.x, v[i], d);
      d = fma(x.y, v[i + 1], d);
    }
#pragma unroll
    for (int off = W; off < 32; off <<= 1) d += __shfl_xor_sync(0xffffffffu, d, off);
    if (g == 0) wpart[(par * QL_NW + warp) * W + q] = d;
    __syncthreads();
    // ---- 2. the CTA's partial vector (fixed warp order)
    double cs = 0.0;
#pragma unroll
    for (int ww = 0; ww < QL_NW; ++ww) cs += wpart[(par * QL_NW + ww) * W + q];
    // ---- 3. the cluster's sum
    double dq = cs;
    if (C > 1) {
      const uint32_t fullp = full0 + 8 * par;
      const uint32_t ph = (uint32_t)((j >> 1) & 1);
      double* own = cslot + ((size_t)par * C + c) * W;
      bool ok = true;
      if (warp == 0) {
        if (g == 0) own[q] = cs;
        fence_proxy_async_smem();
        __syncwarp();
        if (lane < C && lane != c) {
          const uint32_t rbar = mapa_shared(fullp, (uint32_t)lane);
          bulk_copy_to_peer(mapa_shared(smem_u32(own), (uint32_t)lane), smem_u32(own), (uint32_t)(8 * W), rbar);
          if (c == 0)
            bulk_copy_to_peer(mapa_shared(smem_u32(rowj + par * W), (uint32_t)lane), smem_u32(rowj + par * W),
                              (uint32_t)(8 * W), rbar);
        }
        if (lane == 0) mbar_arrive_expect_tx(fullp, (uint32_t)((C - 1) * 8 * W + (c == 0 ? 0 : 8 * W)));
        ok = mbar_wait_cluster(fullp, ph, a.err, 33);
      }
      // the CTA leaves the loop together if the (bounded) wait ran out
      if (__syncthreads_or(ok ? 0 : 1)) break;
      if (warp != 0) (void)mbar_try_wait_cluster(fullp, ph);  // acquire of the completed phase
      dq = 0.0;
#pragma unroll
      for (int cc = 0; cc < QL_MAXC; ++cc)
        if (cc < C) dq += (cc == c) ? cs : cslot[((size_t)par * C + cc) * W + q];
    }
    // ---- 4. Householder vector, w, T column; the update
    const double ss = __shfl_sync(0xffffffffu, dq, j);  // ||x2||^2 (lane j of group 0)
    const double chi1 = rowj[par * W + j];
    const double nx2 = sqrt(ss);
    double scale, alpha, tau;
    const bool trivial = nx2 == 0.0;
    if (trivial) {
      scale = 1.0;
      alpha = -chi1;
      tau = 0.5;
    } else {
      const double nx = sqrt(fma(chi1, chi1, ss));  // ||[chi1; x2]||
      alpha = -((chi1 < 0.0) ? -1.0 : 1.0) * nx;
      const double cma = chi1 - alpha;
      scale = 1.0 / cma;
      const double qq = nx2 * fabs(scale);  // ||x2|| / |chi1 - alpha|
      tau = 0.5 + 0.5 * (qq * qq);
    }
    const double rtau = 1.0 / tau;
    const double tq = rowj[par * W + q] + scale * dq;  // a1(q) + u2^T a2(q)
    if (c == 0 && warp == 0 && g == 0 && q < a.w) {
      if (q < j) a.T[q + (long)j * a.ldt] = tq;
      else if (q == j) a.T[j + (long)j * a.ldt] = tau;
    }
    // column j becomes u2 (alpha at row j); the columns right of it lose
    // u w_q, u read back from the broadcast column (u = x scale below row
    // j, 1 at row j, 0 above: rows <= j of xs hold zeros, row j is fixed
    // up by its own lane group)
    if (q == j) {
      if (low) {
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const int gi = gfirst + i;
          v[i] = gi > j ? (trivial ? v[i] : v[i] * scale) : (gi == j ? alpha : v[i]);
        }
      } else if (!trivial) {
#pragma unroll
        for (int i = 0; i < 32; ++i) v[i] *= scale;
      }
    } else if (q > j) {
      const double wq = tq * rtau;
#pragma unroll
      for (int i = 0; i < 32; i += 2) {
        const double2 x = *reinterpret_cast<const double2*>(xs + g * 32 + i);
        v[i] = fma(-(trivial ? x.x : x.x * scale), wq, v[i]);
        v[i + 1] = fma(-(trivial ? x.y : x.y * scale), wq, v[i + 1]);
      }
      if (low && j >= gfirst && j < gfirst + 32) {
        const int ij = j - gfirst;
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (i == ij) v[i] -= wq;
      }
    }
    __syncwarp();  // xs is rewritten for the next column
  }
  // ---- store through the tile
  __syncwarp();
#pragma unroll
  for (int i = 0; i < 32; ++i) tile[(g * 32 + i) * (W + 1) + q] = v[i];
  __syncwarp();
#pragma unroll 4
  for (int e = lane; e < WR * W; e += 32) {
    const int qq = e / WR, rr = e % WR;
    const int li = wrow0 + rr;
    if (qq < a.w && li < rows) {
      const double x = tile[rr * (W + 1) + qq];
      a.P[(long)(r0 + li) + (long)qq * a.ld] = x;
      if (a.U) {
        const int gi = r0 + li;
        a.U[gi + (long)qq * a.ldu] = gi > qq ? x : (gi == qq ? 1.0 : 0.0);
      }
    }
  }
  // no CTA leaves while another may still copy into its shared memory
  if (C > 1) cluster.sync();
}

struct QrLeafConfig {
  bool ready = false;
  int max_cluster = 1;
};
QrLeafConfig g_ql;

int qleaf_setup() {
  if (g_ql.ready) return FLA_SUCCESS;
  const int smem = (int)std::max({qleaf_smem_bytes(8, QL_MAXC), qleaf_smem_bytes(16, QL_MAXC),
                                  qleaf_smem_bytes(32, QL_MAXC)});
  for (auto kern : {qr_leaf_kernel<8>, qr_leaf_kernel<16>, qr_leaf_kernel<32>}) {
    FB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    FB_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  }
  g_ql.max_cluster = 1;
  for (int cs = QL_MAXC; cs >= 2; cs >>= 1) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs);
    cfg.blockDim = dim3(QL_THREADS);
    cfg.dynamicSmemBytes = (size_t)smem;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    bool ok = true;
    for (auto kern : {qr_leaf_kernel<8>, qr_leaf_kernel<16>, qr_leaf_kernel<32>}) {
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, kern, &cfg) != cudaSuccess || n <= 0) ok = false;
      cudaGetLastError();
    }
    if (ok) {
      g_ql.max_cluster = cs;
      break;
    }
  }
  g_ql.ready = true;
  return FLA_SUCCESS;
}

// Leaf width for an M x w piece (0: none fits): the narrowest of 8, 16, 32
// holding w, if its cluster holds M rows (512 * 32 / W rows per CTA).
int qleaf_width(long M, int w) {
  for (int W : {8, 16, 32}) {
    if (w > W) continue;
    const long cap = (long)g_ql.max_cluster * QL_THREADS * (32 / W);
    return M <= cap ? W : 0;
  }
  return 0;
}

int qleaf_launch(double* P, long ld, long M, int w, int W, double* T, long ldt, double* U, long ldu,
                 cudaStream_t st) {
  const long per = (long)QL_THREADS * (32 / W);
  const int C = (int)((M + per - 1) / per);
  QrLeafArgs la;
  la.P = P;
  la.ld = ld;
  la.M = (int)M;
  la.w = w;
  la.R = (int)((M + C - 1) / C);
  la.T = T;
  la.ldt = ldt;
  la.U = U;
  la.ldu = ldu;
  la.err = ctx().d_status + ST_ERROR;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(QL_THREADS);
  cfg.dynamicSmemBytes = qleaf_smem_bytes(W, C);
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const int ps = prof_begin(st);
  if (W == 8) FB_CK(cudaLaunchKernelEx(&cfg, qr_leaf_kernel<8>, la));
  else if (W == 16) FB_CK(cudaLaunchKernelEx(&cfg, qr_leaf_kernel<16>, la));
  else FB_CK(cudaLaunchKernelEx(&cfg, qr_leaf_kernel<32>, la));
  prof_end(ps, st, PROF_PANEL, 0.0);
  count_launch();
  return FLA_SUCCESS;
}

// U (M x b, ld ldu) := the unit lower trapezoid of P (ones on the diagonal,
// zeros above, P below).
__global__ void qr_unit_lower_kernel(const double* __restrict__ P, long ldp, double* __restrict__ U, long ldu,
                                     int M, int b) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)M * b) return;
  const int col = (int)(idx / M), row = (int)(idx % M);
  U[row + (long)col * ldu] = row > col ? P[row + (long)col * ldp] : (row == col ? 1.0 : 0.0);
}

// Factor the M x w piece P (ld) in place; Tb (ld ldtb) receives its w x w
// T and U (ld ldu, aligned with P: U[i + q ldu] is element (i, q) of the
// piece) its unit lower trapezoid, rows 0 .. M - 1.  Wk (w x w, ld ldw) is
// scratch.
int panel_rec(double* P, long ld, long M, int w, double* Tb, long ldtb, double* U, long ldu, double* Wk,
              long ldw, cudaStream_t st) {
  if (w <= 0 || M <= 0) return FLA_SUCCESS;
  const int W = qleaf_width(M, w);
  if (W > 0) return qleaf_launch(P, ld, M, w, W, Tb, ldtb, U, ldu, st);
  if (w <= 8) {
    if (qr_coop_panel(P, ld, M, w, Tb, ldtb, st) != FLA_SUCCESS) return FLA_FAILURE;
    return unit_lower_copy(P, ld, U, ldu, M, w, st);
  }
  // split: the left half a multiple of 8 columns
  const int w1 = std::max(8, (w / 2) & ~7);
  const int w2 = w - w1;
  if (panel_rec(P, ld, M, w1, Tb, ldtb, U, ldu, Wk, ldw, st) != FLA_SUCCESS) return FLA_FAILURE;
  // B := (I - U1 T11^-T U1^T) B on the right half: W := U1^T B,
  // W := T11^-T W (through T11^-1 for the wider halves), B -= U1 W
  double* B = P + (long)w1 * ld;
  double* W1 = Wk;
  if (gemm_f64(st, true, false, w1, w2, M, 1.0, U, ldu, B, ld, 0.0, W1, ldw) != FLA_SUCCESS) return FLA_FAILURE;
  if (w1 >= 32) {
    double* Ti = Wk + (long)ldw * w2;          // w1 x w1
    double* W2 = Ti + (long)ldw * w1;          // w1 x w2
    if (tri_inverse(Tb, ldtb, w1, false, false, Ti, ldw, st) != FLA_SUCCESS) return FLA_FAILURE;
    if (gemm_f64(st, true, false, w1, w2, w1, 1.0, Ti, ldw, W1, ldw, 0.0, W2, ldw) != FLA_SUCCESS)
      return FLA_FAILURE;
    W1 = W2;
  } else if (trsm_block(Tb, ldtb, W1, ldw, w1, w2, false, true, false, st) != FLA_SUCCESS) {
    return FLA_FAILURE;
  }
  if (gemm_f64(st, false, false, M, w2, w1, -1.0, U, ldu, W1, ldw, 1.0, B, ld) != FLA_SUCCESS) return FLA_FAILURE;
  if (M <= w1) return FLA_SUCCESS;
  // the lower right part, then T12 = U1^T U2 over rows w1 .. M - 1
  if (panel_rec(B + w1, ld, M - w1, w2, Tb + w1 + (long)w1 * ldtb, ldtb, U + w1 + (long)w1 * ldu, ldu, Wk, ldw,
                st) != FLA_SUCCESS)
    return FLA_FAILURE;
  const int w2e = (int)std::min<long>(w2, M - w1);
  return gemm_f64(st, true, false, w1, w2e, M - w1, 1.0, U + w1, ldu, U + w1 + (long)w1 * ldu, ldu, 0.0,
                  Tb + (long)w1 * ldtb, ldtb);
}

}  // namespace

int unit_lower_copy(const double* P, long ldp, double* U, long ldu, long M, int b, cudaStream_t st) {
  const long total = M * b;
  if (total <= 0) return FLA_SUCCESS;
  qr_unit_lower_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(P, ldp, U, ldu, (int)M, b);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// Factor the M x w panel P (ld) in place (M >= w); Tb (ld ldtb) receives
// the panel's w x w upper triangular T and U (ld ldu >= M, w columns) its
// unit lower trapezoid, ready for the trailing update.  Wk (ld ldw >= w, 3w
// columns) is scratch.
int qr_panel_factor(double* P, long ld, long M, int w, double* Tb, long ldtb, double* U, long ldu, double* Wk,
                    long ldw, cudaStream_t st) {
  if (qleaf_setup() != FLA_SUCCESS) return FLA_FAILURE;
  if (w <= 0 || M <= 0) return FLA_SUCCESS;
  // the leaves write U from their own first row down; the zeros above the
  // diagonal of the later pieces lie in the top w x w block
  FB_CK(cudaMemset2DAsync(U, sizeof(double) * ldu, 0, sizeof(double) * w, w, st));
  return panel_rec(P, ld, M, w, Tb, ldtb, U, ldu, Wk, ldw, st);
}

}  // namespace fb
