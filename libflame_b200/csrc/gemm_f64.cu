// FP64 GEMM engine on the B200 FP64 tensor cores (DMMA, mma.sync m8n8k4 f64),
// fed by TMA through a multi-stage mbarrier pipeline.
//
//   C := alpha * op(A) * op(B) + beta * C        (column-major)
//
// Replaces the reference's level-3 BLAS calls on the factorization path
// (dgemm_/dsyrk_ reached through FLA_Gemm_external / FLA_Herk_external,
// src/base/flamec/wrappers/blas/3/external/FLA_Gemm_external.c:92,
// FLA_Herk_external.c:83).  GEMM_LOWER writes only the lower triangle
// (i - j >= diag_off), which is the SYRK update of the Cholesky.
//
// Tile: 64 (m) x 64 (n) per CTA with 4 warps and 3 stages, four CTAs per SM
// (or 128 x 64 with 8 warps and 4 stages, two CTAs per SM); k staged 16 at a
// time.  Warps form a (BM/32) x 2 grid, each owning a 32 x 32 sub-tile as
// 4 x 4 m8n8 DMMA accumulators; thread 0 also issues the TMA loads
// (refilling a stage once all warps have released it).  Several CTAs share
// an SM so one CTA's prologue and epilogue overlap the others' MMAs.
//
// Shared-memory layout: TMA boxes are 128 bytes wide (16 doubles) with the
// 128-byte swizzle (16-byte chunk index XOR row index mod 8).  An operand
// whose MMA-row index (m of A, n of B) is the contiguous one is stored as
// boxes of 16 rows x 16 k; one whose k is contiguous as rows of 16 k.  The
// lanes of each DMMA fragment take rows in the orders PERM16 / PERM8 below,
// which make every fragment load hit 16 distinct 8-byte bank pairs per
// half-warp; the accumulator rows/columns follow the same orders.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "common.h"
#include "dev_util.cuh"

namespace fb {

namespace {

constexpr int BN = 64, BK = 16;

// Tile shapes: BM = 128 (8 warps, 4 stages, 2 CTAs per SM) or BM = 64
// (4 warps, 3 stages, 4 CTAs per SM), BN = 64; and 128 x 32 (4 warps) for
// products with at most 32 columns (the refinement residual B - A X).  Each
// warp owns a 32 x 32 sub-tile.
template <int BM_, int BN_ = BN>
struct Tile {
  static constexpr int BM = BM_;
  static constexpr int BNT = BN_;
  static constexpr int WM = BM / 32;                 // warps along m
  static constexpr int WN = BN_ / 32;                // warps along n
  static constexpr int WARPS = WM * WN;
  static constexpr int THREADS = WARPS * 32;
  static constexpr int STAGES = BM == 128 ? 4 : 3;
  static constexpr int MINB = BM == 128 ? 2 : 4;      // CTAs per SM
  static constexpr int A_STAGE_BYTES = BM * BK * 8;
  static constexpr int B_STAGE_BYTES = BN_ * BK * 8;
  static constexpr int STAGE_BYTES = A_STAGE_BYTES + B_STAGE_BYTES;
  static constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 2048 /*align*/ + 256 /*barriers*/;
};

// Row order of the 8 lane groups of a fragment when the operand's MMA-row
// index is contiguous in memory (16-row box, two 8-row halves):
//   half 0: 0 1 8 9 2 3 10 11      half 1: 4 5 12 13 6 7 14 15
__device__ __forceinline__ int perm16_tab(int half, int g) {
  return (g & 1) + ((g >> 1) & 1) * 8 + ((g >> 2) & 1) * 2 + half * 4;
}
// Row order when k is the contiguous index: 0 2 4 6 1 3 5 7.
__device__ __forceinline__ int perm8_tab(int g) { return (g & 3) * 2 + (g >> 2); }

// Byte offset in a stage tile of element (r, k) where r is the MMA-row index
// (m for A, n for B), for the two storage kinds:
//   r contiguous: (r>>4)*2048 + k*128 + ((((r&15)>>1) ^ (k&7)) << 4) + (r&1)*8
//   k contiguous: r*128 + (((k>>1) ^ (r&7)) << 4) + (k&1)*8
// A lane reads k = 4*kk + t (kk = 0..3 inside a 16-wide k stage, t = lane&3).
// Every term above occupies its own bits, so the offset splits into a
// per-lane base (independent of kk) XOR a per-kk constant:
//   r contiguous: base ^ ((kk << 9) | ((kk & 1) << 6))
//   k contiguous: base ^ (kk << 5)
// and, the stage tiles being 2048-byte aligned, the XOR can be applied to the
// shared-memory address itself (one LOP3 per fragment load).
__device__ __forceinline__ uint32_t base_rcontig(int r, int t) {
  return (uint32_t)((r >> 4) * 2048 + t * 128 + ((((r & 15) >> 1) ^ t) << 4) + ((r & 1) << 3));
}
__device__ __forceinline__ uint32_t base_kcontig(int r, int t) {
  return (uint32_t)(r * 128 + ((t & 1) << 3) + ((((t >> 1) ^ (r & 1))) << 4) + (((r & 7) >> 1) << 5));
}
template <bool KC>
__device__ __forceinline__ constexpr uint32_t kk_xor(int kk) {
  return KC ? (uint32_t)(kk << 5) : (uint32_t)((kk << 9) | ((kk & 1) << 6));
}
__device__ __forceinline__ double lds_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared.f64 %0, [%1];" : "=d"(v) : "r"(addr));
  return v;
}

template <bool A_K, bool B_K, int BM_, int BN_ = BN>
__global__ void __launch_bounds__(Tile<BM_, BN_>::THREADS, Tile<BM_, BN_>::MINB)
    dgemm_tma_kernel(const __grid_constant__ CUtensorMap mapA,
                     const __grid_constant__ CUtensorMap mapB, double* __restrict__ C, long ldc,
                     int M, int N, int K, double alpha, double beta, int mode, long diag_off,
                     int* err, const int* guard, int guard_limit, int k_chunk, long c_zstride) {
  using TC = Tile<BM_, BN_>;
  constexpr int BN = TC::BNT;  // shadows the default 64 for this instantiation
  constexpr int BM = TC::BM, STAGES = TC::STAGES, THREADS = TC::THREADS, CONSUMER_WARPS = TC::WARPS;
  constexpr int A_STAGE_BYTES = TC::A_STAGE_BYTES, STAGE_BYTES = TC::STAGE_BYTES;
  extern __shared__ unsigned char smem_raw[];
  if (guard && *((volatile const int*)guard) < guard_limit) return;
  const int tile_m = blockIdx.x * BM;
  const int tile_n = blockIdx.y * BN;
  if (mode == GEMM_LOWER) {
    // skip tiles strictly above the band i - j >= diag_off
    long max_i = (long)tile_m + BM - 1, min_j = tile_n;
    if (max_i - min_j < diag_off) return;
  }
  if (beta != 0.0) {
    // Bring this tile of C from HBM into L2 while the k-loop runs, so the
    // epilogue reads hit L2: 64 columns x 8 lines of 128 B (128 rows).
    const int t = threadIdx.x;
    for (int l = t; l < BN * (BM / 16); l += THREADS) {
      const int col = l / (BM / 16), seg = l % (BM / 16);
      const int r = tile_m + seg * 16, cc = tile_n + col;
      if (r < M && cc < N)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(C + (long)r + (long)cc * ldc));
    }
  }
  uintptr_t base = (reinterpret_cast<uintptr_t>(smem_raw) + 2047) & ~uintptr_t(2047);
  unsigned char* sm = reinterpret_cast<unsigned char*>(base);
  uint64_t* bars = reinterpret_cast<uint64_t*>(sm + STAGES * STAGE_BYTES);
  const uint32_t sm_base = smem_u32(sm);
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + STAGES);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // split K (k_chunk > 0, a multiple of BK): slice blockIdx.z of the k range
  // into its own partial product at C + blockIdx.z * c_zstride
  const int ks = blockIdx.z * k_chunk;
  const int Kz = k_chunk ? min(K - ks, k_chunk) : K;
  C += (long)blockIdx.z * c_zstride;
  const int KT = (Kz + BK - 1) / BK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, CONSUMER_WARPS);
    }
    fence_barrier_init();
  }
  __syncthreads();

  // Producer (thread 0): issue the TMA loads of k-tile kt into stage kt % STAGES.
  auto issue = [&](int kt) {
    int st = kt % STAGES;
    uint32_t fb_ = full0 + 8 * st;
    mbar_arrive_expect_tx(fb_, STAGE_BYTES);
    uint32_t dA = sm_base + st * STAGE_BYTES, dB = dA + A_STAGE_BYTES;
    int k0 = ks + kt * BK;
    if (A_K) {
      tma_load_2d(dA, &mapA, k0, tile_m, fb_);  // box {16 k, 128 m}
    } else {
#pragma unroll
      for (int b = 0; b < BM / 16; ++b) tma_load_2d(dA + b * (BK * 128), &mapA, tile_m + 16 * b, k0, fb_);
    }
    if (B_K) {
      tma_load_2d(dB, &mapB, k0, tile_n, fb_);  // box {16 k, 64 n}
    } else {
#pragma unroll
      for (int b = 0; b < BN / 16; ++b) tma_load_2d(dB + b * (BK * 128), &mapB, tile_n + 16 * b, k0, fb_);
    }
  };
  int issued = 0;
  if (threadIdx.x == 0) {
    prefetch_tmap(&mapA);
    prefetch_tmap(&mapB);
    for (; issued < STAGES - 1 && issued < KT; ++issued) issue(issued);
  }

  // ---------------- consumers ----------------
  const int wm = warp % TC::WM, wn = warp / TC::WM;
  const int g = lane >> 2, t = lane & 3;
  // Fragment row indices within the CTA tile.
  int ra[4];
  uint32_t aoff[4], boff[4];  // shared-memory bases of the fragments
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    ra[f] = A_K ? (wm * 32 + 8 * f + perm8_tab(g)) : (wm * 32 + 16 * (f >> 1) + perm16_tab(f & 1, g));
    const int rb = B_K ? (wn * 32 + 8 * f + perm8_tab(g)) : (wn * 32 + 16 * (f >> 1) + perm16_tab(f & 1, g));
    aoff[f] = A_K ? base_kcontig(ra[f], t) : base_rcontig(ra[f], t);
    boff[f] = A_STAGE_BYTES + (B_K ? base_kcontig(rb, t) : base_rcontig(rb, t));
  }
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  bool ok = true;
  for (int kt = 0; kt < KT; ++kt) {
    int s = kt % STAGES;
    if (threadIdx.x == 0 && issued < KT) {
      // stage of k-tile `issued` was last used by k-tile issued - STAGES
      int ps = issued - STAGES;
      if (ps >= 0 && !mbar_wait(empty0 + 8 * (issued % STAGES), (ps / STAGES) & 1, err, 11)) {
        ok = false;
      } else {
        issue(issued);
        ++issued;
      }
    }
    if (!ok) break;
    if (!mbar_wait(full0 + 8 * s, (kt / STAGES) & 1, err, 12)) { ok = false; break; }
    const uint32_t tS = sm_base + s * STAGE_BYTES;  // 2048-byte aligned
    uint32_t pa[4], pb[4];
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      pa[f] = tS + aoff[f];
      pb[f] = tS + boff[f];
    }
#pragma unroll
    for (int kk = 0; kk < BK / 4; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        a[f] = lds_f64(pa[f] ^ kk_xor<A_K>(kk));
        b[f] = lds_f64(pb[f] ^ kk_xor<B_K>(kk));
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma_884(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    // Release the stage.  Its refill is a TMA write (async proxy) issued as
    // soon as the last warp arrives, so each lane first waits for its own
    // shared-memory reads of the stage to complete (CTA fence) and orders
    // them before async-proxy writes (proxy fence).  Without the fences a
    // warp's last fragment loads could still be in flight when its arrive
    // reached the barrier: with other kernels resident on the SM, a few tiles
    // in 10^8 to 10^9 took one A fragment of one warp (8 rows x 32 columns of
    // C) from the refilled stage.
    __threadfence_block();
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_arrive(empty0 + 8 * s);
  }
  // Every thread reaches this barrier, also after a wait that ran out (each
  // wait is bounded), so a failure cannot leave part of the CTA blocked.
  if (!__syncthreads_and(ok ? 1 : 0)) {
    // drain: thread 0 waits (bounded) for the copies still in flight
    if (threadIdx.x == 0)
      for (int kt = (issued > STAGES ? issued - STAGES : 0); kt < issued; ++kt)
        mbar_wait(full0 + 8 * (kt % STAGES), (kt / STAGES) & 1, nullptr, 0);
    return;
  }

  // ---------------- epilogue ----------------
  // acc[i][j][e] is C(ra[i] of lane group g, column of lane group h = 2t+e
  // of B fragment j).  The accumulators go through shared memory (the stage
  // buffers are free once every warp is past the k-loop) so that C is read
  // and written in coalesced 16-byte pieces along its columns.
  double* sC = reinterpret_cast<double*>(sm);  // BM x BN, ld LDC
  constexpr int LDC = BM + 2;
#pragma unroll
  for (int j = 0; j < 4; ++j)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int h = 2 * t + e;
      const int col = B_K ? (wn * 32 + 8 * j + perm8_tab(h)) : (wn * 32 + 16 * (j >> 1) + perm16_tab(j & 1, h));
#pragma unroll
      for (int i = 0; i < 4; ++i) sC[ra[i] + col * LDC] = acc[i][j][e];
    }
  __syncthreads();
  const bool vec = ((reinterpret_cast<uintptr_t>(C) & 15u) == 0) && ((ldc & 1) == 0);
  // thread -> (row pair, column): BM/2 row pairs x THREADS/(BM/2) columns per pass
  constexpr int RP = BM / 2;
  const int rp = threadIdx.x % RP, c0 = threadIdx.x / RP;
  const int row = tile_m + 2 * rp;
#pragma unroll 4
  for (int cl = c0; cl < BN; cl += THREADS / RP) {
    const int col = tile_n + cl;
    if (col >= N || row >= M) continue;
    double* cp = C + (long)row + (long)col * ldc;
    const double a0 = alpha * sC[2 * rp + cl * LDC], a1 = alpha * sC[2 * rp + 1 + cl * LDC];
    const bool ok0 = mode != GEMM_LOWER || (long)row - (long)col >= diag_off;
    const bool ok1 = (row + 1 < M) && (mode != GEMM_LOWER || (long)row + 1 - (long)col >= diag_off);
    if (vec && ok0 && ok1) {
      double2 v;
      if (beta != 0.0) {
        const double2 c = *reinterpret_cast<const double2*>(cp);
        v.x = fma(beta, c.x, a0);
        v.y = fma(beta, c.y, a1);
      } else {
        v.x = a0;
        v.y = a1;
      }
      *reinterpret_cast<double2*>(cp) = v;
    } else {
      if (ok0) cp[0] = (beta != 0.0) ? fma(beta, cp[0], a0) : a0;
      if (ok1) cp[1] = (beta != 0.0) ? fma(beta, cp[1], a1) : a1;
    }
  }
}

// Fallback for operands the TMA path cannot address (a base or leading
// dimension that is not 16-byte aligned; only small odd-sized blocks at the
// edge of a factorization reach it): 32x32 C tiles, 16-deep k slices in SMEM,
// one thread per C element column pair.
__global__ void __launch_bounds__(256) dgemm_simt_kernel(int ta, int tb, int M, int N, int K, double alpha,
                                                         const double* __restrict__ A, long lda,
                                                         const double* __restrict__ B, long ldb, double beta,
                                                         double* __restrict__ C, long ldc, int mode, long diag_off,
                                                         const int* guard, int guard_limit) {
  if (guard && *((volatile const int*)guard) < guard_limit) return;
  __shared__ double sA[16][33], sB[16][33];
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 32; e += 256) {
      const int kk = e >> 5, r = e & 31;
      const int i = i0 + r, j = j0 + r, k = k0 + kk;
      sA[kk][r] = (i < M && k < K) ? (ta ? A[k + (long)i * lda] : A[i + (long)k * lda]) : 0.0;
      sB[kk][r] = (j < N && k < K) ? (tb ? B[j + (long)k * ldb] : B[k + (long)j * ldb]) : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = fma(sA[kk][tx], sB[kk][ty + 8 * q], acc[q]);
    __syncthreads();
  }
  const int i = i0 + tx;
  if (i >= M) return;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int j = j0 + ty + 8 * q;
    if (j >= N) continue;
    if (mode == GEMM_LOWER && (long)i - (long)j < diag_off) continue;
    double* cp = C + i + (long)j * ldc;
    double v = alpha * acc[q];
    if (beta != 0.0) v = fma(beta, *cp, v);
    *cp = v;
  }
}

// ---------------------------------------------------------------------------
// Host side: tensor maps through the driver entry point (no -lcuda).
// ---------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;
std::once_flag g_encode_once;

bool get_encode() {
  std::call_once(g_encode_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  return g_encode != nullptr;
}

// Map over a column-major rows x cols FP64 matrix; box = {box_rows, box_cols}.
bool make_map(CUtensorMap* map, const double* p, long rows, long cols, long ld, int box_rows,
              int box_cols) {
  if (!get_encode()) return false;
  cuuint64_t dims[2] = {(cuuint64_t)(rows > 0 ? rows : 1), (cuuint64_t)(cols > 0 ? cols : 1)};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 8};
  cuuint32_t box[2] = {(cuuint32_t)box_rows, (cuuint32_t)box_cols};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = g_encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(p), dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                        CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <bool A_K, bool B_K, int BM_, int BN_>
void set_attrs() {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(dgemm_tma_kernel<A_K, B_K, BM_, BN_>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         Tile<BM_, BN_>::SMEM_BYTES);
    done = true;
  }
}
template <bool A_K, bool B_K, int BM_, int BN_ = BN>
void launch(dim3 grid, cudaStream_t st, const CUtensorMap& mA, const CUtensorMap& mB, double* C, long ldc, long m,
            long n, long k, double alpha, double beta, GemmMode mode, long diag_off, int* err, const int* guard,
            int guard_limit, int k_chunk, long c_zstride) {
  set_attrs<A_K, B_K, BM_, BN_>();
  dgemm_tma_kernel<A_K, B_K, BM_, BN_><<<grid, Tile<BM_, BN_>::THREADS, Tile<BM_, BN_>::SMEM_BYTES, st>>>(
      mA, mB, C, ldc, (int)m, (int)n, (int)k, alpha, beta, mode, diag_off, err, guard, guard_limit, k_chunk,
      c_zstride);
}

// C := alpha * sum_z P_z + beta * C over the S partial products of a split-K
// GEMM (P_z at P + z * zs, ld ldp), summed in z order (deterministic).
__global__ void splitk_reduce_kernel(const double* __restrict__ P, long ldp, long zs, int S, int m, int n,
                                     double alpha, double beta, double* __restrict__ C, long ldc) {
  const long total = (long)m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    const double* p = P + i + j * ldp;
    double s = 0.0;
    for (int z = 0; z < S; ++z) s += p[(long)z * zs];
    double* c = C + i + j * ldc;
    *c = beta != 0.0 ? fma(beta, *c, alpha * s) : alpha * s;
  }
}

// Partial products of C = A^T B for small outputs (m, n <= 64) with a long
// k (the W = U1^T B and T12 = U1^T U2 products of the QR panel recursion):
// CTA z multiplies rows [z kc, (z+1) kc) of A (k x m) and B (k x n) with
// FP64 FMAs, 32 rows at a time through shared memory, each of the 256
// threads owning a TB x TB block of the output (16 TB >= m, n), and writes
// its m x n partial to P + z m n; splitk_reduce_warp_kernel adds the
// partials.  A 128 x 64 DMMA tile would spend most of its work on padding
// for these shapes.
constexpr int SK_ROWS = 32;
template <int TB>
__global__ void __launch_bounds__(256) gemm_tn_small_kernel(const double* __restrict__ A, long lda,
                                                            const double* __restrict__ B, long ldb, int m, int n,
                                                            long k, long kc, double* __restrict__ P) {
  constexpr int D = 16 * TB;  // output block covered by the CTA
  __shared__ double As[SK_ROWS][D + 1], Bs[SK_ROWS][D + 1];
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const long k0 = blockIdx.x * kc, k1 = min(k, k0 + kc);
  double acc[TB][TB] = {};
  for (long kb = k0; kb < k1; kb += SK_ROWS) {
    const int rows = (int)(k1 - kb < SK_ROWS ? k1 - kb : SK_ROWS);
    for (int e = tid; e < SK_ROWS * D; e += 256) {
      const int r = e % SK_ROWS, c = e / SK_ROWS;
      As[r][c] = (r < rows && c < m) ? A[(kb + r) + (long)c * lda] : 0.0;
      Bs[r][c] = (r < rows && c < n) ? B[(kb + r) + (long)c * ldb] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int r = 0; r < SK_ROWS; ++r) {
      double av[TB], bv[TB];
#pragma unroll
      for (int t = 0; t < TB; ++t) {
        av[t] = As[r][tx + 16 * t];
        bv[t] = Bs[r][ty + 16 * t];
      }
#pragma unroll
      for (int t = 0; t < TB; ++t)
#pragma unroll
        for (int u = 0; u < TB; ++u) acc[t][u] = fma(av[t], bv[u], acc[t][u]);
    }
    __syncthreads();
  }
  double* Pz = P + (long)blockIdx.x * m * n;
#pragma unroll
  for (int t = 0; t < TB; ++t)
#pragma unroll
    for (int u = 0; u < TB; ++u) {
      const int i = tx + 16 * t, j = ty + 16 * u;
      if (i < m && j < n) Pz[i + (long)j * m] = acc[t][u];
    }
}

// C := alpha sum_z P_z + beta C for S partials of m x n (contiguous, m x n
// apart): one warp per element, lane l adding partials l, l + 32, ..., then
// a fixed shuffle tree (the same order on every run).
__global__ void splitk_reduce_warp_kernel(const double* __restrict__ P, int S, int m, int n, double alpha,
                                          double beta, double* __restrict__ C, long ldc) {
  const long e = ((long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (e >= (long)m * n) return;
  double s = 0.0;
  for (int z = lane; z < S; z += 32) s += P[(long)z * m * n + e];
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
  if (lane == 0) {
    double* c = C + (e % m) + (e / m) * ldc;
    *c = beta != 0.0 ? fma(beta, *c, alpha * s) : alpha * s;
  }
}

// Tile height: 64 (four CTAs per SM hide one another's prologue and
// epilogue best on the rank-128 updates of the factorizations: 26.6 against
// 25.0 TFLOP/s at 16256 x 16256 x 128); FLA_B200_GEMM_BM=128 selects the
// 128-row tile.
int tile_bm() {
  static int bm = 0;
  if (bm == 0) {
    bm = 64;
    if (const char* e = std::getenv("FLA_B200_GEMM_BM"))
      if (std::atoi(e) == 128) bm = 128;
  }
  return bm;
}

}  // namespace

int gemm_f64(cudaStream_t st, bool ta, bool tb, long m, long n, long k, double alpha,
             const double* A, long lda, const double* B, long ldb, double beta, double* C,
             long ldc, GemmMode mode, long diag_off, const int* guard, int guard_limit, long kmax) {
  if (m <= 0 || n <= 0) return FLA_SUCCESS;
  if (k <= 0 || alpha == 0.0) {
    // C := beta*C only; k == 0 never occurs on the factorization path with
    // beta != 1, so only the trivial case is supported here.
    if (beta == 1.0) return FLA_SUCCESS;
  }
  if (ta && !tb && mode == GEMM_FULL && !guard && m <= 64 && n <= 64 && k >= 1024) {
    // slices of 128 rows, at most two per SM
    const int sms = ctx().num_sms;
    long S = std::max<long>(1, std::min<long>(2L * sms, k / 128));
    const long kc = ((k + S - 1) / S + SK_ROWS - 1) / SK_ROWS * SK_ROWS;
    S = (k + kc - 1) / kc;
    double* Pz = (double*)ws_get(st == ctx().side ? WS_SPLITK_SIDE : WS_SPLITK, sizeof(double) * (size_t)(S * m * n));
    if (!Pz) return FLA_FAILURE;
    const int ps = prof_begin(st);
    if (m <= 32 && n <= 32)
      gemm_tn_small_kernel<2><<<(unsigned)S, 256, 0, st>>>(A, lda, B, ldb, (int)m, (int)n, k, kc, Pz);
    else
      gemm_tn_small_kernel<4><<<(unsigned)S, 256, 0, st>>>(A, lda, B, ldb, (int)m, (int)n, k, kc, Pz);
    count_launch();
    splitk_reduce_warp_kernel<<<(unsigned)((m * n * 32 + 255) / 256), 256, 0, st>>>(Pz, (int)S, (int)m, (int)n,
                                                                                   alpha, beta, C, ldc);
    count_launch();
    prof_end(ps, st, PROF_GEMM, 2.0 * (double)m * (double)n * (double)k);
    FB_CK(cudaGetLastError());
    return FLA_SUCCESS;
  }
  if (!tma_ok(A, lda) || !tma_ok(B, ldb)) {
    dim3 g((unsigned)((m + 31) / 32), (unsigned)((n + 31) / 32));
    const int ps = prof_begin(st);
    dgemm_simt_kernel<<<g, 256, 0, st>>>(ta ? 1 : 0, tb ? 1 : 0, (int)m, (int)n, (int)k, alpha, A, lda, B, ldb, beta,
                                         C, ldc, mode, diag_off, guard, guard_limit);
    prof_end(ps, st, PROF_GEMM, 2.0 * (double)m * (double)n * (double)k);
    count_launch();
    FB_CK(cudaGetLastError());
    return FLA_SUCCESS;
  }
  // A operand: op(A) is m x k.  ta = false: stored m x k, m contiguous.
  //            ta = true: stored k x m, k contiguous.
  // B operand: op(B) is k x n.  tb = false: stored k x n, k contiguous.
  //            tb = true: stored n x k, n contiguous.
  CUtensorMap mA, mB;
  // products with at most 32 columns and a long k (the refinement residual
  // R = B - A X): 128 x 32 tiles, k split to fill the GPU
  const bool narrow = (n <= 32 && mode == GEMM_FULL && !guard && k >= 2048);
  const int BMv = narrow ? 128 : tile_bm();
  const int BNv = narrow ? 32 : BN;
  bool okA = ta ? make_map(&mA, A, k, m, lda, 16, BMv) : make_map(&mA, A, m, k, lda, 16, BK);
  bool okB = tb ? make_map(&mB, B, n, k, ldb, 16, BK) : make_map(&mB, B, k, n, ldb, 16, BNv);
  if (!okA || !okB) {
    set_last_error("gemm_f64: cuTensorMapEncodeTiled failed");
    return FLA_FAILURE;
  }
  dim3 grid((unsigned)((m + BMv - 1) / BMv), (unsigned)((n + BNv - 1) / BNv));
  int* err = ctx().d_status + ST_ERROR;
  // Split K when the output has too few tiles to occupy the GPU and K is
  // long (the W = U^T B products of the QR updates and of FLA_Apply_Q_UT):
  // slices of K go to blockIdx.z, each into its own partial product, and one
  // reduction adds them in a fixed order.
  const long tiles = (long)grid.x * grid.y;
  const int sms = ctx().num_sms;
  long S = 1, kc = 0, ldp = 0, zs = 0;
  double* Pz = nullptr;
  const bool capped = mode == GEMM_FULL && !guard && kmax > 0 && k > kmax;
  if (mode == GEMM_FULL && !guard && (((tiles * 2 <= sms || narrow) && k >= 2048) || capped)) {
    S = std::min<long>(std::min<long>(((narrow ? 4L : 2L) * sms + tiles - 1) / tiles, k / 512), 64);
    if (capped) S = std::min<long>(std::max<long>(S, (k + kmax - 1) / kmax), 64);
    if (S > 1) {
      kc = ((k + S - 1) / S + BK - 1) / BK * BK;
      S = (k + kc - 1) / kc;
      ldp = (m + 1) & ~1L;
      zs = ldp * n;
      Pz = (double*)ws_get(st == ctx().side ? WS_SPLITK_SIDE : WS_SPLITK, sizeof(double) * (size_t)(S * zs));
      if (!Pz) return FLA_FAILURE;
      grid.z = (unsigned)S;
    }
  }
  double* Cl = S > 1 ? Pz : C;
  const long ldcl = S > 1 ? ldp : ldc;
  const double al = S > 1 ? 1.0 : alpha, be = S > 1 ? 0.0 : beta;
  const int pslot = prof_begin(st);
#define FB_GEMM_LAUNCH(AK, BK_)                                                                                  \
  (narrow ? launch<AK, BK_, 128, 32>(grid, st, mA, mB, Cl, ldcl, m, n, k, al, be, mode, diag_off, err, guard,   \
                                     guard_limit, (int)kc, zs)                                                  \
   : BMv == 64 ? launch<AK, BK_, 64>(grid, st, mA, mB, Cl, ldcl, m, n, k, al, be, mode, diag_off, err, guard,   \
                                     guard_limit, (int)kc, zs)                                                  \
               : launch<AK, BK_, 128>(grid, st, mA, mB, Cl, ldcl, m, n, k, al, be, mode, diag_off, err, guard,  \
                                      guard_limit, (int)kc, zs))
  if (ta && !tb) FB_GEMM_LAUNCH(true, true);
  else if (ta && tb) FB_GEMM_LAUNCH(true, false);
  else if (!ta && !tb) FB_GEMM_LAUNCH(false, true);
  else FB_GEMM_LAUNCH(false, false);
#undef FB_GEMM_LAUNCH
  if (S > 1) {
    const long total = m * n;
    splitk_reduce_kernel<<<(unsigned)std::min<long>(4L * sms, (total + 255) / 256), 256, 0, st>>>(
        Pz, ldp, zs, (int)S, (int)m, (int)n, alpha, beta, C, ldc);
    count_launch();
  }
  prof_end(pslot, st, PROF_GEMM,
           mode == GEMM_LOWER && m == n ? (double)m * (double)(m + 1) * (double)k
                                        : 2.0 * (double)m * (double)n * (double)k);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

}  // namespace fb

// Direct entry to the engine for tests and benchmarks (device pointers).
extern "C" int FLA_B200_dgemm(int ta, int tb, long m, long n, long k, double alpha,
                              const double* A, long lda, const double* B, long ldb, double beta,
                              double* C, long ldc, int lower_only) {
  if (!fb::ctx().initialized) FLA_Init();
  fb::op_begin(fb::ctx().stream);
  int r = fb::gemm_f64(fb::ctx().stream, ta != 0, tb != 0, m, n, k, alpha, A, lda, B, ldb, beta,
                       C, ldc, lower_only ? fb::GEMM_LOWER : fb::GEMM_FULL, 0, nullptr);
  fb::op_end(fb::ctx().stream);
  if (r != FLA_SUCCESS) return r;
  return fb::sync_all();
}
