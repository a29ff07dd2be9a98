// Low-precision building blocks of the mixed-precision solvers.
//
//   lp_gemm:   C (FP32, column-major) := alpha * A * B^T + beta * C with A
//              (m x k) and B (n x k) held in 16-bit (BF16 or FP16) with k
//              contiguous ("packed"), FP32 accumulation on the tensor cores
//              (mma.sync m16n8k16), a 3-stage cp.async pipeline and ldmatrix
//              fragment loads.  GEMM_LOWER writes only i - j >= diag_off.
//   pack16:    dst(r, kk) := src(r, kk) rounded to 16 bits, dst k-contiguous,
//              src FP32 or FP64 with arbitrary (row, column) strides, through
//              a 32 x 32 shared-memory tile so both sides stay coalesced.
//   convert:   2-D FP64 <-> FP32 copies.
//   sgemm:     FP32 SIMT GEMM (C := alpha op(A) op(B) + beta C), for the
//              correction solves, whose right-hand sides are few.
//
// These replace the single-precision BLAS the reference's dsgesv_/dsposv_
// reach through sgetrf_/spotrf_ (src/map/common/lapacksrc/f2c/dsgesv.c,
// dsposv.c), with the factorization's trailing updates on tensor cores.
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <algorithm>

#include <string>

#include "common.h"
#include "lowprec.h"

namespace fb {

namespace {

constexpr int LBM = 128, LBN = 128, LBK = 32, LSTAGES = 3, LTHREADS = 256;
constexpr int LPAD = 8;                       // 16-bit elements of padding per row
constexpr int LROW = LBK + LPAD;              // 40 halves = 80 bytes per row
constexpr int LSTAGE_HALVES = (LBM + LBN) * LROW;
constexpr int LSMEM = LSTAGES * LSTAGE_HALVES * 2;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, bool pred) {
  const int sz = pred ? 16 : 0;  // zero-fill when out of range
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}
__device__ __forceinline__ void ldmatrix_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2,
                                            uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
template <bool FP16>
__device__ __forceinline__ void mma16816(float* d, const uint32_t* a, const uint32_t* b) {
  if (FP16)
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
  else
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// 8 warps: 2 along m x 4 along n, warp tile 64 x 32 (4 m16 x 4 n8 MMAs).
template <bool FP16>
__global__ void __launch_bounds__(LTHREADS) lp_gemm_kernel(const uint16_t* __restrict__ A, long lda,
                                                           const uint16_t* __restrict__ B, long ldb,
                                                           float* __restrict__ C, long ldc, int M, int N, int K,
                                                           float alpha, float beta, int mode, long diag_off,
                                                           const int* guard, int guard_limit) {
  extern __shared__ __align__(16) uint16_t lsm[];
  if (guard && *((volatile const int*)guard) < guard_limit) return;
  const int tile_m = blockIdx.x * LBM, tile_n = blockIdx.y * LBN;
  if (mode == GEMM_LOWER && (long)(tile_m + LBM - 1) - tile_n < diag_off) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 1, wn = warp >> 1;
  const int KT = (K + LBK - 1) / LBK;

  // stage kt: A rows tile_m.. (LBM x LBK), B rows tile_n.. (LBN x LBK); 16-byte
  // chunks (8 halves): 4 per row, 512 per operand, 2 per thread each
  auto load_stage = [&](int kt) {
    uint16_t* sA = lsm + (kt % LSTAGES) * LSTAGE_HALVES;
    uint16_t* sB = sA + LBM * LROW;
    const int k0 = kt * LBK;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int ch = tid + q * LTHREADS;
      const int r = ch >> 2, kc = (ch & 3) * 8;
      const int gk = k0 + kc;
      const bool okA = (tile_m + r < M) && (gk < K);
      const bool okB = (tile_n + r < N) && (gk < K);
      const uint16_t* srcA = okA ? A + (long)(tile_m + r) * lda + gk : A;
      const uint16_t* srcB = okB ? B + (long)(tile_n + r) * ldb + gk : B;
      cp_async16(smem_addr(sA + r * LROW + kc), srcA, okA);
      cp_async16(smem_addr(sB + r * LROW + kc), srcB, okB);
    }
  };

  float acc[4][4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

#pragma unroll
  for (int s = 0; s < LSTAGES - 1; ++s) {
    if (s < KT) load_stage(s);
    cp_async_commit();
  }
  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<LSTAGES - 2>();
    __syncthreads();
    if (kt + LSTAGES - 1 < KT) load_stage(kt + LSTAGES - 1);
    cp_async_commit();
    const uint16_t* sA = lsm + (kt % LSTAGES) * LSTAGE_HALVES;
    const uint16_t* sB = sA + LBM * LROW;
#pragma unroll
    for (int ks = 0; ks < LBK; ks += 16) {
      uint32_t af[4][4], bf[4][2];
#pragma unroll
      for (int mi = 0; mi < 4; ++mi) {
        const int r = wm * 64 + mi * 16 + (lane & 15);
        const int c = ks + (lane >> 4) * 8;
        ldmatrix_x4(smem_addr(sA + r * LROW + c), af[mi][0], af[mi][1], af[mi][2], af[mi][3]);
      }
#pragma unroll
      for (int nj = 0; nj < 4; nj += 2) {
        const int r = wn * 32 + nj * 8 + (lane & 7) + ((lane >> 4) & 1) * 8;
        const int c = ks + ((lane >> 3) & 1) * 8;
        ldmatrix_x4(smem_addr(sB + r * LROW + c), bf[nj][0], bf[nj][1], bf[nj + 1][0], bf[nj + 1][1]);
      }
#pragma unroll
      for (int mi = 0; mi < 4; ++mi)
#pragma unroll
        for (int nj = 0; nj < 4; ++nj) mma16816<FP16>(acc[mi][nj], af[mi], bf[nj]);
    }
  }
  cp_async_wait<0>();

  // epilogue: acc[mi][nj] = rows (g, g+8) x cols (2t, 2t+1) of a 16 x 8 tile
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mi = 0; mi < 4; ++mi)
#pragma unroll
    for (int nj = 0; nj < 4; ++nj)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int row = tile_m + wm * 64 + mi * 16 + g + (e >> 1) * 8;
        const int col = tile_n + wn * 32 + nj * 8 + 2 * t + (e & 1);
        if (row >= M || col >= N) continue;
        if (mode == GEMM_LOWER && (long)row - col < diag_off) continue;
        float* cp = C + row + (long)col * ldc;
        float v = alpha * acc[mi][nj][e];
        if (beta != 0.f) v = fmaf(beta, *cp, v);
        *cp = v;
      }
}

// dst[r * ldd + kk] := src(r, kk), src(r, kk) at src[r * rs + kk * cs]
// MODE 0: BF16; 1: FP16; 2: FP16 hi plane at dst and lo plane (the
// remainder times 2^11) at dst + plane.
template <typename TS, int MODE>
__global__ void __launch_bounds__(256) pack16_kernel(const TS* __restrict__ src, long rs, long cs,
                                                     uint16_t* __restrict__ dst, long ldd, int rows, int kdim,
                                                     float scale, long plane) {
  __shared__ float tile[32][33];
  const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
  // read: coalesce along whichever index is contiguous in the source
  const bool rfast = (rs == 1);
  for (int yy = ty; yy < 32; yy += 8) {
    const int r = r0 + (rfast ? tx : yy), k = k0 + (rfast ? yy : tx);
    float v = 0.f;
    if (r < rows && k < kdim) v = (float)src[(long)r * rs + (long)k * cs] * scale;
    if (rfast) tile[yy][tx] = v; else tile[tx][yy] = v;   // tile[k - k0][r - r0]
  }
  __syncthreads();
  // write: kk fastest; columns kdim .. (kdim rounded up to 8) are written as
  // zeros, so 16-byte loads of the last chunk read no stale values
  const int kpad = (kdim + 7) & ~7;
  for (int yy = ty; yy < 32; yy += 8) {
    const int r = r0 + yy, k = k0 + tx;
    if (r < rows && k < kpad) {
      const float v = tile[tx][yy];
      uint16_t h;
      if (MODE >= 1) {
        __half hv = __float2half_rn(v);
        h = *reinterpret_cast<uint16_t*>(&hv);
        if (MODE == 2) {
          __half lv = __float2half_rn((v - __half2float(hv)) * 2048.0f);
          dst[plane + (long)r * ldd + k] = *reinterpret_cast<uint16_t*>(&lv);
        }
      } else {
        __nv_bfloat16 bv = __float2bfloat16_rn(v);
        h = *reinterpret_cast<uint16_t*>(&bv);
      }
      dst[(long)r * ldd + k] = h;
    }
  }
}

template <typename TD, typename TS>
__global__ void convert2d_kernel(const TS* __restrict__ src, long lds, TD* __restrict__ dst, long ldd, int m,
                                 int n) {
  const long total = (long)m * n;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long i = e % m, j = e / m;
    dst[i + j * ldd] = (TD)src[i + j * lds];
  }
}

// FP32 SIMT GEMM: 64 x 64 tiles, 256 threads, 4 x 4 outputs per thread.
__global__ void __launch_bounds__(256) sgemm_kernel(int ta, int tb, int M, int N, int K, float alpha,
                                                    const float* __restrict__ A, long lda,
                                                    const float* __restrict__ B, long ldb, float beta,
                                                    float* __restrict__ C, long ldc) {
  __shared__ float sA[16][64 + 4], sB[16][64 + 4];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = blockIdx.x * 64, j0 = blockIdx.y * 64;
  float acc[4][4] = {};
  for (int k0 = 0; k0 < K; k0 += 16) {
    for (int e = threadIdx.x; e < 16 * 64; e += 256) {
      const int kk = e >> 6, r = e & 63;
      const int i = i0 + r, j = j0 + r, k = k0 + kk;
      sA[kk][r] = (i < M && k < K) ? (ta ? A[k + (long)i * lda] : A[i + (long)k * lda]) : 0.f;
      sB[kk][r] = (j < N && k < K) ? (tb ? B[j + (long)k * ldb] : B[k + (long)j * ldb]) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < 16; ++kk) {
      float a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = sA[kk][tx + 16 * q];
        b[q] = sB[kk][ty + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = fmaf(a[p], b[q], acc[p][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = i0 + tx + 16 * p, j = j0 + ty + 16 * q;
      if (i < M && j < N) {
        float* cp = C + i + (long)j * ldc;
        float v = alpha * acc[p][q];
        if (beta != 0.f) v = fmaf(beta, *cp, v);
        *cp = v;
      }
    }
}


// ---------------------------------------------------------------------------
// FP32-accurate tensor-core GEMM ("3xTF32"): every FP32 operand x is split
// into hi = tf32(x) and lo = tf32(x - hi) (packed by pack_tf32x3), and
// A B^T is accumulated as Ahi Bhi^T + Ahi Blo^T + Alo Bhi^T with
// mma.sync m16n8k8 TF32 -> FP32, about 2^-21 relative per product: the
// low-precision factorization then carries nearly FP32 accuracy, which the
// refinement needs for condition numbers around 1e5 and beyond.
// Tile 128 x 64, k 16 per stage, 3 stages, 8 warps (4 along m x 2 along n),
// warp tile 32 x 32.
constexpr int TBM = 128, TBN = 64, TBK = 16, TSTAGES = 3;
constexpr int TROW = TBK + 4;  // floats per shared row (80 bytes: conflict-free ldmatrix)
constexpr int TSTAGE_FLOATS = 2 * (TBM + TBN) * TROW;  // hi and lo planes
constexpr int TSMEM = TSTAGES * TSTAGE_FLOATS * 4;

__device__ __forceinline__ void mma1688_tf32(float* d, const uint32_t* a, const uint32_t* b) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A: hi plane at A, lo plane at A + aplane (rows of k floats, ld lda);
// likewise B.
__global__ void __launch_bounds__(LTHREADS, 2) lp_gemm_tf32x3_kernel(
    const float* __restrict__ A, long lda, long aplane, const float* __restrict__ B, long ldb, long bplane,
    float* __restrict__ C, long ldc, int M, int N, int K, float alpha, float beta, int mode, long diag_off,
    const int* guard, int guard_limit) {
  extern __shared__ __align__(16) float tsm[];
  if (guard && *((volatile const int*)guard) < guard_limit) return;
  const int tile_m = blockIdx.x * TBM, tile_n = blockIdx.y * TBN;
  if (mode == GEMM_LOWER && (long)(tile_m + TBM - 1) - tile_n < diag_off) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = warp & 3, wn = warp >> 2;
  const int KT = (K + TBK - 1) / TBK;
  // stage layout: Ahi [TBM][TROW], Alo, Bhi [TBN][TROW], Blo
  auto load_stage = [&](int kt) {
    float* sAh = tsm + (kt % TSTAGES) * TSTAGE_FLOATS;
    float* sAl = sAh + TBM * TROW;
    float* sBh = sAl + TBM * TROW;
    float* sBl = sBh + TBN * TROW;
    const int k0 = kt * TBK;
    // A: 128 rows x 4 chunks of 16 bytes per plane = 512 chunks, 2 per thread
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int ch = tid + q * LTHREADS;
      const int r = ch >> 2, kc = (ch & 3) * 4;
      const bool ok = (tile_m + r < M) && (k0 + kc < K);
      const float* src = ok ? A + (long)(tile_m + r) * lda + k0 + kc : A;
      cp_async16(smem_addr(sAh + r * TROW + kc), src, ok);
      cp_async16(smem_addr(sAl + r * TROW + kc), ok ? src + aplane : A, ok);
    }
    // B: 64 rows x 4 chunks = 256 chunks, 1 per thread
    {
      const int r = tid >> 2, kc = (tid & 3) * 4;
      const bool ok = (tile_n + r < N) && (k0 + kc < K);
      const float* src = ok ? B + (long)(tile_n + r) * ldb + k0 + kc : B;
      cp_async16(smem_addr(sBh + r * TROW + kc), src, ok);
      cp_async16(smem_addr(sBl + r * TROW + kc), ok ? src + bplane : B, ok);
    }
  };
  float acc[2][4][4];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;
#pragma unroll
  for (int s = 0; s < TSTAGES - 1; ++s) {
    if (s < KT) load_stage(s);
    cp_async_commit();
  }
  for (int kt = 0; kt < KT; ++kt) {
    cp_async_wait<TSTAGES - 2>();
    __syncthreads();
    if (kt + TSTAGES - 1 < KT) load_stage(kt + TSTAGES - 1);
    cp_async_commit();
    const float* sAh = tsm + (kt % TSTAGES) * TSTAGE_FLOATS;
    const float* sAl = sAh + TBM * TROW;
    const float* sBh = sAl + TBM * TROW;
    const float* sBl = sBh + TBN * TROW;
#pragma unroll
    for (int ks = 0; ks < TBK; ks += 8) {
      uint32_t ah[2][4], al[2][4], bh[4][2], bl[4][2];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi) {
        const int r = wm * 32 + mi * 16 + (lane & 15);
        const int c = ks + (lane >> 4) * 4;
        ldmatrix_x4(smem_addr(sAh + r * TROW + c), ah[mi][0], ah[mi][1], ah[mi][2], ah[mi][3]);
        ldmatrix_x4(smem_addr(sAl + r * TROW + c), al[mi][0], al[mi][1], al[mi][2], al[mi][3]);
      }
#pragma unroll
      for (int nj = 0; nj < 4; nj += 2) {
        const int r = wn * 32 + nj * 8 + (lane & 7) + ((lane >> 4) & 1) * 8;
        const int c = ks + ((lane >> 3) & 1) * 4;
        ldmatrix_x4(smem_addr(sBh + r * TROW + c), bh[nj][0], bh[nj][1], bh[nj + 1][0], bh[nj + 1][1]);
        ldmatrix_x4(smem_addr(sBl + r * TROW + c), bl[nj][0], bl[nj][1], bl[nj + 1][0], bl[nj + 1][1]);
      }
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
#pragma unroll
        for (int nj = 0; nj < 4; ++nj) {
          mma1688_tf32(acc[mi][nj], al[mi], bh[nj]);
          mma1688_tf32(acc[mi][nj], ah[mi], bl[nj]);
          mma1688_tf32(acc[mi][nj], ah[mi], bh[nj]);
        }
    }
  }
  cp_async_wait<0>();
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int mi = 0; mi < 2; ++mi)
#pragma unroll
    for (int nj = 0; nj < 4; ++nj)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const int row = tile_m + wm * 32 + mi * 16 + g + (e >> 1) * 8;
        const int col = tile_n + wn * 32 + nj * 8 + 2 * t + (e & 1);
        if (row >= M || col >= N) continue;
        if (mode == GEMM_LOWER && (long)row - col < diag_off) continue;
        float* cp = C + row + (long)col * ldc;
        float v = alpha * acc[mi][nj][e];
        if (beta != 0.f) v = fmaf(beta, *cp, v);
        *cp = v;
      }
}

__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// hi[r * ldd + kk] = tf32(v), lo (= hi + plane) = tf32(v - hi) for
// v = scale * src(r, kk); columns kdim .. round4(kdim) are zeroed.
template <typename TS>
__global__ void __launch_bounds__(256) pack_tf32x3_kernel(const TS* __restrict__ src, long rs, long cs,
                                                          float* __restrict__ dst, long ldd, long plane, int rows,
                                                          int kdim, float scale) {
  __shared__ float tile[32][33];
  const int r0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const bool rfast = (rs == 1);
  for (int yy = ty; yy < 32; yy += 8) {
    const int r = r0 + (rfast ? tx : yy), k = k0 + (rfast ? yy : tx);
    float v = 0.f;
    if (r < rows && k < kdim) v = (float)src[(long)r * rs + (long)k * cs] * scale;
    if (rfast) tile[yy][tx] = v; else tile[tx][yy] = v;
  }
  __syncthreads();
  const int kpad = (kdim + 3) & ~3;
  for (int yy = ty; yy < 32; yy += 8) {
    const int r = r0 + yy, k = k0 + tx;
    if (r < rows && k < kpad) {
      const float v = tile[tx][yy];
      const float hi = tf32_round(v);
      dst[(long)r * ldd + k] = hi;
      dst[plane + (long)r * ldd + k] = tf32_round(v - hi);
    }
  }
}

bool g_lp_attr = false;
void lp_attrs() {
  if (g_lp_attr) return;
  cudaFuncSetAttribute(lp_gemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, LSMEM);
  cudaFuncSetAttribute(lp_gemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, LSMEM);
  cudaFuncSetAttribute(lp_gemm_tf32x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, TSMEM);
  g_lp_attr = true;
}

}  // namespace

int lp_gemm(cudaStream_t st, LowPrec prec, long m, long n, long k, float alpha, const uint16_t* A, long lda,
            const uint16_t* B, long ldb, float beta, float* C, long ldc, GemmMode mode, long diag_off,
            const int* guard, int guard_limit, long aplane, long bplane) {
  if (m <= 0 || n <= 0) return FLA_SUCCESS;
  if (prec == LP_TF32X3) {
    // A and B are float hi planes (ld counted in floats); the lo plane of
    // each follows at the operand's plane offset (see pack_operand).
    lp_attrs();
    const float* fa = reinterpret_cast<const float*>(A);
    const float* fb_ = reinterpret_cast<const float*>(B);
    if ((lda % 4) || (ldb % 4) || ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)) {
      set_last_error("lp_gemm: packed operands need 16-byte aligned rows");
      return FLA_FAILURE;
    }
    dim3 grid((unsigned)((m + TBM - 1) / TBM), (unsigned)((n + TBN - 1) / TBN));
    const int ps = prof_begin(st);
    lp_gemm_tf32x3_kernel<<<grid, LTHREADS, TSMEM, st>>>(fa, lda, aplane, fb_, ldb, bplane, C,
                                                         ldc, (int)m, (int)n, (int)k, alpha, beta, mode, diag_off,
                                                         guard, guard_limit);
    prof_end(ps, st, PROF_GEMM,
             mode == GEMM_LOWER && m == n ? (double)m * (double)(m + 1) * (double)k : 2.0 * m * (double)n * k);
    count_launch();
    FB_CK(cudaGetLastError());
    return FLA_SUCCESS;
  }
  if ((lda % 8) || (ldb % 8) || ((reinterpret_cast<uintptr_t>(A) | reinterpret_cast<uintptr_t>(B)) & 15)) {
    set_last_error("lp_gemm: packed operands need 16-byte aligned rows");
    return FLA_FAILURE;
  }
  static const bool use_mma_sync = [] {
    const char* e = std::getenv("FLA_B200_LP_GEMM");
    return e && std::string(e) == "mma";
  }();
  if (prec == LP_FP16X3 || (!use_mma_sync && k > 0))
    return tc_gemm16(st, prec == LP_BF16, prec == LP_FP16X3, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, mode,
                     diag_off, guard, guard_limit, aplane, bplane);
  lp_attrs();
  dim3 grid((unsigned)((m + LBM - 1) / LBM), (unsigned)((n + LBN - 1) / LBN));
  const int ps = prof_begin(st);
  if (prec == LP_FP16)
    lp_gemm_kernel<true><<<grid, LTHREADS, LSMEM, st>>>(A, lda, B, ldb, C, ldc, (int)m, (int)n, (int)k, alpha, beta,
                                                        mode, diag_off, guard, guard_limit);
  else
    lp_gemm_kernel<false><<<grid, LTHREADS, LSMEM, st>>>(A, lda, B, ldb, C, ldc, (int)m, (int)n, (int)k, alpha,
                                                         beta, mode, diag_off, guard, guard_limit);
  prof_end(ps, st, PROF_GEMM,
           mode == GEMM_LOWER && m == n ? (double)m * (double)(m + 1) * (double)k : 2.0 * m * (double)n * k);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

template <typename TS>
int pack16(cudaStream_t st, LowPrec prec, const TS* src, long rs, long cs, uint16_t* dst, long ldd, long rows,
           long kdim, float scale, long plane) {
  if (rows <= 0 || kdim <= 0) return FLA_SUCCESS;
  if (prec == LP_TF32X3) {
    dim3 g((unsigned)((rows + 31) / 32), (unsigned)((((kdim + 3) & ~3L) + 31) / 32));
    pack_tf32x3_kernel<TS><<<g, 256, 0, st>>>(src, rs, cs, reinterpret_cast<float*>(dst), ldd, plane,
                                              (int)rows, (int)kdim, scale);
    count_launch();
    FB_CK(cudaGetLastError());
    return FLA_SUCCESS;
  }
  dim3 grid((unsigned)((rows + 31) / 32), (unsigned)((((kdim + 7) & ~7L) + 31) / 32));
  if (prec == LP_FP16X3)
    pack16_kernel<TS, 2><<<grid, 256, 0, st>>>(src, rs, cs, dst, ldd, (int)rows, (int)kdim, scale, plane);
  else if (prec == LP_FP16)
    pack16_kernel<TS, 1><<<grid, 256, 0, st>>>(src, rs, cs, dst, ldd, (int)rows, (int)kdim, scale, 0);
  else
    pack16_kernel<TS, 0><<<grid, 256, 0, st>>>(src, rs, cs, dst, ldd, (int)rows, (int)kdim, scale, 0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}
template int pack16<float>(cudaStream_t, LowPrec, const float*, long, long, uint16_t*, long, long, long, float, long);
template int pack16<double>(cudaStream_t, LowPrec, const double*, long, long, uint16_t*, long, long, long, float,
                            long);

template <typename TD, typename TS>
int convert2d(cudaStream_t st, const TS* src, long lds, TD* dst, long ldd, long m, long n) {
  if (m <= 0 || n <= 0) return FLA_SUCCESS;
  const int blocks = (int)std::min<long>(4096, (m * n + 255) / 256);
  convert2d_kernel<TD, TS><<<blocks, 256, 0, st>>>(src, lds, dst, ldd, (int)m, (int)n);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}
template int convert2d<float, double>(cudaStream_t, const double*, long, float*, long, long, long);
template int convert2d<double, float>(cudaStream_t, const float*, long, double*, long, long, long);

int sgemm(cudaStream_t st, bool ta, bool tb, long m, long n, long k, float alpha, const float* A, long lda,
          const float* B, long ldb, float beta, float* C, long ldc) {
  if (m <= 0 || n <= 0) return FLA_SUCCESS;
  dim3 grid((unsigned)((m + 63) / 64), (unsigned)((n + 63) / 64));
  const int ps = prof_begin(st);
  sgemm_kernel<<<grid, 256, 0, st>>>(ta ? 1 : 0, tb ? 1 : 0, (int)m, (int)n, (int)k, alpha, A, lda, B, ldb, beta, C,
                                     ldc);
  prof_end(ps, st, PROF_OTHER, 2.0 * m * (double)n * k);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

}  // namespace fb

// Direct entry to the 16-bit tensor-core GEMM for tests: C (FP32, ld ldc)
// := alpha * A * B^T + beta * C with A (m x k) and B (n x k) given in FP32
// column-major and packed here.  prec: 0 = BF16, 1 = FP16, 2 = 3xTF32,
// 3 = split FP16 (FP32-accurate).
extern "C" int FLA_B200_lp_gemm(int prec, long m, long n, long k, float alpha, const float* A, long lda,
                                const float* B, long ldb, float beta, float* C, long ldc) {
  using namespace fb;
  if (!ctx().initialized) FLA_Init();
  const LowPrec p = prec == 3 ? LP_FP16X3 : prec == 2 ? LP_TF32X3 : (prec == 1 ? LP_FP16 : LP_BF16);
  const long kp = (k + 7) & ~7L;
  uint16_t* pa = (uint16_t*)ws_get(WS_MISC, lp_packed_bytes(p, m, kp));
  uint16_t* pb = (uint16_t*)ws_get(WS_MISC2, lp_packed_bytes(p, n, kp));
  if (!pa || !pb) return FLA_FAILURE;
  cudaStream_t st = ctx().stream;
  op_begin(st);
  const long pla = kp * std::max<long>(1, m), plb = kp * std::max<long>(1, n);
  if (pack16<float>(st, p, A, 1, lda, pa, kp, m, k, 1.f, pla) != FLA_SUCCESS) return FLA_FAILURE;
  if (pack16<float>(st, p, B, 1, ldb, pb, kp, n, k, 1.f, plb) != FLA_SUCCESS) return FLA_FAILURE;
  if (lp_gemm(st, p, m, n, k, alpha, pa, kp, pb, kp, beta, C, ldc, GEMM_FULL, 0, nullptr, 0x7fffffff, pla, plb) !=
      FLA_SUCCESS)
    return FLA_FAILURE;
  op_end(st);
  return sync_all();
}
