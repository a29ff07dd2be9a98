// 16-bit GEMM on the fifth-generation tensor cores (tcgen05) for the
// mixed-precision factorizations:
//
//   C (FP32, column-major) := alpha * A * B^T + beta * C
//   A: m x k, B: n x k, FP16 or BF16, k contiguous (row r at A + r * lda)
//
// Persistent kernel, at most one CTA per SM, looping over 128 x TN output
// tiles (TN = 128), six warps with fixed roles:
//   * warp 0 (one thread) streams the k-blocks of A (128 x 64) and B (TN x 64)
//     with 2D TMA loads (128-byte swizzle) into an S-stage ring of shared
//     memory buffers, each stage completing an mbarrier transaction count;
//   * warp 1 (one thread) issues tcgen05.mma (M = 128, N = TN, K = 16, FP32
//     accumulate) into one of two TMEM accumulators, releases each stage with
//     tcgen05.commit on the stage's "empty" mbarrier, and after a tile's last
//     k-block commits the accumulator's "full" mbarrier;
//   * warps 2-9 drain the accumulator (warp w reads TMEM lanes 32 (w mod 4) +
//     0..31, i.e. tile rows, and half of the tile's columns) with
//     tcgen05.ld, update C column by column (32 consecutive rows per store:
//     coalesced) and arrive on the accumulator's "empty" mbarrier; eight
//     warps keep enough loads of C in flight to run at the memory's pace.
// With two accumulators the epilogue of one tile (the FP32 C read and write)
// runs while the MMAs of the next tile proceed.
// The shared-memory operand descriptors describe K-major tiles with the
// 128-byte swizzle (rows of 128 bytes, 8-row atoms 1024 bytes apart); the
// K = 16 sub-steps of a 64-wide k-block advance the start address by 32
// bytes inside the swizzle atom.
//
// Every mbarrier wait is bounded (kWaitLimitNs); on expiry the kernel
// records the error in the status block and raises a CTA-wide abort flag
// that every role checks: the producer waits (bounded) for its own TMA loads
// still in flight, nothing more is stored, the TMEM is freed and the CTA
// returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "common.h"
#include "dev_util.cuh"
#include "lowprec.h"

namespace fb {

namespace {

constexpr int TC_BM = 128;
constexpr int TC_BK = 64;  // 64 16-bit values = 128 bytes = one swizzle row
constexpr int TC_THREADS = 320;  // producer, MMA, eight epilogue warps
constexpr int TC_EPI_WARPS = 8;

template <int TN, int STAGES, bool SPLIT>
struct TcCfg {
  static constexpr uint32_t A_BYTES = TC_BM * TC_BK * 2;  // one plane
  static constexpr uint32_t B_BYTES = TN * TC_BK * 2;
  static constexpr uint32_t NPLANE = SPLIT ? 2 : 1;
  static constexpr uint32_t STAGE_BYTES = NPLANE * (A_BYTES + B_BYTES);
  static constexpr uint32_t BAR_OFF = STAGES * STAGE_BYTES;
  // stages, then 2*STAGES + 5 mbarriers (stage full / empty, accumulator
  // full / empty, final) and the TMEM address slot, plus slack to align the ring
  // to 1024 bytes (the swizzle atom)
  static constexpr uint32_t SMEM_BYTES = BAR_OFF + 8 * (2 * STAGES + 5) + 16 + 1024;
  // FP32 columns of one accumulator (TN wide; a pair for the split form) and
  // of the two accumulators the CTA allocates (a power of 2 <= 512)
  static constexpr uint32_t ACC_COLS = NPLANE * TN;
  static constexpr uint32_t TMEM_COLS = 2 * ACC_COLS;
};

// K-major, 128-byte swizzle, 8-row atoms 1024 bytes apart (SBO), version 1.
__device__ __forceinline__ uint64_t umma_desc_k_sw128(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(1024u >> 4) << 32) |
         ((uint64_t)1u << 46) | ((uint64_t)2u << 61);
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                           uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tc_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Bounded mbarrier wait that also gives up as soon as another role of the
// CTA has raised the abort flag; false on timeout or abort (a timeout sets
// the flag and records `code` in *err).
__device__ __forceinline__ bool tc_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* err,
                                        int code) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    for (int i = 0; i < 32; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
    if (globaltimer_ns() - t0 > kWaitLimitNs) {
      atomicExch(err, code);
      *abort_flag = 1;
      return false;
    }
  }
}

template <int TN, int STAGES, bool SPLIT>
__global__ void __launch_bounds__(TC_THREADS, 1)
    tc_gemm16_kernel(const __grid_constant__ CUtensorMap mA, const __grid_constant__ CUtensorMap mB,
                     const __grid_constant__ CUtensorMap mAl, const __grid_constant__ CUtensorMap mBl, float* C,
                     long ldc, int M, int N, int K, float alpha, float beta, uint32_t idesc, int lower,
                     long diag_off, const int* guard, int guard_limit, int* err) {
  using Cfg = TcCfg<TN, STAGES, SPLIT>;
  extern __shared__ uint8_t smem_raw[];
  if (guard && *((volatile const int*)guard) < guard_limit) return;
  const int tiles_m = (M + TC_BM - 1) / TC_BM, tiles_n = (N + TN - 1) / TN;
  const int ntiles = tiles_m * tiles_n;
  const int nk = (K + TC_BK - 1) / TC_BK;
  // tile t: rows tm * 128.., columns tn * TN..; tiles entirely outside the
  // written triangle are skipped by every role alike
  auto tile_of = [&](int t, int& m0, int& n0) -> bool {
    m0 = (t % tiles_m) * TC_BM;
    n0 = (t / tiles_m) * TN;
    return !lower || (long)(m0 + TC_BM - 1) - (long)n0 >= diag_off;
  };

  const uint32_t raw = smem_u32(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t* gbase = smem_raw + (base - raw);
  // full[s] = bar0 + 8s, empty[s] = bar0 + 8(S+s), accf[b] = bar0 + 8(2S+b),
  // acce[b] = bar0 + 8(2S+2+b)
  const uint32_t bar0 = base + Cfg::BAR_OFF;
  auto full = [&](int s_) { return bar0 + 8u * s_; };
  auto empty = [&](int s_) { return bar0 + 8u * (STAGES + s_); };
  auto accf = [&](int b_) { return bar0 + 8u * (2 * STAGES + b_); };
  auto acce = [&](int b_) { return bar0 + 8u * (2 * STAGES + 2 + b_); };
  const uint32_t fin = bar0 + 8u * (2 * STAGES + 4);  // every MMA of the CTA done
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(gbase + Cfg::BAR_OFF + 8 * (2 * STAGES + 5));
  __shared__ int s_abort;
  volatile int* abort_flag = &s_abort;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s_ = 0; s_ < STAGES; ++s_) {
      mbar_init(full(s_), 1);
      mbar_init(empty(s_), 1);
    }
    for (int b_ = 0; b_ < 2; ++b_) {
      mbar_init(accf(b_), 1);
      mbar_init(acce(b_), TC_EPI_WARPS);  // one arrive per epilogue warp
    }
    mbar_init(fin, 1);
    fence_barrier_init();
    s_abort = 0;
    prefetch_tmap(&mA);
    prefetch_tmap(&mB);
    if (SPLIT) {
      prefetch_tmap(&mAl);
      prefetch_tmap(&mBl);
    }
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(Cfg::TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      // ---- TMA producer
      int kstep = 0;
      for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x) {
        int m0, n0;
        if (!tile_of(t, m0, n0)) continue;
        for (int kb = 0; kb < nk; ++kb, ++kstep) {
          const int s_ = kstep % STAGES, u = kstep / STAGES;
          if (u > 0 && !tc_wait(empty(s_), (uint32_t)((u - 1) & 1), abort_flag, err, 41)) break;
          if (*abort_flag) break;
          const uint32_t sa = base + s_ * Cfg::STAGE_BYTES, sb = sa + Cfg::A_BYTES;
          mbar_arrive_expect_tx(full(s_), Cfg::STAGE_BYTES);
          tma_load_2d(sa, &mA, kb * TC_BK, m0, full(s_));
          tma_load_2d(sb, &mB, kb * TC_BK, n0, full(s_));
          if (SPLIT) {
            const uint32_t sal = sb + Cfg::B_BYTES, sbl = sal + Cfg::A_BYTES;
            tma_load_2d(sal, &mAl, kb * TC_BK, m0, full(s_));
            tma_load_2d(sbl, &mBl, kb * TC_BK, n0, full(s_));
          }
        }
      }
      // drain: the last load issued into each stage has landed (bounded)
      for (int q = (kstep > STAGES ? kstep - STAGES : 0); q < kstep; ++q)
        mbar_wait(full(q % STAGES), (uint32_t)((q / STAGES) & 1), err, 42);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---- MMA issuer
      int kstep = 0, lt = 0;
      for (int t = blockIdx.x; t < ntiles && !*abort_flag; t += gridDim.x) {
        int m0, n0;
        if (!tile_of(t, m0, n0)) continue;
        const int b_ = lt & 1, ua = lt >> 1;
        // the epilogue has drained this accumulator's previous tile
        if (ua > 0 && !tc_wait(acce(b_), (uint32_t)((ua - 1) & 1), abort_flag, err, 45)) break;
        if (*abort_flag) break;
        tc_fence_after();
        const uint32_t dacc = tmem + (uint32_t)b_ * Cfg::ACC_COLS;
        for (int kb = 0; kb < nk; ++kb, ++kstep) {
          const int s_ = kstep % STAGES, u = kstep / STAGES;
          if (!tc_wait(full(s_), (uint32_t)(u & 1), abort_flag, err, 43)) break;
          tc_fence_after();
          const uint32_t sa = base + s_ * Cfg::STAGE_BYTES, sb = sa + Cfg::A_BYTES;
#pragma unroll
          for (int k = 0; k < TC_BK / 16; ++k) {
            const uint32_t acc = (kb > 0 || k > 0) ? 1u : 0u;
            tc_mma_f16(dacc, umma_desc_k_sw128(sa + 32 * k), umma_desc_k_sw128(sb + 32 * k), idesc, acc);
            if (SPLIT) {
              const uint32_t sal = sb + Cfg::B_BYTES, sbl = sal + Cfg::A_BYTES;
              tc_mma_f16(dacc + TN, umma_desc_k_sw128(sa + 32 * k), umma_desc_k_sw128(sbl + 32 * k), idesc, acc);
              tc_mma_f16(dacc + TN, umma_desc_k_sw128(sal + 32 * k), umma_desc_k_sw128(sb + 32 * k), idesc, 1u);
            }
          }
          tc_commit(empty(s_));  // stage free once these MMAs are done
        }
        if (*abort_flag) break;
        tc_commit(accf(b_));  // the tile's accumulator is complete
        ++lt;
      }
      // nothing of this CTA's may still run on the tensor cores when its
      // TMEM is freed
      if (kstep > 0) {
        tc_commit(fin);
        mbar_wait(fin, 0, err, 46);
      }
    }
  } else {
    // ---- epilogue: warps 2-9, warp w owns TMEM lanes 32 (w mod 4) + 0..31
    // and columns [h TN/2, (h+1) TN/2) of the tile, h = (w - 2) / 4
    const int q = warp & 3, h = (warp - 2) >> 2;
    int lt = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      int m0, n0;
      if (!tile_of(t, m0, n0)) continue;
      const int b_ = lt & 1, ua = lt >> 1;
      const bool got = tc_wait(accf(b_), (uint32_t)(ua & 1), abort_flag, err, 44);
      tc_fence_after();
      if (!__all_sync(0xffffffffu, (got && !*abort_flag) ? 1 : 0)) break;
      const int row = m0 + q * 32 + lane;
      const uint32_t tl = tmem + (uint32_t)b_ * Cfg::ACC_COLS + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
      for (int c0 = h * (TN / 2); c0 < (h + 1) * (TN / 2) && n0 + c0 < N; c0 += 32) {
        float v[32];
        tc_ld32(tl + c0, v);
        if (SPLIT) {
          float v2[32];
          tc_ld32(tl + TN + c0, v2);
#pragma unroll
          for (int j = 0; j < 32; ++j) v[j] = fmaf(v2[j], 1.0f / 2048.0f, v[j]);
        }
        if (row < M) {
          // all 32 loads of C first (a store between them would serialize
          // each load on its memory latency), then the stores
          bool ok[32];
          float cv[32];
#pragma unroll
          for (int j = 0; j < 32; ++j) {
            const int col = n0 + c0 + j;
            ok[j] = col < N && (!lower || (long)row - (long)col >= diag_off);
            cv[j] = (ok[j] && beta != 0.f) ? __ldcs(C + row + (long)col * ldc) : 0.f;
          }
#pragma unroll
          for (int j = 0; j < 32; ++j)
            if (ok[j]) __stcs(C + row + (long)(n0 + c0 + j) * ldc, fmaf(alpha, v[j], beta * cv[j]));
        }
      }
      // accumulator drained: the MMA warp may reuse it
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acce(b_));
      ++lt;
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(Cfg::TMEM_COLS)
                 : "memory");
  }
}

PFN_cuTensorMapEncodeTiled_v12000 g_enc16 = nullptr;
std::once_flag g_enc16_once;

bool get_enc16() {
  std::call_once(g_enc16_once, [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_enc16 = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  });
  return g_enc16 != nullptr;
}

// rows x kdim 16-bit operand, k contiguous (row pitch ld elements), box of
// box_rows rows x 64 k-values, 128-byte swizzle, zero fill out of bounds.
bool make_map16(CUtensorMap* map, const uint16_t* p, long rows, long kdim, long ld, int box_rows) {
  if (!get_enc16()) return false;
  cuuint64_t dims[2] = {(cuuint64_t)(kdim > 0 ? kdim : 1), (cuuint64_t)(rows > 0 ? rows : 1)};
  cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  cuuint32_t box[2] = {(cuuint32_t)TC_BK, (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  return g_enc16(map, CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<uint16_t*>(p), dims, strides, box, estr,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

constexpr int TC_TN = 128;
constexpr int TC_STAGES = 3;

template <bool SPLIT>
void tc_set_attr() {
  static bool done = false;
  if (!done) {
    cudaFuncSetAttribute(tc_gemm16_kernel<TC_TN, TC_STAGES, SPLIT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TcCfg<TC_TN, TC_STAGES, SPLIT>::SMEM_BYTES);
    done = true;
  }
}

}  // namespace

// C := alpha A B^T + beta C on the tcgen05 tensor cores (see the top of
// this file); A, B packed 16-bit, k contiguous, lda / ldb multiples of 8 and
// 16-byte aligned bases (the TMA rules).  split: FP16 hi planes at A / B and
// lo planes (scaled by 2^11) aplane / bplane elements further.  GEMM_LOWER
// writes i - j >= diag_off only and skips tiles with nothing to write.
int tc_gemm16(cudaStream_t st, bool bf16, bool split, long m, long n, long k, float alpha, const uint16_t* A,
              long lda, const uint16_t* B, long ldb, float beta, float* C, long ldc, GemmMode mode, long diag_off,
              const int* guard, int guard_limit, long aplane, long bplane) {
  if (m <= 0 || n <= 0) return FLA_SUCCESS;
  if (k <= 0) {
    set_last_error("tc_gemm16: k must be positive");
    return FLA_FAILURE;
  }
  CUtensorMap mA, mB, mAl, mBl;
  if (!make_map16(&mA, A, m, k, lda, TC_BM) || !make_map16(&mB, B, n, k, ldb, TC_TN)) {
    set_last_error("tc_gemm16: cuTensorMapEncodeTiled failed");
    return FLA_FAILURE;
  }
  if (split) {
    if (!make_map16(&mAl, A + aplane, m, k, lda, TC_BM) || !make_map16(&mBl, B + bplane, n, k, ldb, TC_TN)) {
      set_last_error("tc_gemm16: cuTensorMapEncodeTiled failed");
      return FLA_FAILURE;
    }
  } else {
    mAl = mA;
    mBl = mB;
  }
  // instruction descriptor: FP32 accumulator, A/B FP16 (0) or BF16 (1),
  // both K-major, N = TN, M = 128
  const uint32_t fmt = bf16 ? 1u : 0u;
  const uint32_t idesc = (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(TC_TN >> 3) << 17) |
                         ((uint32_t)(TC_BM >> 4) << 24);
  const long ntiles = ((m + TC_BM - 1) / TC_BM) * ((n + TC_TN - 1) / TC_TN);
  dim3 grid((unsigned)std::min<long>(ntiles, ctx().num_sms));
  const int ps = prof_begin(st);
  const int lower = mode == GEMM_LOWER ? 1 : 0;
  int* err = ctx().d_status + ST_ERROR;
  if (split) {
    tc_set_attr<true>();
    tc_gemm16_kernel<TC_TN, TC_STAGES, true><<<grid, TC_THREADS, TcCfg<TC_TN, TC_STAGES, true>::SMEM_BYTES, st>>>(
        mA, mB, mAl, mBl, C, ldc, (int)m, (int)n, (int)k, alpha, beta, idesc, lower, diag_off, guard, guard_limit,
        err);
  } else {
    tc_set_attr<false>();
    tc_gemm16_kernel<TC_TN, TC_STAGES, false><<<grid, TC_THREADS, TcCfg<TC_TN, TC_STAGES, false>::SMEM_BYTES, st>>>(
        mA, mB, mAl, mBl, C, ldc, (int)m, (int)n, (int)k, alpha, beta, idesc, lower, diag_off, guard, guard_limit,
        err);
  }
  const double fl = mode == GEMM_LOWER && m == n ? (double)m * (double)(m + 1) * (double)k : 2.0 * m * (double)n * k;
  prof_end(ps, st, PROF_GEMM, fl);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

}  // namespace fb
