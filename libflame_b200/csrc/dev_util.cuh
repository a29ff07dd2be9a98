// Device-side helpers: mbarriers, TMA, bounded waits, FP64 MMA.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace fb {

// Bounded waits: every spin in this library gives up after this many
// nanoseconds of %globaltimer, records an error code in the status block and
// lets the kernel return.
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // 2 s

__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Wait for phase `parity` of an mbarrier; false (and *err set) on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int* err, int code) {
  if (mbar_try_wait(bar, parity)) return true;
  unsigned long long t0 = globaltimer_ns();
  for (;;) {
    for (int i = 0; i < 64; ++i)
      if (mbar_try_wait(bar, parity)) return true;
    if (globaltimer_ns() - t0 > kWaitLimitNs) {
      if (err) atomicExch(err, code);
      return false;
    }
  }
}

// 2D tiled TMA load into shared memory, completion on an mbarrier.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y,
                                            uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// FP64 tensor-core MMA (DMMA), D = A*B + D, shape m8n8k4.
//   lane l: a = A[l>>2][l&3], b = B[l&3][l>>2], d = D[l>>2][2(l&3) + {0,1}].
__device__ __forceinline__ void dmma_884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Grid-wide barrier for cooperative launches: monotonically increasing
// counter; barrier number `epoch` (1-based) completes when it reaches
// nblocks*epoch.  Bounded: returns false (and sets *err) on timeout.
__device__ __forceinline__ bool grid_barrier(unsigned int* counter, unsigned int nblocks,
                                             unsigned int epoch, int* err, int code) {
  __shared__ int s_bar_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    bool ok = true;
    __threadfence();
    atomicAdd(counter, 1u);
    unsigned int target = nblocks * epoch;
    unsigned long long t0 = 0;
    int spins = 0;
    while (true) {
      unsigned int v = *((volatile unsigned int*)counter);
      if (v >= target) break;
      if (err && *((volatile int*)err) != 0) { ok = false; break; }
      if (++spins == 64) {
        spins = 0;
        unsigned long long t = globaltimer_ns();
        if (t0 == 0) t0 = t;
        else if (t - t0 > kWaitLimitNs) {
          if (err) atomicExch(err, code);
          ok = false;
          break;
        }
      }
    }
    __threadfence();
    s_bar_ok = ok ? 1 : 0;
  }
  __syncthreads();
  return s_bar_ok != 0;
}

}  // namespace fb

namespace fb {

// Copy the b x b (b <= 128) block at A (ld) into S (stride lds) with
// NT threads: each thread issues 16 independent loads before it stores any,
// so the copy costs a few memory latencies instead of one per element.
// keep(r, c) selects the elements copied; the others are written as zero
// when zero_rest, else left alone.
template <int NT, bool ZERO_REST, class Keep>
__device__ __forceinline__ void load_block_f64(const double* __restrict__ A, long ld, int b, double* S, int lds,
                                               Keep keep) {
  constexpr int PER = 128 * 128 / NT;
  constexpr int BATCH = PER < 16 ? PER : 16;
#pragma unroll 1
  for (int j0 = 0; j0 < PER; j0 += BATCH) {
    double v[BATCH];
#pragma unroll
    for (int j = 0; j < BATCH; ++j) {
      const int e = threadIdx.x + (j0 + j) * NT;
      const int r = e & 127, c = e >> 7;
      v[j] = (r < b && c < b && keep(r, c)) ? A[r + (long)c * ld] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < BATCH; ++j) {
      const int e = threadIdx.x + (j0 + j) * NT;
      const int r = e & 127, c = e >> 7;
      if (r < b && c < b && (ZERO_REST || keep(r, c))) S[r + c * lds] = v[j];
    }
  }
}

}  // namespace fb

namespace fb {

// ---- DSMEM pushes completing an mbarrier transaction count on the
// receiving CTA (no cluster-wide fence): the receiver arms its mbarrier with
// the bytes it expects per phase and waits with cluster-scope acquire.
__device__ __forceinline__ uint32_t mapa_shared(uint32_t addr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}

__device__ __forceinline__ void st_async_f64(uint32_t raddr, double v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];" ::"r"(raddr),
               "l"(__double_as_longlong(v)), "r"(rbar)
               : "memory");
}

__device__ __forceinline__ void st_async_b32(uint32_t raddr, uint32_t v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(raddr), "r"(v),
               "r"(rbar)
               : "memory");
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global memory into this CTA's shared memory, completing the bytes
// on the mbarrier bar.  No multicast.
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// Orders this thread's generic-proxy writes to shared memory before later
// async-proxy reads of them (a bulk copy issued after a CTA barrier).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from this CTA's shared memory to a cluster peer's (rdst, from mapa),
// completing the bytes on the peer's mbarrier rbar.  No multicast.
__device__ __forceinline__ void bulk_copy_to_peer(uint32_t rdst, uint32_t src, uint32_t bytes, uint32_t rbar) {
  asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   rdst),
               "r"(src), "r"(bytes), "r"(rbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait_cluster(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait (kWaitLimitNs of %globaltimer) with cluster-scope acquire;
// false (and *err set) on timeout.
__device__ __forceinline__ bool mbar_wait_cluster(uint32_t bar, uint32_t parity, int* err, int code) {
  if (mbar_try_wait_cluster(bar, parity)) return true;
  const unsigned long long t0 = globaltimer_ns();
  for (;;) {
    for (int i = 0; i < 64; ++i)
      if (mbar_try_wait_cluster(bar, parity)) return true;
    if (globaltimer_ns() - t0 > kWaitLimitNs) {
      if (err) atomicExch(err, code);
      return false;
    }
  }
}

}  // namespace fb
