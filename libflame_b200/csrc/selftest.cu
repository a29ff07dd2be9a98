// Concurrency self-test of the FP64 GEMM engine.
//
// The factorizations run their trailing-update GEMM on the main stream
// while the next panel is factored on the second stream, so the GEMM's CTAs
// share SMs with the panel kernels.  This check repeats one update-shaped
// GEMM (C -= A B, beta = 1, the LU's operand layout) on the main stream with
// Cholesky-panel work on the second stream (diagonal-block factorization,
// triangle inverse, the two panel GEMMs and the panel transpose, six panels
// per GEMM) and compares every result bitwise with the result computed
// alone.  A GEMM whose shared-memory pipeline released a stage before its
// reads had completed gave, on some B200s, a few wrong tiles per 10^8 here,
// none with the GEMM alone.
#include <algorithm>

#include "common.h"

namespace fb {

namespace {

// Deterministic values in [-scale/2, scale/2) from a 64-bit hash of the index.
__global__ void st_fill_kernel(double* p, long n, unsigned seed, double scale) {
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    unsigned long long x = (unsigned long long)i * 6364136223846793005ull + seed * 1442695040888963407ull;
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    p[i] = scale * ((double)(x >> 11) * (1.0 / 9007199254740992.0) - 0.5);
  }
}

// A diagonally dominant (hence SPD after symmetrization by the lower
// triangle) b x b block.
__global__ void st_spd_kernel(double* p, int b) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < b) p[i + (long)i * b] += 2.0 * b;
}

__global__ void st_compare_kernel(const double* __restrict__ C, const double* __restrict__ R, long total,
                                  unsigned long long* count) {
  unsigned long long local = 0;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x)
    local += __double_as_longlong(C[e]) != __double_as_longlong(R[e]);
  if (local) atomicAdd(count, local);
}

// Device buffers of one check, freed (after both library streams are idle)
// when the check returns.
struct Buffers {
  std::vector<void*> ptrs;
  ~Buffers() {
    cudaStreamSynchronize(ctx().side);
    cudaStreamSynchronize(ctx().stream);
    for (void* p : ptrs) cudaFree(p);
  }
  double* get(size_t elems) {
    void* p = nullptr;
    if (cudaMalloc(&p, elems * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    ptrs.push_back(p);
    return (double*)p;
  }
};

}  // namespace

int gemm_concurrency_check(long m, long n, long k, int iters, unsigned long long* mismatches) {
  Context& cx = ctx();
  cudaStream_t st = cx.stream, sd = cx.side;
  *mismatches = 0;
  const long ld = (m + 1) & ~1L;  // TMA: 16-byte leading dimensions
  const long ldk = (k + 1) & ~1L;
  const int b = 128;
  const long ps = (std::min<long>(std::max<long>(m, b), 8192) + 1) & ~1L;  // panel rows of the side work
  Buffers mem;
  double* A = mem.get((size_t)ld * k);
  double* B = mem.get((size_t)ldk * n);
  double* C0 = mem.get((size_t)ld * n);
  double* Cw = mem.get((size_t)ld * n);
  double* R = mem.get((size_t)ld * n);
  double* D0 = mem.get((size_t)b * b);
  double* D = mem.get((size_t)b * b);
  double* Li = mem.get((size_t)b * b);
  double* W = mem.get((size_t)ps * b);
  double* X = mem.get((size_t)ps * b);
  double* T = mem.get((size_t)ps * b);
  double* TT = mem.get((size_t)ps * b);
  unsigned long long* count = (unsigned long long*)mem.get(1);
  if (!A || !B || !C0 || !Cw || !R || !D0 || !D || !Li || !W || !X || !T || !TT || !count) {
    set_last_error("FLA_B200_gemm_concurrency_check: device allocation failed");
    return FLA_FAILURE;
  }
  const unsigned fg = (unsigned)(4 * cx.num_sms);
  st_fill_kernel<<<fg, 256, 0, st>>>(A, ld * k, 1, 1.0);
  st_fill_kernel<<<fg, 256, 0, st>>>(B, ldk * n, 2, 1.0);
  st_fill_kernel<<<fg, 256, 0, st>>>(C0, ld * n, 3, 10.0);
  st_fill_kernel<<<fg, 256, 0, st>>>(D0, (long)b * b, 4, 1.0);
  st_spd_kernel<<<1, b, 0, st>>>(D0, b);
  st_fill_kernel<<<fg, 256, 0, st>>>(W, ps * b, 5, 1.0);
  count_launch(6);
  FB_CK(cudaMemsetAsync(count, 0, sizeof(unsigned long long), st));
  FB_CK(cudaGetLastError());
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;
  const size_t cbytes = sizeof(double) * (size_t)ld * n;
  auto update = [&]() {
    return gemm_f64(st, false, false, m, n, k, -1.0, A, ld, B, ldk, 1.0, Cw, ld, GEMM_FULL, 0, nullptr, 0);
  };
  // reference: the update alone
  FB_CK(cudaMemcpyAsync(Cw, C0, cbytes, cudaMemcpyDeviceToDevice, st));
  if (update() != FLA_SUCCESS) return FLA_FAILURE;
  FB_CK(cudaMemcpyAsync(R, Cw, cbytes, cudaMemcpyDeviceToDevice, st));
  cudaEvent_t ev_start = cx.ev[2], ev_side = cx.ev[3];
  for (int it = 0; it < iters; ++it) {
    FB_CK(cudaMemcpyAsync(Cw, C0, cbytes, cudaMemcpyDeviceToDevice, st));
    FB_CK(cudaEventRecord(ev_start, st));
    FB_CK(cudaStreamWaitEvent(sd, ev_start, 0));
    if (update() != FLA_SUCCESS) return FLA_FAILURE;
    for (int q = 0; q < 6; ++q) {
      FB_CK(cudaMemcpyAsync(D, D0, sizeof(double) * b * b, cudaMemcpyDeviceToDevice, sd));
      if (potrf_diag_dev(D, b, b, 0, sd) != FLA_SUCCESS ||
          tri_inverse_lower(D, b, b, false, Li, b, sd) != FLA_SUCCESS ||
          gemm_f64(sd, false, true, ps, b, b, 1.0, W, ps, Li, b, 0.0, X, ps, GEMM_FULL, 0, nullptr, 0) !=
              FLA_SUCCESS ||
          gemm_f64(sd, false, true, ps, b, b, -1.0, X, ps, X, ps, 1.0, T, ps, GEMM_LOWER, 0, nullptr, 0) !=
              FLA_SUCCESS ||
          transpose_dev(X, ps, TT, b, ps, b, false, sd) != FLA_SUCCESS)
        return FLA_FAILURE;
    }
    FB_CK(cudaEventRecord(ev_side, sd));
    FB_CK(cudaStreamWaitEvent(st, ev_side, 0));
    st_compare_kernel<<<fg, 256, 0, st>>>(Cw, R, ld * n, count);
    count_launch();
  }
  FB_CK(cudaGetLastError());
  unsigned long long h = 0;
  FB_CK(cudaMemcpyAsync(&h, count, sizeof(h), cudaMemcpyDeviceToHost, st));
  int info = -1;
  const int rs = status_read(&info);  // synchronizes; reports an expired wait
  if (rs != FLA_SUCCESS) return rs;
  *mismatches = h;
  return FLA_SUCCESS;
}

}  // namespace fb

// C-ABI entry (include/FLAME_b200.h).
extern "C" int FLA_B200_gemm_concurrency_check(long m, long n, long k, int iters, unsigned long long* mismatches) {
  if (!mismatches || m <= 0 || n <= 0 || k <= 0 || iters < 0) {
    fb::set_last_error("FLA_B200_gemm_concurrency_check: invalid argument");
    return FLA_FAILURE;
  }
  if (!fb::ctx().initialized) FLA_Init();
  fb::op_begin(fb::ctx().stream);  // also orders the call after the caller's default-stream work
  const int r = fb::gemm_concurrency_check(m, n, k, iters, mismatches);
  if (r != FLA_SUCCESS) fb::sync_all();
  return r;
}
