// Batched Cholesky and LU with partial pivoting (+ solves) for many small
// matrices of uneven sizes (n <= 512) in one persistent launch.
//
// No counterpart in the reference (which factors one FLA_Obj at a time:
// FLA_Chol, src/lapack/dec/chol/front/flamec/FLA_Chol.c:16-29; FLA_LU_piv,
// src/lapack/dec/lu/piv/front/flamec/FLA_LU_piv.c:16-33); each matrix is
// factored with the reference's semantics: lower Cholesky failing at the
// first non-positive (or NaN) pivot with its zero-based column reported;
// LU with the largest-magnitude pivot, the first row among equals, zero
// pivot columns left unscaled and the first reported, relative pivots.
//
// Design: a persistent grid (one CTA per SM) takes matrices from an atomic
// counter in a host-chosen order (largest first, so the tail of the
// schedule holds the small ones).  A CTA factors one matrix at a time,
// left-looking in panels of nb columns (nb per size bin, from the batched
// autotuner): the panel is loaded into shared memory, updated by all the
// previous columns with register-tiled FMAs (the previous columns streamed
// through shared memory in chunks of 8), factored there, and written back;
// every matrix is read from HBM about n/(2 nb) times instead of n/nb times
// for a right-looking update.  The solve keeps the right-hand sides in
// shared memory and sweeps 32-row blocks: one warp per right-hand side
// solves the diagonal block with shuffles, then all threads update the rows
// below (above for the transposed sweep).
#include <algorithm>
#include <climits>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "common.h"
#include "batched.h"
#include "dev_util.cuh"

namespace fb {

namespace {

constexpr int BT = 256;          // threads per CTA
constexpr int BMAXN = 512;       // largest matrix order
constexpr int BMAXNB = 32;       // widest panel
constexpr int KC = 8;            // columns of the streamed chunk
constexpr int BMAXRHS = 8;       // right-hand sides handled in shared memory

template <typename T>
struct BSmem {
  // panel (BMAXN x BMAXNB), streamed chunk of previous columns (BMAXN x KC),
  // chunk of the panel rows of those columns (BMAXNB x KC), right-hand sides
  static constexpr size_t PANEL = (size_t)BMAXN * (BMAXNB + 1);
  static constexpr size_t CHUNK = (size_t)BMAXN * KC;
  static constexpr size_t CHW = (size_t)BMAXNB * KC;
  static constexpr size_t RHS = (size_t)BMAXN * BMAXRHS;
  static constexpr size_t BYTES = (PANEL + CHUNK + CHW + RHS) * sizeof(T) + 64 * sizeof(int);
};

template <typename T>
__device__ __forceinline__ T tabs(T x) {
  return x < T(0) ? -x : x;
}

// P[r + c * ldp] -= sum_k Lrows(r, k) * Lw(c, k) for r < R, c < w, k < kn,
// with Lrows(r, k) = G[(row0 + r) + (k0 + k) * ld] (previous columns k0 ..
// k0 + kn) and Lw(c, k) = wbase[c * wcs + k * wks]: for the Cholesky the
// panel rows of the same columns, for the LU the U rows of the panel (in
// shared memory).
template <typename T>
__device__ void left_update(T* P, int ldp, int R, int w, const T* G, long ld, int row0, int k0, int kn,
                            const T* wbase, long wcs, long wks, T* sChunk, T* sW) {
  const int tid = threadIdx.x;
  // thread tile: rows rr + 64 i (i < 8), columns cg * 8 .. cg * 8 + 7
  const int rr = tid & 63, cg = tid >> 6;
  T acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int q = 0; q < 8; ++q) acc[i][q] = T(0);
  for (int kc = 0; kc < kn; kc += KC) {
    const int kk = min(KC, kn - kc);
    __syncthreads();
    for (int e = tid; e < R * KC; e += BT) {
      const int r = e % R, q = e / R;
      sChunk[r + q * BMAXN] = (q < kk) ? G[(long)(row0 + r) + (long)(k0 + kc + q) * ld] : T(0);
    }
    for (int e = tid; e < w * KC; e += BT) {
      const int c = e % w, q = e / w;
      sW[c + q * BMAXNB] = (q < kk) ? wbase[(long)c * wcs + (long)(kc + q) * wks] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < KC; ++q) {
      T a[8], b[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = sChunk[rr + 64 * i + q * BMAXN];
#pragma unroll
      for (int j = 0; j < 8; ++j) b[j] = sW[cg * 8 + j + q * BMAXNB];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = rr + 64 * i;
    if (r >= R) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = cg * 8 + j;
      if (c < w) P[r + c * ldp] -= acc[i][j];
    }
  }
  __syncthreads();
}

// Blocked solves with the factor in global memory, right-hand sides X
// (n x nrhs, ld BMAXN) in shared memory.  Lower (unit or not) forward sweep,
// or the transposed (upper) backward sweep with the lower factor (Cholesky:
// L^T; LU: the upper factor U is read as stored, upper = true).
// sD: 32 x 33 shared scratch for op(F)'s diagonal blocks, so the serial
// per-column steps of the warp solves read shared memory, not L2.
template <typename T>
__device__ void block_solve(const T* F, long ld, int n, T* X, int nrhs, bool lower, bool trans, bool unit, T* sD,
                            int ldx = BMAXN) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nt = blockDim.x;
  // op(F) is lower triangular when (lower && !trans) or (!lower && trans)
  const bool fwd = (lower != trans);
  const int nblk = (n + 31) / 32;
  for (int bi = 0; bi < nblk; ++bi) {
    const int b = fwd ? bi : nblk - 1 - bi;
    const int b0 = b * 32, w = min(32, n - b0);
    // op(F)(r, c) = trans ? F[c + r * ld] : F[r + c * ld]; the block into sD
    for (int e = tid; e < w * w; e += nt) {
      const int r = e % w, c = e / w;
      sD[r + c * 33] = trans ? F[(long)(b0 + c) + (long)(b0 + r) * ld] : F[(long)(b0 + r) + (long)(b0 + c) * ld];
    }
    __syncthreads();
    for (int q = warp; q < nrhs; q += nt / 32) {
      T y = lane < w ? X[b0 + lane + q * ldx] : T(0);
      for (int s = 0; s < w; ++s) {
        const int k = fwd ? s : w - 1 - s;
        if (lane == k && !unit) y = y / sD[k + k * 33];
        const T yk = __shfl_sync(0xffffffffu, y, k);
        const bool below = fwd ? (lane > k && lane < w) : (lane < k);
        if (below) y -= sD[lane + k * 33] * yk;
      }
      if (lane < w) X[b0 + lane + q * ldx] = y;
    }
    __syncthreads();
    // remaining rows: fwd rows [b0 + w, n), bwd rows [0, b0)
    const int r_lo = fwd ? b0 + w : 0, r_hi = fwd ? n : b0;
    const int nr = r_hi - r_lo;
    for (int e = tid; e < nr * nrhs; e += nt) {
      const int r = r_lo + e % nr, q = e / nr;
      T s = T(0);
      for (int k = 0; k < w; ++k) {
        const int c = b0 + k;
        const T o = trans ? F[(long)c + (long)r * ld] : F[(long)r + (long)c * ld];
        s = fma(o, X[c + q * ldx], s);
      }
      X[r + q * ldx] -= s;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Cholesky
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(BT, 1) chol_batched_kernel(BatchArgs<T> a) {
  extern __shared__ __align__(16) unsigned char bsm_raw[];
  T* sP = reinterpret_cast<T*>(bsm_raw);
  T* sChunk = sP + BSmem<T>::PANEL;
  T* sW = sChunk + BSmem<T>::CHUNK;
  T* sX = sW + BSmem<T>::CHW;
  __shared__ int s_next, s_fail;
  const int tid = threadIdx.x;
  for (;;) {
    if (tid == 0) s_next = atomicAdd(a.counter, 1);
    __syncthreads();
    const int slot = s_next;
    __syncthreads();
    if (slot >= a.count) break;
    const int mi = a.order[slot];
    const int n = a.n[mi];
    const long ld = a.ld[mi];
    T* G = a.A[mi];
    const int nb = max(1, min(BMAXNB, a.nb_of_size[min(n, BMAXN)]));
    if (tid == 0) s_fail = -1;
    __syncthreads();
    for (int j = 0; j < n; j += nb) {
      const int w = min(nb, n - j), R = n - j;
      const int ldp = BMAXN;
      for (int e = tid; e < R * w; e += BT) {
        const int r = e % R, c = e / R;
        sP[r + c * ldp] = G[(long)(j + r) + (long)(j + c) * ld];
      }
      __syncthreads();
      if (j > 0) left_update<T>(sP, ldp, R, w, G, ld, j, 0, j, G + j, 1, ld, sChunk, sW);
      // factor the panel: columns c of the w x w block and the rows below
      for (int c = 0; c < w; ++c) {
        __shared__ T s_d;
        if (tid == 0) {
          const T d = sP[c + c * ldp];
          if (!(d > T(0))) {
            s_fail = j + c;
            s_d = T(0);
          } else {
            s_d = sqrt(d);
            sP[c + c * ldp] = s_d;
          }
        }
        __syncthreads();
        if (s_fail >= 0) break;
        const T d = s_d;
        const T dinv = T(1) / d;
        for (int r = c + 1 + tid; r < R; r += BT) sP[r + c * ldp] *= dinv;
        __syncthreads();
        const int cols = w - c - 1;
        for (int e = tid; e < (R - c - 1) * cols; e += BT) {
          const int r = c + 1 + e % (R - c - 1), cc = c + 1 + e / (R - c - 1);
          if (r >= cc) sP[r + cc * ldp] -= sP[r + c * ldp] * sP[cc + c * ldp];
        }
        __syncthreads();
      }
      // write back the lower part of the panel (the failing column included)
      for (int e = tid; e < R * w; e += BT) {
        const int r = e % R, c = e / R;
        if (r >= c) G[(long)(j + r) + (long)(j + c) * ld] = sP[r + c * ldp];
      }
      __syncthreads();
      if (s_fail >= 0) break;
    }
    if (tid == 0) a.info[mi] = s_fail;
    // solve with the factor when it succeeded
    if (a.B && s_fail < 0) {
      const int nrhs = a.nrhs;
      T* Bm = a.B[mi];
      const long ldb = a.ldb[mi];
      for (int e = tid; e < n * nrhs; e += BT) sX[e % n + (e / n) * BMAXN] = Bm[(long)(e % n) + (long)(e / n) * ldb];
      __syncthreads();
      block_solve<T>(G, ld, n, sX, nrhs, true, false, false, sChunk);
      block_solve<T>(G, ld, n, sX, nrhs, true, true, false, sChunk);
      for (int e = tid; e < n * nrhs; e += BT) Bm[(long)(e % n) + (long)(e / n) * ldb] = sX[e % n + (e / n) * BMAXN];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// FP64 Cholesky, orders up to 1024, updates on the FP64 tensor cores
// ---------------------------------------------------------------------------
// One CTA of 16 warps per matrix (persistent over the schedule), left-looking
// in panels of 32 columns:
//   1. P := A(j:n, j:j+32) - L(j:n, 0:j) L(j:j+32, 0:j)^T with DMMA m8n8k4
//      tiles: the previous columns stream through shared memory 8 at a time
//      (cp.async, double-buffered) and each warp accumulates 4 x 4 8x8 tiles
//      in registers; panels taller than 512 rows take several passes of 512
//      rows, each staging the panel's own 32 rows (the B operand) beside its
//      rows, so no warp holds more than 16 tiles;
//   2. warp 0 factors the 32 x 32 diagonal block in registers (lane r holds
//      row r; shuffles broadcast the pivot column): sqrt, reciprocal scaling
//      and the rank-1 update as FLA_Chol's unblocked variant, stopping at the
//      first pivot that is not > 0 (NaN included);
//   3. every thread solves rows below with the block: x := x L11^-T by
//      columns (reciprocal multiply, then axpy), as dtrsm Right/Lower/Trans.
// The per-column work of a panel stays inside one warp: no CTA barrier per
// column.  Optionally the log-determinant sum_i log L(i, i) per matrix and
// the solve of up to 8 right-hand sides in the same launch.
constexpr int DT = 512;                 // threads per CTA
constexpr int DMAXN = 1024;             // largest order
constexpr int DNB = 32;                 // panel width
constexpr int DKC = 16;                 // previous columns per staged chunk (one warp each)
constexpr int DPASS = 512;              // rows per update pass
constexpr int DPO = 36;                 // offset of the pass rows in a staged column (doubles)
constexpr int DRP = 2 + DPO + DPASS + 10;  // staged column stride: shift slot, panel rows, gap, pass rows, spare
constexpr size_t DCHUNK = (size_t)DRP * DKC;
constexpr size_t DSMEM_BYTES = (2 * DCHUNK + (size_t)DNB * (DNB + 1) + DNB) * sizeof(double) + 256;
static_assert((size_t)DMAXN * BMAXRHS <= 2 * DCHUNK, "right-hand sides reuse the chunk buffers");

// Stage columns k0 .. k0 + 15 of G with bulk copies issued by one warp:
// lane (part, q) copies column k0 + q's panel rows j .. j + min(32, R) - 1
// (part 0) or its pass rows j + p0 .. j + p0 + np - 1 (part 1).  A bulk copy
// needs 16-byte aligned ends, so a column whose first element sits 8 bytes
// past a boundary (odd leading dimensions) is copied from one element
// earlier into one slot earlier: element r of staged column q lies at
// buf + q DRP + shift[q] + r (panel rows) or + DPO + r (pass rows), shift[q]
// = 2 - (misaligned).  The copies may read one element before the first
// row and one after the last: rows j - 1 >= 31 and, since the staged
// columns are left of the panel (column < j <= n - 1), at most one element
// into the next column's storage.  Rows past R are left unwritten; they only
// feed output rows or columns that are discarded.
__device__ __forceinline__ void dchunk_issue_bulk(double* buf, int* shift, uint32_t bar, const double* G, long ld,
                                                  int j, int R, int p0, int np, int k0) {
  const int lane = threadIdx.x & 31, q = lane & 15, part = lane >> 4;
  const double* src = G + (long)j + (long)(k0 + q) * ld + (part ? p0 : 0);
  const int cnt = part ? np : min(DNB, R);
  const int off = (int)((reinterpret_cast<uintptr_t>(src) >> 3) & 1);
  const int sh = 2 - off;
  const uint32_t bytes = (uint32_t)(8 * ((cnt + off + 1) & ~1));
  const unsigned total = __reduce_add_sync(0xffffffffu, bytes);
  if (lane == 0) mbar_arrive_expect_tx(bar, total);
  if (part == 0) shift[q] = sh;
  __syncwarp();
  double* dst = buf + q * DRP + sh + (part ? DPO : 0) - off;
  bulk_copy_g2s(smem_u32(dst), src - off, bytes, bar);
}

__global__ void __launch_bounds__(DT, 1) chol_batched_dmma_kernel(BatchArgs<double> a) {
  extern __shared__ __align__(16) unsigned char bsm_raw[];
  double* sC = reinterpret_cast<double*>(bsm_raw);  // [2][DKC][DRP]
  double* sL = sC + 2 * DCHUNK;                     // L11, row-major [DNB][DNB + 1]
  double* sR = sL + DNB * (DNB + 1);                // 1 / L11(k, k)
  __shared__ int s_next, s_fail;
  __shared__ int s_shift[2][DKC];                   // column shifts of the two staged chunks
  __shared__ __align__(8) unsigned long long s_bar[2];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const unsigned full = 0xffffffffu;
  const uint32_t bar0 = smem_u32(&s_bar[0]);
  if (tid == 0) {
    mbar_init(bar0, 1);
    mbar_init(bar0 + 8, 1);
    fence_barrier_init();
  }
  __syncthreads();
  uint32_t uses[2] = {0u, 0u};  // completed phases per buffer (the same in every thread)
  bool ok = true;               // false after a wait ran out (the results are then garbage)
  for (;;) {
    if (tid == 0) s_next = atomicAdd(a.counter, 1);
    __syncthreads();
    const int slot = s_next;
    __syncthreads();
    if (slot >= a.count) break;
    const int mi = a.order[slot];
    const int n = a.n[mi];
    const long ld = a.ld[mi];
    double* G = a.A[mi];
    if (tid == 0) s_fail = -1;
    __syncthreads();
    for (int j = 0; j < n; j += DNB) {
      const int w = min(DNB, n - j), R = n - j;
      // ---- 1. the panel update, in passes of up to 512 rows
      if (j > 0) {
        const int nch = j / DKC;  // j is a multiple of 32, DKC = 16
        for (int p0 = 0; p0 < R; p0 += DPASS) {
          const int np = min(DPASS, R - p0);
          double acc[4][4][2];
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int ct = 0; ct < 4; ++ct) acc[i][ct][0] = acc[i][ct][1] = 0.0;
          if (warp == 0) dchunk_issue_bulk(sC, s_shift[0], bar0, G, ld, j, R, p0, np, 0);
          for (int ch = 0; ch < nch; ++ch) {
            const int bsel = ch & 1;
            if (warp == 0 && ch + 1 < nch)
              dchunk_issue_bulk(sC + (bsel ^ 1) * DCHUNK, s_shift[bsel ^ 1], bar0 + 8 * (bsel ^ 1), G, ld, j, R, p0,
                                np, (ch + 1) * DKC);
            // after a wait has run out (error flag set) the rest is not waited for
            if (ok && !mbar_wait(bar0 + 8 * bsel, uses[bsel] & 1u, a.err, 41)) ok = false;
            ++uses[bsel];
            const double* C = sC + bsel * DCHUNK;
#pragma unroll
            for (int kk = 0; kk < DKC; kk += 4) {
              const int cq = kk + (lane & 3);
              const double* Ck = C + cq * DRP + s_shift[bsel][cq] + (lane >> 2);
              double b[4];
#pragma unroll
              for (int ct = 0; ct < 4; ++ct) b[ct] = Ck[ct * 8];
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                const int rt = warp + 16 * i;  // 8-row tile of the pass
                if (rt * 8 < np) {
                  const double av = Ck[DPO + rt * 8];
#pragma unroll
                  for (int ct = 0; ct < 4; ++ct) dmma_884(acc[i][ct][0], acc[i][ct][1], av, b[ct]);
                }
              }
            }
            __syncthreads();  // the buffer is refilled two chunks later
          }
          // P -= acc (lower part of the diagonal block only)
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const int r = p0 + (warp + 16 * i) * 8 + (lane >> 2);
            if (r >= p0 + np) continue;
#pragma unroll
            for (int ct = 0; ct < 4; ++ct)
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int c = ct * 8 + 2 * (lane & 3) + e;
                if (c < w && r >= c) G[(long)(j + r) + (long)(j + c) * ld] -= acc[i][ct][e];
              }
          }
        }
        __syncthreads();
      }
      // ---- 2. the diagonal block in warp 0
      if (warp == 0) {
        double d[DNB];
#pragma unroll
        for (int c = 0; c < DNB; ++c) d[c] = (lane < w && c < w && c <= lane) ? G[(long)(j + lane) + (long)(j + c) * ld] : 0.0;
        // A run-time loop over the columns (a fully unrolled one is tens of
        // KB of straight-line code that one warp runs once per panel, missing
        // the instruction cache throughout); select chains over
        // compile-time indices keep d in registers, and column c reaches
        // the other lanes through shared memory (sL's first two rows as a
        // two-slot buffer, written back only after the loop).
        double* scol = sL;
        int fail = -1;
#pragma unroll 1
        for (int c = 0; c < w; ++c) {
          double dc = d[0];  // this lane's entry of column c
#pragma unroll
          for (int q = 1; q < DNB; ++q)
            if (q == c) dc = d[q];
          const double piv = __shfl_sync(full, dc, c);
          if (!(piv > 0.0)) {  // the same value in every lane
            fail = c;
            break;
          }
          const double rs = rsqrt(piv);  // one sequence: the chain's latency
          const double sq = piv * rs;
          const double nc = lane == c ? sq : (lane > c ? dc * rs : dc);  // L(lane, c)
#pragma unroll
          for (int q = 0; q < DNB; ++q)
            if (q == c) d[q] = nc;
          double* col = scol + (c & 1) * DNB;
          col[lane] = nc;
          __syncwarp();
#pragma unroll
          for (int q = 0; q < DNB; ++q) {
            const double lq = col[q];  // L(q, c)
            if (q > c && lane >= q) d[q] = fma(-nc, lq, d[q]);
          }
        }
        __syncwarp();
#pragma unroll
        for (int c = 0; c < DNB; ++c) {
          if (lane < w && c < w && c <= lane) G[(long)(j + lane) + (long)(j + c) * ld] = d[c];
          sL[lane * (DNB + 1) + c] = (c <= lane) ? d[c] : 0.0;
        }
        double dl = d[0];  // this lane's diagonal entry, without indexing d by a run-time value
#pragma unroll
        for (int c = 1; c < DNB; ++c)
          if (c == lane) dl = d[c];
        if (lane < w) sR[lane] = 1.0 / dl;
        if (lane == 0) s_fail = fail >= 0 ? j + fail : -1;
      }
      __syncthreads();
      if (s_fail >= 0) break;
      // ---- 3. rows below the block: x := x L11^-T
      for (int r = j + w + tid; r < n; r += DT) {
        double x[DNB];
#pragma unroll
        for (int c = 0; c < DNB; ++c) x[c] = c < w ? G[(long)r + (long)(j + c) * ld] : 0.0;
#pragma unroll
        for (int k = 0; k < DNB; ++k) {
          if (k < w) {
            x[k] *= sR[k];
#pragma unroll
            for (int jj = k + 1; jj < DNB; ++jj) x[jj] = fma(-sL[jj * (DNB + 1) + k], x[k], x[jj]);
          }
        }
#pragma unroll
        for (int c = 0; c < DNB; ++c)
          if (c < w) G[(long)r + (long)(j + c) * ld] = x[c];
      }
      __syncthreads();
    }
    if (tid == 0) a.info[mi] = s_fail;
    // log-determinant (fixed order: lane-strided partial sums, shuffle tree)
    if (a.logdet && warp == 0) {
      double sl = 0.0;
      if (s_fail < 0)
        for (int i = lane; i < n; i += 32) sl += log(G[(long)i + (long)i * ld]);
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) sl += __shfl_xor_sync(full, sl, off);
      if (lane == 0) a.logdet[mi] = s_fail < 0 ? sl : __longlong_as_double(0x7ff8000000000000ll);
    }
    // solve with the factor when it succeeded
    if (a.B && s_fail < 0) {
      const int nrhs = a.nrhs;
      double* Bm = a.B[mi];
      const long ldb = a.ldb[mi];
      double* sX = sC;
      for (int e = tid; e < n * nrhs; e += DT) sX[e % n + (e / n) * DMAXN] = Bm[(long)(e % n) + (long)(e / n) * ldb];
      __syncthreads();
      block_solve<double>(G, ld, n, sX, nrhs, true, false, false, sL, DMAXN);
      block_solve<double>(G, ld, n, sX, nrhs, true, true, false, sL, DMAXN);
      for (int e = tid; e < n * nrhs; e += DT) Bm[(long)(e % n) + (long)(e / n) * ldb] = sX[e % n + (e / n) * DMAXN];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// LU with partial pivoting
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(BT, 1) lu_batched_kernel(BatchArgs<T> a) {
  extern __shared__ __align__(16) unsigned char bsm_raw[];
  T* sP = reinterpret_cast<T*>(bsm_raw);
  T* sChunk = sP + BSmem<T>::PANEL;
  T* sW = sChunk + BSmem<T>::CHUNK;
  T* sX = sW + BSmem<T>::CHW;
  int* s_piv = reinterpret_cast<int*>(sX + BSmem<T>::RHS);  // nb pivots of the panel
  __shared__ int s_next, s_null;
  __shared__ T s_rv[BT / 32];
  __shared__ int s_ri[BT / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (;;) {
    if (tid == 0) s_next = atomicAdd(a.counter, 1);
    __syncthreads();
    const int slot = s_next;
    __syncthreads();
    if (slot >= a.count) break;
    const int mi = a.order[slot];
    const int n = a.n[mi];
    const long ld = a.ld[mi];
    T* G = a.A[mi];
    int* piv = a.piv[mi];
    const int nb = max(1, min(BMAXNB, a.nb_of_size[min(n, BMAXN)]));
    if (tid == 0) s_null = -1;
    __syncthreads();
    const int ldp = BMAXN;
    for (int j = 0; j < n; j += nb) {
      const int w = min(nb, n - j);
      // 1. load the whole block column, apply the earlier interchanges to it
      for (int e = tid; e < n * w; e += BT) {
        const int r = e % n, c = e / n;
        sP[r + c * ldp] = G[(long)r + (long)(j + c) * ld];
      }
      __syncthreads();
      if (tid < w)
        for (int i = 0; i < j; ++i) {
          const int t = i + piv[i];
          if (t != i) {
            const T x = sP[i + tid * ldp];
            sP[i + tid * ldp] = sP[t + tid * ldp];
            sP[t + tid * ldp] = x;
          }
        }
      __syncthreads();
      // 2. U rows of the block column (unit lower solve with L(0:j, 0:j)) and
      //    the left-looking update of rows j..n, 32 columns of L at a time
      for (int b0 = 0; b0 < j; b0 += 32) {
        const int bw = min(32, j - b0);
        // diagonal block: one warp per panel column
        for (int c = warp; c < w; c += BT / 32) {
          T y = lane < bw ? sP[b0 + lane + c * ldp] : T(0);
          for (int k = 0; k < bw; ++k) {
            const T yk = __shfl_sync(0xffffffffu, y, k);
            if (lane > k && lane < bw) y -= G[(long)(b0 + lane) + (long)(b0 + k) * ld] * yk;
          }
          if (lane < bw) sP[b0 + lane + c * ldp] = y;
        }
        __syncthreads();
        // rows b0+bw .. n: P(r, c) -= L(r, b0:b0+bw) U(b0:b0+bw, c)
        const int R = n - (b0 + bw);
        if (R > 0) left_update<T>(sP + (b0 + bw), ldp, R, w, G, ld, b0 + bw, b0, bw, sP + b0, ldp, 1, sChunk, sW);
      }
      // 3. factor rows j..n of the panel with partial pivoting
      for (int c = 0; c < w; ++c) {
        const int jc = j + c;
        T bv = T(-1);
        int bi = INT_MAX;
        for (int r = jc + tid; r < n; r += BT) {
          const T v = tabs(sP[r + c * ldp]);
          if (v > bv || (v == bv && r < bi)) { bv = v; bi = r; }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
          const T ov = __shfl_xor_sync(0xffffffffu, bv, off);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
          if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        if (lane == 0) { s_rv[warp] = bv; s_ri[warp] = bi; }
        __syncthreads();
        if (tid == 0) {
          T v = s_rv[0];
          int i0 = s_ri[0];
          for (int q = 1; q < BT / 32; ++q)
            if (s_rv[q] > v || (s_rv[q] == v && s_ri[q] < i0)) { v = s_rv[q]; i0 = s_ri[q]; }
          if (i0 == INT_MAX) i0 = jc;  // no orderable entry (NaN): keep the row
          s_piv[c] = i0;
        }
        __syncthreads();
        const int r = s_piv[c];
        const T p = sP[r + c * ldp];
        if (p == T(0)) {
          if (tid == 0 && s_null < 0) s_null = jc;
        } else {
          if (r != jc)
            for (int cc = tid; cc < w; cc += BT) {
              const T x = sP[jc + cc * ldp];
              sP[jc + cc * ldp] = sP[r + cc * ldp];
              sP[r + cc * ldp] = x;
            }
          __syncthreads();
          const T pinv = T(1) / p;
          for (int rr = jc + 1 + tid; rr < n; rr += BT) sP[rr + c * ldp] *= pinv;
          __syncthreads();
          const int cols = w - c - 1, rows = n - jc - 1;
          for (int e = tid; e < rows * cols; e += BT) {
            const int rr = jc + 1 + e % rows, cc = c + 1 + e / rows;
            sP[rr + cc * ldp] -= sP[rr + c * ldp] * sP[jc + cc * ldp];
          }
        }
        __syncthreads();
      }
      // 4. write the block column back, record the pivots
      for (int e = tid; e < n * w; e += BT) {
        const int r = e % n, c = e / n;
        G[(long)r + (long)(j + c) * ld] = sP[r + c * ldp];
      }
      if (tid < w) piv[j + tid] = s_piv[tid] - (j + tid);
      __syncthreads();
      // 5. this panel's interchanges on the earlier columns 0..j-1
      for (int col = tid; col < j; col += BT)
        for (int c = 0; c < w; ++c) {
          const int r0 = j + c, t = s_piv[c];
          if (t != r0) {
            const T x = G[(long)r0 + (long)col * ld];
            G[(long)r0 + (long)col * ld] = G[(long)t + (long)col * ld];
            G[(long)t + (long)col * ld] = x;
          }
        }
      __threadfence_block();
      __syncthreads();
    }
    if (tid == 0) a.info[mi] = s_null;
    if (a.B && s_null < 0) {
      const int nrhs = a.nrhs;
      T* Bm = a.B[mi];
      const long ldb = a.ldb[mi];
      for (int e = tid; e < n * nrhs; e += BT) sX[e % n + (e / n) * BMAXN] = Bm[(long)(e % n) + (long)(e / n) * ldb];
      __syncthreads();
      if (tid < nrhs)
        for (int i = 0; i < n; ++i) {
          const int t = i + piv[i];
          if (t != i) {
            const T x = sX[i + tid * BMAXN];
            sX[i + tid * BMAXN] = sX[t + tid * BMAXN];
            sX[t + tid * BMAXN] = x;
          }
        }
      __syncthreads();
      block_solve<T>(G, ld, n, sX, nrhs, true, false, true, sChunk);
      block_solve<T>(G, ld, n, sX, nrhs, false, false, false, sChunk);
      for (int e = tid; e < n * nrhs; e += BT) Bm[(long)(e % n) + (long)(e / n) * ldb] = sX[e % n + (e / n) * BMAXN];
    }
    __syncthreads();
  }
}

template <typename T>
int launch_batched(bool lu, BatchArgs<T> args, cudaStream_t st) {
  if constexpr (sizeof(T) == 8) {
    if (!lu) {
      // FP64 Cholesky: the DMMA kernel (orders up to 1024)
      static bool dattr = false;
      if (!dattr) {
        FB_CK(cudaFuncSetAttribute(chol_batched_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)DSMEM_BYTES));
        dattr = true;
      }
      const int grid = std::min(ctx().num_sms, std::max(1, args.count));
      const int ps = prof_begin(st);
      chol_batched_dmma_kernel<<<grid, DT, DSMEM_BYTES, st>>>(args);
      prof_end(ps, st, PROF_OTHER, 0.0);
      count_launch();
      FB_CK(cudaGetLastError());
      return FLA_SUCCESS;
    }
  }
  static bool attr[2] = {false, false};
  const size_t smem = BSmem<T>::BYTES;
  if (!attr[lu ? 1 : 0]) {
    if (lu)
      FB_CK(cudaFuncSetAttribute(lu_batched_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    else
      FB_CK(cudaFuncSetAttribute(chol_batched_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr[lu ? 1 : 0] = true;
  }
  const int grid = std::min(ctx().num_sms, std::max(1, args.count));
  const int ps = prof_begin(st);
  if (lu)
    lu_batched_kernel<T><<<grid, BT, smem, st>>>(args);
  else
    chol_batched_kernel<T><<<grid, BT, smem, st>>>(args);
  prof_end(ps, st, PROF_OTHER, 0.0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// per-device panel width by matrix order (autotuned), index 0..BMAXN
struct NbTable {
  std::vector<int> host;
  int* dev = nullptr;
  bool tuned = false;
};
NbTable g_nb[2][2];  // [lu][fp64]
std::mutex g_nb_mu;

int* nb_table(bool lu, bool f64) {
  NbTable& t = g_nb[lu ? 1 : 0][f64 ? 1 : 0];
  if (!t.dev) {
    t.host.assign(BMAXN + 1, 32);
    for (int n = 0; n <= BMAXN; ++n) t.host[n] = n <= 32 ? 16 : 32;  // default before tuning
    if (cudaMalloc(&t.dev, sizeof(int) * (BMAXN + 1)) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    cudaMemcpy(t.dev, t.host.data(), sizeof(int) * (BMAXN + 1), cudaMemcpyHostToDevice);
  }
  return t.dev;
}

}  // namespace

// Host driver: order the matrices (largest first), launch once.
template <typename T>
int batched_factor(bool lu, int count, const int* h_n, T** d_A, const long* d_ld, const int* d_n, int** d_piv,
                   int nrhs, T** d_B, const long* d_ldb, int* d_info, cudaStream_t st, T* d_logdet) {
  if (count <= 0) return FLA_SUCCESS;
  std::vector<int> order(count);
  for (int i = 0; i < count; ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return h_n[x] > h_n[y]; });
  int* dwork = (int*)ws_get(WS_MISC, sizeof(int) * ((size_t)count + 64));
  if (!dwork) return FLA_FAILURE;
  FB_CK(cudaMemsetAsync(dwork, 0, sizeof(int), st));
  FB_CK(cudaMemcpyAsync(dwork + 32, order.data(), sizeof(int) * count, cudaMemcpyHostToDevice, st));
  BatchArgs<T> a;
  a.count = count;
  a.order = dwork + 32;
  a.counter = dwork;
  a.n = d_n;
  a.ld = d_ld;
  a.A = d_A;
  a.piv = d_piv;
  a.nrhs = nrhs;
  a.B = d_B;
  a.ldb = d_ldb;
  a.info = d_info;
  a.logdet = d_logdet;
  a.err = ctx().d_status + ST_ERROR;
  a.nb_of_size = nb_table(lu, sizeof(T) == 8);
  if (!a.nb_of_size) return FLA_FAILURE;
  // the host order must stay valid until the copy is done
  FB_CK(cudaStreamSynchronize(st));
  return launch_batched<T>(lu, a, st);
}
template int batched_factor<double>(bool, int, const int*, double**, const long*, const int*, int**, int, double**,
                                    const long*, int*, cudaStream_t, double*);
template int batched_factor<float>(bool, int, const int*, float**, const long*, const int*, int**, int, float**,
                                   const long*, int*, cudaStream_t, float*);

// Panel width per size bin: time every candidate width on a sample of each
// bin's sizes (a scratch batch of SPD / general matrices) and keep the
// fastest; bins are the orders 1-32, 33-64, 65-128, 129-256, 257-512.
int batched_tune(bool lu, bool f64, int samples_per_bin, double* times_out) {
  std::lock_guard<std::mutex> lk(g_nb_mu);
  NbTable& t = g_nb[lu ? 1 : 0][f64 ? 1 : 0];
  if (!nb_table(lu, f64)) return FLA_FAILURE;
  const int bins[6] = {1, 33, 65, 129, 257, 513};
  const int cands[4] = {8, 16, 24, 32};
  cudaStream_t st = ctx().stream;
  const size_t es = f64 ? 8 : 4;
  for (int b = 0; b < 5; ++b) {
    const int lo = bins[b], hi = bins[b + 1] - 1;
    const int cnt = std::max(1, samples_per_bin);
    std::vector<int> hn(cnt);
    size_t total = 0;
    for (int i = 0; i < cnt; ++i) {
      hn[i] = lo + (int)((long)(hi - lo) * i / std::max(1, cnt - 1));
      total += (size_t)hn[i] * hn[i];
    }
    // scratch: matrices (diagonally dominant: both factorizations succeed),
    // pointers, sizes, pivots, info
    char* buf = (char*)ws_get(WS_MISC2, total * es + (size_t)cnt * (8 * 3 + 8) + (size_t)cnt * hi * 4 + 4096);
    if (!buf) return FLA_FAILURE;
    std::vector<void*> hp(cnt), hpiv(cnt);
    std::vector<long> hld(cnt);
    size_t off = 0;
    char* mats = buf;
    char* meta = buf + ((total * es + 255) & ~(size_t)255);
    int* pivs = (int*)(meta + (size_t)cnt * 32 + 256);
    for (int i = 0; i < cnt; ++i) {
      hp[i] = mats + off * es;
      hpiv[i] = pivs + (size_t)i * hi;
      hld[i] = hn[i];
      off += (size_t)hn[i] * hn[i];
    }
    void** dA = (void**)meta;
    long* dld = (long*)(meta + (size_t)cnt * 8);
    int* dn = (int*)(meta + (size_t)cnt * 16);
    int* dinfo = (int*)(meta + (size_t)cnt * 20);
    void** dpiv = (void**)(meta + (size_t)cnt * 24);
    FB_CK(cudaMemcpy(dA, hp.data(), sizeof(void*) * cnt, cudaMemcpyHostToDevice));
    FB_CK(cudaMemcpy(dld, hld.data(), sizeof(long) * cnt, cudaMemcpyHostToDevice));
    FB_CK(cudaMemcpy(dn, hn.data(), sizeof(int) * cnt, cudaMemcpyHostToDevice));
    FB_CK(cudaMemcpy(dpiv, hpiv.data(), sizeof(void*) * cnt, cudaMemcpyHostToDevice));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    int bestnb = t.host[hi];
    for (int ci = 0; ci < 4; ++ci) {
      const int c = cands[ci];
      for (int nn = lo; nn <= hi; ++nn) t.host[nn] = c;
      FB_CK(cudaMemcpy(t.dev, t.host.data(), sizeof(int) * (BMAXN + 1), cudaMemcpyHostToDevice));
      float ms = 1e30f;
      for (int rep = 0; rep < 2; ++rep) {
        if (batched_fill_dominant(f64, cnt, dA, dn, dld, st) != FLA_SUCCESS) return FLA_FAILURE;
        cudaEventRecord(e0, st);
        int r = f64 ? batched_factor<double>(lu, cnt, hn.data(), (double**)dA, dld, dn, (int**)dpiv, 0, nullptr,
                                             nullptr, dinfo, st)
                    : batched_factor<float>(lu, cnt, hn.data(), (float**)dA, dld, dn, (int**)dpiv, 0, nullptr,
                                            nullptr, dinfo, st);
        if (r != FLA_SUCCESS) return FLA_FAILURE;
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float x = 0.f;
        cudaEventElapsedTime(&x, e0, e1);
        ms = std::min(ms, x);
      }
      if (times_out) times_out[b * 4 + ci] = ms;
      if (ms < best) {
        best = ms;
        bestnb = c;
      }
    }
    for (int nn = lo; nn <= hi; ++nn) t.host[nn] = bestnb;
    FB_CK(cudaMemcpy(t.dev, t.host.data(), sizeof(int) * (BMAXN + 1), cudaMemcpyHostToDevice));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  t.tuned = true;
  return FLA_SUCCESS;
}

int batched_nb(bool lu, bool f64, int n) {
  NbTable& t = g_nb[lu ? 1 : 0][f64 ? 1 : 0];
  if (t.host.empty()) nb_table(lu, f64);
  return t.host.empty() ? 0 : t.host[std::min(std::max(n, 0), BMAXN)];
}

// ---------------------------------------------------------------------------
// Diagonally dominant fill for the tuner's scratch matrices.
// ---------------------------------------------------------------------------
namespace {
template <typename T>
__global__ void fill_dominant_kernel(T** A, const int* n, const long* ld, int count) {
  const int m = blockIdx.x;
  if (m >= count) return;
  const int nn = n[m];
  T* G = A[m];
  for (int e = threadIdx.x; e < nn * nn; e += blockDim.x) {
    const int r = e % nn, c = e / nn;
    unsigned h = (unsigned)(r * 2654435761u) ^ (unsigned)(c * 2246822519u) ^ (unsigned)m;
    h ^= h >> 13;
    h *= 0x5bd1e995u;
    h ^= h >> 15;
    const T v = (T)((h & 0xffff) / 65536.0 - 0.5);
    G[r + (long)c * ld[m]] = (r == c) ? (T)(nn + 1) : (r > c ? v : (T)0.5 * v);
  }
}
}  // namespace

int batched_fill_dominant(bool f64, int count, void** dA, const int* dn, const long* dld, cudaStream_t st) {
  if (f64)
    fill_dominant_kernel<double><<<count, 256, 0, st>>>((double**)dA, dn, dld, count);
  else
    fill_dominant_kernel<float><<<count, 256, 0, st>>>((float**)dA, dn, dld, count);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

}  // namespace fb

// ===========================================================================
// C ABI (no counterpart in the reference).
// ===========================================================================
namespace {

template <typename T>
int batched_entry(bool lu, int count, const int* n, T** A, const int* lda, int** piv, int nrhs, T** B,
                  const int* ldb, int* info, T* logdet = nullptr) {
  using namespace fb;
  if (!ctx().initialized) FLA_Init();
  if (count < 0) {
    set_last_error("batched: count < 0");
    return FLA_FAILURE;
  }
  if (count == 0) return FLA_SUCCESS;
  if (nrhs < 0 || nrhs > BMAXRHS) {
    set_last_error("batched: nrhs must be 0.." + std::to_string(BMAXRHS));
    return FLA_FAILURE;
  }
  const int maxn = (!lu && sizeof(T) == 8) ? DMAXN : BMAXN;  // FP64 Cholesky: the DMMA kernel
  for (int i = 0; i < count; ++i) {
    if (n[i] < 0 || n[i] > maxn || lda[i] < std::max(1, n[i]) || (nrhs > 0 && ldb[i] < std::max(1, n[i]))) {
      set_last_error("batched: matrix " + std::to_string(i) + " has n outside 0.." + std::to_string(maxn) +
                     " or a short leading dimension");
      return FLA_FAILURE;
    }
    if (!is_device_ptr(A[i]) || (lu && !is_device_ptr(piv[i])) || (nrhs > 0 && !is_device_ptr(B[i]))) {
      set_last_error("batched: matrix " + std::to_string(i) + ": buffers must be device memory");
      return FLA_FAILURE;
    }
  }
  cudaStream_t st = ctx().stream;
  // device copies of the argument arrays
  const size_t c = (size_t)count;
  // layout: A, B, piv pointers, ld, ldb (8 bytes each), n, info (4 bytes each)
  char* m = (char*)ws_get(WS_MISC2, c * (8 * 6 + 4 * 2) + 1024);
  if (!m) return FLA_FAILURE;
  T* dlogdet = logdet ? (T*)(m + c * 48 + 512) : nullptr;  // after the int arrays
  T** dA = (T**)m;
  T** dB = (T**)(m + c * 8);
  int** dpiv = (int**)(m + c * 16);
  long* dld = (long*)(m + c * 24);
  long* dldb = (long*)(m + c * 32);
  int* dn = (int*)(m + c * 40);
  int* dinfo = (int*)(m + c * 44);
  std::vector<long> hld(count), hldb(count, 1);
  for (int i = 0; i < count; ++i) {
    hld[i] = lda[i];
    if (nrhs > 0) hldb[i] = ldb[i];
  }
  if (status_reset() != FLA_SUCCESS) return FLA_FAILURE;  // starts the op timing
  FB_CK(cudaMemcpyAsync(dA, A, sizeof(T*) * c, cudaMemcpyHostToDevice, st));
  if (nrhs > 0) FB_CK(cudaMemcpyAsync(dB, B, sizeof(T*) * c, cudaMemcpyHostToDevice, st));
  if (lu) FB_CK(cudaMemcpyAsync(dpiv, piv, sizeof(int*) * c, cudaMemcpyHostToDevice, st));
  FB_CK(cudaMemcpyAsync(dld, hld.data(), sizeof(long) * c, cudaMemcpyHostToDevice, st));
  FB_CK(cudaMemcpyAsync(dldb, hldb.data(), sizeof(long) * c, cudaMemcpyHostToDevice, st));
  FB_CK(cudaMemcpyAsync(dn, n, sizeof(int) * c, cudaMemcpyHostToDevice, st));
  if (batched_factor<T>(lu, count, n, dA, dld, dn, lu ? dpiv : nullptr, nrhs, nrhs > 0 ? dB : nullptr, dldb, dinfo,
                        st, dlogdet) != FLA_SUCCESS)
    return FLA_FAILURE;
  FB_CK(cudaMemcpyAsync(info, dinfo, sizeof(int) * c, cudaMemcpyDeviceToHost, st));
  if (logdet) FB_CK(cudaMemcpyAsync(logdet, dlogdet, sizeof(T) * c, cudaMemcpyDeviceToHost, st));
  // ends the op timing; a wait that ran out makes the call fail
  if (status_read(nullptr) != FLA_SUCCESS) return FLA_FAILURE;
  return sync_all();
}

}  // namespace

extern "C" {

// Lower Cholesky of `count` matrices A[i] (device, column-major, order n[i]
// <= 512, leading dimension lda[i]); info[i] (host) receives FLA_SUCCESS or
// the zero-based failing column, as FLA_Chol.  With nrhs > 0 (<= 8) each
// B[i] (n[i] x nrhs, ldb[i]) is overwritten by the solution of A X = B in
// the same launch (matrices that fail are not solved).
FLA_Error FLA_Chol_batched(FLA_Uplo uplo, int count, const int* n, double** A, const int* lda, int nrhs, double** B,
                           const int* ldb, int* info) {
  if (uplo != FLA_LOWER_TRIANGULAR) {
    fb::set_last_error("FLA_Chol_batched: only FLA_LOWER_TRIANGULAR is provided");
    return FLA_FAILURE;
  }
  return batched_entry<double>(false, count, n, A, lda, nullptr, nrhs, B, ldb, info);
}
// No counterpart in the reference.  FLA_Chol_batched (FP64, lower) that also
// returns logdet[i] = sum_j log L_i(j, j) (host array of count doubles;
// NaN for matrices that fail), for batches of Gaussian-process likelihoods.
FLA_Error FLA_B200_Chol_batched_logdet(int count, const int* n, double** A, const int* lda, int nrhs, double** B,
                                       const int* ldb, double* logdet, int* info) {
  if (!logdet && count > 0) {
    fb::set_last_error("FLA_B200_Chol_batched_logdet: logdet is null");
    return FLA_FAILURE;
  }
  return batched_entry<double>(false, count, n, A, lda, nullptr, nrhs, B, ldb, info, logdet);
}
FLA_Error FLA_B200_Chol_batched_f32(int count, const int* n, float** A, const int* lda, int nrhs, float** B,
                                    const int* ldb, int* info) {
  return batched_entry<float>(false, count, n, A, lda, nullptr, nrhs, B, ldb, info);
}
// LU with partial pivoting of `count` square matrices; piv[i] (device, n[i]
// ints) receives relative pivots as FLA_LU_piv; info[i] FLA_SUCCESS or the
// first zero-pivot column.  nrhs > 0: B[i] := A^-1 B[i] in the same launch.
FLA_Error FLA_LU_piv_batched(int count, const int* n, double** A, const int* lda, int** piv, int nrhs, double** B,
                             const int* ldb, int* info) {
  return batched_entry<double>(true, count, n, A, lda, piv, nrhs, B, ldb, info);
}
FLA_Error FLA_B200_LU_piv_batched_f32(int count, const int* n, float** A, const int* lda, int** piv, int nrhs,
                                      float** B, const int* ldb, int* info) {
  return batched_entry<float>(true, count, n, A, lda, piv, nrhs, B, ldb, info);
}
// Autotuner of the batched kernels: for each size bin (orders 1-32, 33-64,
// 65-128, 129-256, 257-512) times the panel widths 8, 16, 24, 32 on
// `samples` scratch matrices and keeps the fastest for later calls on this
// device.  times (optional, 20 doubles) receives the bin x width timings
// in ms.
int FLA_B200_batched_tune(int lu, int f64, int samples, double* times) {
  if (!fb::ctx().initialized) FLA_Init();
  return fb::batched_tune(lu != 0, f64 != 0, samples, times);
}
// Panel width the batched kernels use for order n.
int FLA_B200_batched_nb(int lu, int f64, int n) {
  if (!fb::ctx().initialized) FLA_Init();
  return fb::batched_nb(lu != 0, f64 != 0, n);
}

}  // extern "C"
