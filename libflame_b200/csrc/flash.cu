// FLASH hierarchical (storage-by-blocks) objects and the FLASH front-ends of
// the factorizations: FLASH users drop in by flattening to HBM and running
// the same kernels as the FLA_* entry points.
//
// Reference: objects src/base/flamec/hierarchy/main/FLASH_Obj.c
// (FLASH_Obj_create_helper :175-270: depth 0 is a plain FLA_Obj; otherwise
// a top object of element type FLA_MATRIX whose buffer holds the leaf
// objects, the leaves' storage carved out of one allocation), copies
// FLASH_Copy_other.c:81-139, views FLASH_View.c:600-750; front-ends
// src/lapack/dec/chol/front/flamec/FLASH_Chol.c:15-30,
// src/lapack/dec/lu/piv/front/flamec/FLASH_LU_piv.c:15-41 (depth 1 only),
// src/lapack/dec/q/qrut/front/flamec/FLASH_QR_UT.c (depth 1, b_alg ==
// b_flash, min_dim % b_flash == 0), FLASH_QR_UT_create_hier_matrices.c,
// FLASH_QR_UT_solve.c, and the algorithm-by-blocks' placement of each
// block column's T in the diagonal block TW(j, j)
// (src/lapack/dec/q/qrut/vars/flamec/FLA_QR_UT_blk_var3.c).
//
// Here hierarchies have depth 1 (what the LU and QR front-ends of the
// reference accept; the Cholesky's depth > 1 is rejected with a message).
// An m x n object with b_m x b_n blocks is an nbm x nbn grid of leaves (the
// last row and column of blocks smaller) stored in one HBM allocation: the
// leaves one after another in column-major block order, each column-major
// with its own row count as leading dimension, so element (i, j) lies at
//   m (bj b_n) + (bi b_m) w(bj) + (i - bi b_m) + (j - bj b_n) r(bi)
// with bi = i / b_m, bj = j / b_n, r(bi) the block's rows and w(bj) its
// columns.  A front-end gathers the blocks into a column-major HBM copy
// (one kernel), calls the flat entry point on it, and scatters the result
// back; the SuperMatrix task queue of the reference has no counterpart
// (the flat GPU path already overlaps panels with updates).
#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "common.h"

namespace fb {

namespace {

size_t elem_size(FLA_Datatype dt) {
  switch (dt) {
    case FLA_DOUBLE: return 8;
    case FLA_FLOAT: return 4;
    case FLA_INT: return 4;
    default: return 0;
  }
}

bool is_hier(const FLA_Obj& H) { return H.base && H.base->elemtype == FLA_MATRIX; }

// Geometry of a depth-1 hierarchical object.
struct Hier {
  void* storage = nullptr;
  long m = 0, n = 0;    // scalar size
  long bm = 1, bn = 1;  // block size
  size_t es = 0;
  FLA_Datatype dt = FLA_DOUBLE;
};

bool hier_of(const FLA_Obj& H, Hier* h) {
  if (!is_hier(H)) return false;
  const FLA_Obj* leaves = static_cast<const FLA_Obj*>(H.base->buffer);
  h->m = (long)H.base->m_inner;
  h->n = (long)H.base->n_inner;
  h->dt = H.base->datatype;
  h->es = elem_size(h->dt);
  if (H.base->m == 0 || H.base->n == 0 || !leaves) {
    h->storage = nullptr;
    return true;
  }
  h->storage = leaves[0].base->buffer;
  h->bm = std::max<long>(1, (long)leaves[0].m);
  h->bn = std::max<long>(1, (long)leaves[0].n);
  return true;
}

// F (mf x nf window, ld ldf, device) <-> the window at scalar offset
// (i0, j0) of the hierarchical storage H.
template <typename T>
__global__ void hier_copy_kernel(T* __restrict__ H, long m, long n, long bm, long bn, T* __restrict__ F, long ldf,
                                 long i0, long j0, long mf, long nf, int to_flat) {
  const long total = mf * nf;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long ii = e % mf, jj = e / mf;
    const long i = i0 + ii, j = j0 + jj;
    const long bi = i / bm, bj = j / bn;
    const long rows = min(bm, m - bi * bm), wj = min(bn, n - bj * bn);
    const long off = m * bj * bn + bi * bm * wj + (i - bi * bm) + (j - bj * bn) * rows;
    if (to_flat) F[ii + jj * ldf] = H[off];
    else H[off] = F[ii + jj * ldf];
  }
}

int hier_copy(const Hier& h, void* F, long ldf, long i0, long j0, long mf, long nf, bool to_flat, cudaStream_t st) {
  if (mf <= 0 || nf <= 0) return FLA_SUCCESS;
  const unsigned grid = (unsigned)std::min<long>(4L * ctx().num_sms, (mf * nf + 255) / 256);
  if (h.es == 8)
    hier_copy_kernel<double><<<grid, 256, 0, st>>>((double*)h.storage, h.m, h.n, h.bm, h.bn, (double*)F, ldf, i0, j0,
                                                   mf, nf, to_flat ? 1 : 0);
  else
    hier_copy_kernel<float><<<grid, 256, 0, st>>>((float*)h.storage, h.m, h.n, h.bm, h.bn, (float*)F, ldf, i0, j0, mf,
                                                  nf, to_flat ? 1 : 0);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// A column-major HBM copy of a hierarchical object (or a plain view of a
// flat one), as an FLA_Obj the flat entry points accept.
struct Flat {
  FLA_Obj obj{};
  bool own_view = false;
  Hier h;
  bool hier = false;
  void* p = nullptr;
  long ld = 0;
};

int flat_in(const FLA_Obj& X, int slot, bool copy, Flat* f) {
  if (!is_hier(X)) {
    f->obj = X;
    f->hier = false;
    return FLA_SUCCESS;
  }
  f->hier = true;
  hier_of(X, &f->h);
  const long m = f->h.m, n = f->h.n;
  f->ld = std::max<long>(1, (m + 1) & ~1L);  // even: 16-byte aligned columns for the TMA paths
  f->p = ws_get(slot, f->h.es * (size_t)f->ld * (size_t)std::max<long>(n, 1));
  if (!f->p) return FLA_FAILURE;
  if (copy && hier_copy(f->h, f->p, f->ld, 0, 0, m, n, true, ctx().stream) != FLA_SUCCESS) return FLA_FAILURE;
  FLA_Obj_create_without_buffer(f->h.dt, (dim_t)m, (dim_t)n, &f->obj);
  FLA_Obj_attach_buffer(f->p, 1, (dim_t)f->ld, &f->obj);
  f->own_view = true;
  return FLA_SUCCESS;
}

int flat_out(Flat* f, bool copy_back) {
  int r = FLA_SUCCESS;
  if (f->hier && copy_back)
    r = hier_copy(f->h, f->p, f->ld, 0, 0, f->h.m, f->h.n, false, ctx().stream);
  if (f->own_view) FLA_Obj_free_without_buffer(&f->obj);
  f->own_view = false;
  if (r == FLA_SUCCESS) r = sync_all();
  return r;
}

// Flat T (b x k, ld ldt) <-> the diagonal b x b blocks of a hierarchical TW
// (the upper triangles; block q holds T's columns q b .. q b + b - 1).
template <int TO_TW>
__global__ void tw_diag_kernel(double* __restrict__ TW, long m, long n, long b, double* __restrict__ T, long ldt,
                               long k) {
  const long total = b * k;
  for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const long r = e % b, c = e / b;
    const long q = c / b, cc = c - q * b;
    if (r > cc) continue;
    const long i = q * b + r, j = c;  // element (i, j) of TW (diagonal block q)
    const long bi = i / b, bj = j / b;
    const long rows = min(b, m - bi * b), wj = min(b, n - bj * b);
    const long off = m * bj * b + bi * b * wj + (i - bi * b) + (j - bj * b) * rows;
    if (TO_TW) TW[off] = T[r + c * ldt];
    else T[r + c * ldt] = TW[off];
  }
}

int tw_diag(const Hier& tw, double* T, long ldt, long k, bool to_tw) {
  const long total = tw.bm * k;
  if (total <= 0) return FLA_SUCCESS;
  const unsigned grid = (unsigned)std::min<long>(4L * ctx().num_sms, (total + 255) / 256);
  if (to_tw)
    tw_diag_kernel<1><<<grid, 256, 0, ctx().stream>>>((double*)tw.storage, tw.m, tw.n, tw.bm, T, ldt, k);
  else
    tw_diag_kernel<0><<<grid, 256, 0, ctx().stream>>>((double*)tw.storage, tw.m, tw.n, tw.bm, T, ldt, k);
  count_launch();
  FB_CK(cudaGetLastError());
  return FLA_SUCCESS;
}

// Flat T (b_alg x n) for the entry points from a hierarchical TW: the
// diagonal blocks' upper triangles for the first k columns, zero elsewhere.
int t_from_tw(const FLA_Obj& TW, long k, long n, Flat* T) {
  Hier tw;
  hier_of(TW, &tw);
  const long b = tw.bm;
  T->hier = false;
  T->ld = std::max<long>(2, (b + 1) & ~1L);
  const size_t bytes = sizeof(double) * (size_t)T->ld * (size_t)std::max<long>(n, 1);
  T->p = ws_get(WS_FLASH3, bytes);
  if (!T->p) return FLA_FAILURE;
  FB_CK(cudaMemsetAsync(T->p, 0, bytes, ctx().stream));
  if (tw_diag(tw, (double*)T->p, T->ld, k, false) != FLA_SUCCESS) return FLA_FAILURE;
  FLA_Obj_create_without_buffer(FLA_DOUBLE, (dim_t)b, (dim_t)n, &T->obj);
  FLA_Obj_attach_buffer(T->p, 1, (dim_t)T->ld, &T->obj);
  T->own_view = true;
  return FLA_SUCCESS;
}

bool depth1(const FLA_Obj& H) {
  if (!is_hier(H)) return false;
  const FLA_Obj* leaves = static_cast<const FLA_Obj*>(H.base->buffer);
  return !leaves || H.base->m == 0 || H.base->n == 0 || !is_hier(leaves[0]);
}

bool whole(const FLA_Obj& H) {
  return H.offm == 0 && H.offn == 0 && H.m == H.base->m && H.n == H.base->n;
}

}  // namespace

}  // namespace fb

using namespace fb;

extern "C" {

// FLASH_Obj.c:20-47: the number of FLA_MATRIX levels above the leaves.
dim_t FLASH_Obj_depth(FLA_Obj H) {
  dim_t d = 0;
  FLA_Obj X = H;
  while (is_hier(X) && X.base->m > 0 && X.base->n > 0) {
    ++d;
    X = static_cast<const FLA_Obj*>(X.base->buffer)[0];
  }
  return d;
}

// FLASH_Obj.c:49-81: the leaf blocksizes of the top-left block, per level.
dim_t FLASH_Obj_blocksizes(FLA_Obj H, dim_t* b_m, dim_t* b_n) {
  const dim_t d = FLASH_Obj_depth(H);
  Hier h;
  if (d >= 1 && hier_of(H, &h)) {
    if (b_m) b_m[0] = (dim_t)h.bm;
    if (b_n) b_n[0] = (dim_t)h.bn;
  }
  return d;
}

// FLASH_View.c:600-690: scalar dimensions of a (whole) object.
dim_t FLASH_Obj_scalar_length(FLA_Obj H) { return is_hier(H) ? H.base->m_inner : H.m; }
dim_t FLASH_Obj_scalar_width(FLA_Obj H) { return is_hier(H) ? H.base->n_inner : H.n; }
dim_t FLASH_Obj_scalar_min_dim(FLA_Obj H) {
  return std::min(FLASH_Obj_scalar_length(H), FLASH_Obj_scalar_width(H));
}
dim_t FLASH_Obj_scalar_max_dim(FLA_Obj H) {
  return std::max(FLASH_Obj_scalar_length(H), FLASH_Obj_scalar_width(H));
}

// FLASH_Obj.c:151-270: depth 0 is a plain FLA_Obj_create; depth 1 here (the
// leaves' storage one HBM allocation, zeroed).
FLA_Error FLASH_Obj_create_ext(FLA_Datatype datatype, dim_t m, dim_t n, dim_t depth, dim_t* b_m, dim_t* b_n,
                               FLA_Obj* H) {
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(H != nullptr, "FLASH_Obj_create", "null object pointer");
  if (depth == 0) return FLA_Obj_create(datatype, m, n, 0, 0, H);
  FB_REQUIRE(depth == 1, "FLASH_Obj_create", "only hierarchies of depth 1 are supported");
  FB_REQUIRE(b_m && b_n && b_m[0] > 0 && b_n[0] > 0, "FLASH_Obj_create", "blocksizes must be positive");
  const size_t es = elem_size(datatype);
  FB_REQUIRE(es > 0, "FLASH_Obj_create", "datatype must be FLA_DOUBLE, FLA_FLOAT or FLA_INT");
  const dim_t bm = b_m[0], bn = b_n[0];
  const dim_t nbm = (m + bm - 1) / bm, nbn = (n + bn - 1) / bn;
  void* storage = nullptr;
  if (m > 0 && n > 0) {
    if (cudaMalloc(&storage, es * (size_t)m * (size_t)n) != cudaSuccess) {
      cudaGetLastError();
      set_last_error("FLASH_Obj_create: cudaMalloc failed");
      return FLA_FAILURE;
    }
    FB_CK(cudaMemset(storage, 0, es * (size_t)m * (size_t)n));
  }
  FLA_Obj_create_without_buffer(datatype, nbm, nbn, H);
  FLA_Base_obj* top = H->base;
  top->elemtype = FLA_MATRIX;
  top->m_inner = m;
  top->n_inner = n;
  top->rs = 1;
  top->cs = nbm > 0 ? nbm : 1;
  H->m_inner = m;
  H->n_inner = n;
  FLA_Obj* leaves = (nbm > 0 && nbn > 0) ? new FLA_Obj[(size_t)nbm * nbn] : nullptr;
  for (dim_t bj = 0; bj < nbn; ++bj) {
    const dim_t w = std::min(bn, n - bj * bn);
    for (dim_t bi = 0; bi < nbm; ++bi) {
      const dim_t r = std::min(bm, m - bi * bm);
      const size_t off = (size_t)m * bj * bn + (size_t)bi * bm * w;
      FLA_Obj& L = leaves[bi + bj * nbm];
      FLA_Obj_create_without_buffer(datatype, r, w, &L);
      FLA_Obj_attach_buffer(static_cast<char*>(storage) + es * off, 1, r, &L);
      L.base->m_index = bi;
      L.base->n_index = bj;
    }
  }
  top->buffer = leaves;
  return FLA_SUCCESS;
}

FLA_Error FLASH_Obj_create(FLA_Datatype datatype, dim_t m, dim_t n, dim_t depth, dim_t* b_mn, FLA_Obj* H) {
  return FLASH_Obj_create_ext(datatype, m, n, depth, b_mn, b_mn, H);
}

// FLASH_Obj.c:638-700.
void FLASH_Obj_free(FLA_Obj* H) {
  if (!H || !H->base) return;
  if (!is_hier(*H)) {
    FLA_Obj_free(H);
    return;
  }
  FLA_Obj* leaves = static_cast<FLA_Obj*>(H->base->buffer);
  const size_t cnt = (size_t)H->base->m * H->base->n;
  if (leaves && cnt > 0) {
    cudaDeviceSynchronize();
    cudaFree(leaves[0].base->buffer);
    for (size_t q = 0; q < cnt; ++q) FLA_Obj_free_without_buffer(&leaves[q]);
    delete[] leaves;
  }
  H->base->buffer = nullptr;
  FLA_Obj_free_without_buffer(H);
}

// FLASH_Copy_other.c:81-136: F (flat, host or device) <-> the window of H
// at scalar offset (i, j) with F's size.
FLA_Error FLASH_Copy_flat_to_hier(FLA_Obj F, dim_t i, dim_t j, FLA_Obj H) {
  if (!ctx().initialized) FLA_Init();
  Hier h;
  FB_REQUIRE(hier_of(H, &h) && depth1(H), "FLASH_Copy_flat_to_hier", "H must be a hierarchical object of depth 1");
  FB_REQUIRE(!is_hier(F) && F.base && F.base->datatype == h.dt, "FLASH_Copy_flat_to_hier",
             "F must be a flat object of H's datatype");
  FB_REQUIRE((long)(i + F.m) <= h.m && (long)(j + F.n) <= h.n, "FLASH_Copy_flat_to_hier", "F does not fit in H");
  Staged s;
  if (stage(F, WS_STAGE_A, &s, true, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (hier_copy(h, s.dev, s.ld, (long)i, (long)j, (long)F.m, (long)F.n, false, ctx().stream) != FLA_SUCCESS)
    return FLA_FAILURE;
  return sync_all();
}

FLA_Error FLASH_Copy_hier_to_flat(dim_t i, dim_t j, FLA_Obj H, FLA_Obj F) {
  if (!ctx().initialized) FLA_Init();
  Hier h;
  FB_REQUIRE(hier_of(H, &h) && depth1(H), "FLASH_Copy_hier_to_flat", "H must be a hierarchical object of depth 1");
  FB_REQUIRE(!is_hier(F) && F.base && F.base->datatype == h.dt, "FLASH_Copy_hier_to_flat",
             "F must be a flat object of H's datatype");
  FB_REQUIRE((long)(i + F.m) <= h.m && (long)(j + F.n) <= h.n, "FLASH_Copy_hier_to_flat", "F does not fit in H");
  Staged s;
  if (stage(F, WS_STAGE_A, &s, false, false) != FLA_SUCCESS) return FLA_FAILURE;
  if (hier_copy(h, s.dev, s.ld, (long)i, (long)j, (long)F.m, (long)F.n, true, ctx().stream) != FLA_SUCCESS)
    return FLA_FAILURE;
  if (unstage(s) != FLA_SUCCESS) return FLA_FAILURE;
  return sync_all();
}

// FLASH_Obj.c:765-780.
FLA_Error FLASH_Obj_flatten(FLA_Obj H, FLA_Obj F) { return FLASH_Copy_hier_to_flat(0, 0, H, F); }
FLA_Error FLASH_Obj_hierarchify(FLA_Obj F, FLA_Obj H) { return FLASH_Copy_flat_to_hier(F, 0, 0, H); }

// FLASH_Obj.c:591-636.
FLA_Error FLASH_Obj_create_hier_copy_of_flat_ext(FLA_Obj F, dim_t depth, dim_t* b_m, dim_t* b_n, FLA_Obj* H) {
  FB_REQUIRE(F.base && !is_hier(F), "FLASH_Obj_create_hier_copy_of_flat", "F must be a flat object");
  if (FLASH_Obj_create_ext(F.base->datatype, F.m, F.n, depth, b_m, b_n, H) != FLA_SUCCESS) return FLA_FAILURE;
  if (depth == 0) {
    Staged s;
    if (stage(F, WS_STAGE_A, &s, true, false) != FLA_SUCCESS) return FLA_FAILURE;
    if (F.m > 0 && F.n > 0)
      FB_CK(cudaMemcpy2DAsync(H->base->buffer, H->base->cs * s.esize, s.dev, s.ld * s.esize, F.m * s.esize, F.n,
                              cudaMemcpyDeviceToDevice, ctx().stream));
    return sync_all();
  }
  return FLASH_Copy_flat_to_hier(F, 0, 0, *H);
}

FLA_Error FLASH_Obj_create_hier_copy_of_flat(FLA_Obj F, dim_t depth, dim_t* b_mn, FLA_Obj* H) {
  return FLASH_Obj_create_hier_copy_of_flat_ext(F, depth, b_mn, b_mn, H);
}

FLA_Error FLASH_Obj_create_flat_copy_of_hier(FLA_Obj H, FLA_Obj* F) {
  Hier h;
  FB_REQUIRE(hier_of(H, &h) && depth1(H), "FLASH_Obj_create_flat_copy_of_hier",
             "H must be a hierarchical object of depth 1");
  if (FLA_Obj_create(h.dt, (dim_t)h.m, (dim_t)h.n, 0, 0, F) != FLA_SUCCESS) return FLA_FAILURE;
  return FLASH_Copy_hier_to_flat(0, 0, H, *F);
}

// src/lapack/dec/chol/front/flamec/FLASH_Chol.c:15-30: same return values
// as FLA_Chol (the failing column, or FLA_SUCCESS).
FLA_Error FLASH_Chol(FLA_Uplo uplo, FLA_Obj A) {
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(is_hier(A) && depth1(A) && whole(A), "FLASH_Chol",
             "A must be a whole hierarchical object of depth 1");
  Flat fa;
  if (flat_in(A, WS_FLASH0, true, &fa) != FLA_SUCCESS) return FLA_FAILURE;
  const FLA_Error r = FLA_Chol(uplo, fa.obj);
  if (flat_out(&fa, true) != FLA_SUCCESS) return FLA_FAILURE;
  return r;
}

// src/lapack/dec/chol/front/flamec/FLASH_Chol_solve.c.
FLA_Error FLASH_Chol_solve(FLA_Uplo uplo, FLA_Obj A, FLA_Obj B, FLA_Obj X) {
  if (!ctx().initialized) FLA_Init();
  Flat fa, fb_, fx;
  if (flat_in(A, WS_FLASH0, true, &fa) != FLA_SUCCESS || flat_in(B, WS_FLASH1, true, &fb_) != FLA_SUCCESS ||
      flat_in(X, WS_FLASH2, false, &fx) != FLA_SUCCESS)
    return FLA_FAILURE;
  const FLA_Error r = FLA_Chol_solve(uplo, fa.obj, fb_.obj, fx.obj);
  if (flat_out(&fa, false) != FLA_SUCCESS || flat_out(&fb_, false) != FLA_SUCCESS ||
      flat_out(&fx, r == FLA_SUCCESS) != FLA_SUCCESS)
    return FLA_FAILURE;
  return r;
}

// src/lapack/dec/lu/piv/front/flamec/FLASH_LU_piv.c:15-41: depth 1; p may be
// hierarchical (blocks of one column) or flat; returns as FLA_LU_piv.
FLA_Error FLASH_LU_piv(FLA_Obj A, FLA_Obj p) {
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(is_hier(A) && depth1(A) && whole(A), "FLASH_LU_piv",
             "FLASH_LU_piv() currently only supports matrices of depth 1");
  Flat fa, fp;
  if (flat_in(A, WS_FLASH0, true, &fa) != FLA_SUCCESS || flat_in(p, WS_FLASH1, true, &fp) != FLA_SUCCESS)
    return FLA_FAILURE;
  const FLA_Error r = FLA_LU_piv(fa.obj, fp.obj);
  if (flat_out(&fa, true) != FLA_SUCCESS || flat_out(&fp, true) != FLA_SUCCESS) return FLA_FAILURE;
  return r;
}

// src/lapack/dec/lu/piv/front/flamec/FLASH_LU_piv_solve.c.
FLA_Error FLASH_LU_piv_solve(FLA_Obj A, FLA_Obj p, FLA_Obj B, FLA_Obj X) {
  if (!ctx().initialized) FLA_Init();
  Flat fa, fp, fb_, fx;
  if (flat_in(A, WS_FLASH0, true, &fa) != FLA_SUCCESS || flat_in(p, WS_FLASH1, true, &fp) != FLA_SUCCESS ||
      flat_in(B, WS_FLASH2, true, &fb_) != FLA_SUCCESS || flat_in(X, WS_FLASH3, false, &fx) != FLA_SUCCESS)
    return FLA_FAILURE;
  const FLA_Error r = FLA_LU_piv_solve(fa.obj, fp.obj, fb_.obj, fx.obj);
  if (flat_out(&fa, false) != FLA_SUCCESS || flat_out(&fp, false) != FLA_SUCCESS ||
      flat_out(&fb_, false) != FLA_SUCCESS || flat_out(&fx, r == FLA_SUCCESS) != FLA_SUCCESS)
    return FLA_FAILURE;
  return r;
}

// src/lapack/dec/q/qrut/front/flamec/FLASH_QR_UT_create_hier_matrices.c:
// A := hierarchical copy of A_flat; TW: min_dim x min_dim with b_flash
// blocks (depth 1).
FLA_Error FLASH_QR_UT_create_hier_matrices(FLA_Obj A_flat, dim_t depth, dim_t* b_flash, FLA_Obj* A, FLA_Obj* TW) {
  FB_REQUIRE(depth == 1, "FLASH_QR_UT_create_hier_matrices", "FLASH_QR_UT() currently only supports matrices of depth 1");
  if (FLASH_Obj_create_hier_copy_of_flat(A_flat, depth, b_flash, A) != FLA_SUCCESS) return FLA_FAILURE;
  const dim_t mn = std::min(A_flat.m, A_flat.n);
  return FLASH_Obj_create_ext(A_flat.base->datatype, mn, mn, depth, b_flash, b_flash, TW);
}

// src/lapack/dec/q/qrut/front/flamec/FLASH_QR_UT.c: depth 1, the blocks of
// TW square (b_alg == b_flash) and min_dim(A) a multiple of them; the T of
// block column q goes to TW's diagonal block (q, q), as the
// algorithm-by-blocks (FLA_QR_UT_blk_var3) stores it.
FLA_Error FLASH_QR_UT(FLA_Obj A, FLA_Obj TW) {
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(is_hier(A) && depth1(A) && whole(A) && is_hier(TW) && depth1(TW), "FLASH_QR_UT",
             "FLASH_QR_UT() currently only supports matrices of depth 1");
  Hier tw;
  hier_of(TW, &tw);
  FB_REQUIRE(tw.bm == tw.bn, "FLASH_QR_UT", "FLASH_QR_UT() requires that b_alg == b_store");
  const long b = tw.bm, mn = (long)FLASH_Obj_scalar_min_dim(A);
  FB_REQUIRE(mn % b == 0, "FLASH_QR_UT", "FLASH_QR_UT() requires that min_dim( A ) % b_store == 0");
  FB_REQUIRE(tw.m >= mn && tw.n >= mn, "FLASH_QR_UT", "TW must be at least min_dim(A) x min_dim(A)");
  Flat fa, ft;
  if (flat_in(A, WS_FLASH0, true, &fa) != FLA_SUCCESS) return FLA_FAILURE;
  const long n = (long)FLASH_Obj_scalar_width(A);
  ft.ld = std::max<long>(2, (b + 1) & ~1L);
  ft.p = ws_get(WS_FLASH3, sizeof(double) * (size_t)ft.ld * (size_t)std::max<long>(n, 1));
  if (!ft.p) return FLA_FAILURE;
  FLA_Obj_create_without_buffer(FLA_DOUBLE, (dim_t)b, (dim_t)n, &ft.obj);
  FLA_Obj_attach_buffer(ft.p, 1, (dim_t)ft.ld, &ft.obj);
  ft.own_view = true;
  const FLA_Error r = FLA_QR_UT(fa.obj, ft.obj);
  if (r == FLA_SUCCESS && tw_diag(tw, (double*)ft.p, ft.ld, mn, true) != FLA_SUCCESS) return FLA_FAILURE;
  if (flat_out(&fa, true) != FLA_SUCCESS || flat_out(&ft, false) != FLA_SUCCESS) return FLA_FAILURE;
  return r;
}

// src/lapack/util/app/qut/front/flamec/FLASH_Apply_Q_UT.c: the sides and
// directions of FLA_Apply_Q_UT; T from TW's diagonal blocks.
FLA_Error FLASH_Apply_Q_UT(FLA_Side side, FLA_Trans trans, FLA_Direct direct, FLA_Store storev, FLA_Obj A, FLA_Obj TW,
                           FLA_Obj W, FLA_Obj B) {
  (void)W;
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(is_hier(A) && depth1(A) && is_hier(TW) && depth1(TW), "FLASH_Apply_Q_UT",
             "A and TW must be hierarchical objects of depth 1");
  Flat fa, ft, fb_;
  const long k = (long)FLASH_Obj_scalar_min_dim(A);
  if (flat_in(A, WS_FLASH0, true, &fa) != FLA_SUCCESS ||
      t_from_tw(TW, k, (long)FLASH_Obj_scalar_width(A), &ft) != FLA_SUCCESS ||
      flat_in(B, WS_FLASH1, true, &fb_) != FLA_SUCCESS)
    return FLA_FAILURE;
  const FLA_Error r = FLA_Apply_Q_UT(side, trans, direct, storev, fa.obj, ft.obj, ft.obj, fb_.obj);
  if (flat_out(&fa, false) != FLA_SUCCESS || flat_out(&ft, false) != FLA_SUCCESS ||
      flat_out(&fb_, r == FLA_SUCCESS) != FLA_SUCCESS)
    return FLA_FAILURE;
  return r;
}

// src/lapack/util/app/qut/front/flamec/FLASH_Apply_Q_UT_create_workspace.c:
// a hierarchical b_alg x width(B) object (the GPU path keeps its own
// workspace; W is accepted for interface compatibility).
FLA_Error FLASH_Apply_Q_UT_create_workspace(FLA_Obj TW, FLA_Obj B, FLA_Obj* W) {
  Hier tw;
  FB_REQUIRE(hier_of(TW, &tw), "FLASH_Apply_Q_UT_create_workspace", "TW must be hierarchical");
  dim_t bs = (dim_t)tw.bm;
  return FLASH_Obj_create_ext(FLA_DOUBLE, bs, std::max<dim_t>(1, FLASH_Obj_scalar_width(B)), 1, &bs, &bs, W);
}

// src/lapack/dec/q/qrut/front/flamec/FLASH_QR_UT_solve.c: the least-squares
// solution from FLASH_QR_UT's factor.
FLA_Error FLASH_QR_UT_solve(FLA_Obj A, FLA_Obj TW, FLA_Obj B, FLA_Obj X) {
  if (!ctx().initialized) FLA_Init();
  FB_REQUIRE(is_hier(A) && depth1(A) && is_hier(TW) && depth1(TW), "FLASH_QR_UT_solve",
             "A and TW must be hierarchical objects of depth 1");
  Flat fa, ft, fb_, fx;
  const long k = (long)FLASH_Obj_scalar_min_dim(A);
  if (flat_in(A, WS_FLASH0, true, &fa) != FLA_SUCCESS ||
      t_from_tw(TW, k, (long)FLASH_Obj_scalar_width(A), &ft) != FLA_SUCCESS ||
      flat_in(B, WS_FLASH1, true, &fb_) != FLA_SUCCESS || flat_in(X, WS_FLASH2, false, &fx) != FLA_SUCCESS)
    return FLA_FAILURE;
  const FLA_Error r = FLA_QR_UT_solve(fa.obj, ft.obj, fb_.obj, fx.obj);
  if (flat_out(&fa, false) != FLA_SUCCESS || flat_out(&ft, false) != FLA_SUCCESS ||
      flat_out(&fb_, false) != FLA_SUCCESS || flat_out(&fx, r == FLA_SUCCESS) != FLA_SUCCESS)
    return FLA_FAILURE;
  return r;
}

}  // extern "C"
