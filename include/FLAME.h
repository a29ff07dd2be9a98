/*
 * FLAME.h -- public C interface of libflame_b200, a B200-native (sm_100a)
 * implementation of libflame's blocked dense factorizations and solves.
 *
 * This header is a drop-in for the subset of the reference libflame 5.2.0
 * API that the dense-factorization path uses: the type names, constant
 * values, the FLA_Obj view layout and every function signature below are
 * the reference's, so a C program written against the reference FLAME.h
 * compiles and links against libflame_b200.so unchanged for these calls.
 * Each declaration cites the reference file (path within the libflame
 * project) whose interface it replaces.
 *
 * Differences in behaviour, all on the device side:
 *   - FLA_Obj_create allocates the buffer in GPU memory (HBM);
 *   - FLA_Obj_attach_buffer accepts a host pointer or a device pointer and
 *     detects which at call time; operations on host buffers copy to HBM,
 *     run on the GPU and copy back before returning;
 *   - every operation is synchronous at return (results are in place).
 * Only FLA_DOUBLE (and FLA_FLOAT where stated) column-major objects
 * (row stride 1) are supported; anything else is rejected by the argument
 * checks with the reference's abort semantics.
 */
#ifndef LIBFLAME_B200_FLAME_H
#define LIBFLAME_B200_FLAME_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- types: src/base/flamec/include/FLA_type_defs.h:38-70 -------------- */
typedef int FLA_Bool;
typedef int FLA_Error;
typedef int FLA_Quadrant;
typedef int FLA_Datatype;
typedef int FLA_Elemtype;
typedef int FLA_Side;
typedef int FLA_Uplo;
typedef int FLA_Trans;
typedef int FLA_Conj;
typedef int FLA_Diag;
typedef int FLA_Dimension;
typedef int FLA_Pivot_type;
typedef int FLA_Direct;
typedef int FLA_Store;
typedef int FLA_Matrix_type;
typedef int FLA_Precision;
typedef int FLA_Domain;
typedef int FLA_Inv;
#ifndef _DEFINED_DIM_T
#define _DEFINED_DIM_T
typedef unsigned long dim_t;
#endif

/* Base object.  The leading fields are the reference's
 * (src/base/flamec/include/FLA_type_defs.h:132-153, non-SuperMatrix
 * build); the trailing fields are private to this implementation. */
typedef struct FLA_Obj_struct
{
  FLA_Datatype  datatype;
  FLA_Elemtype  elemtype;
  dim_t         m;
  dim_t         n;
  dim_t         rs;
  dim_t         cs;
  dim_t         m_inner;
  dim_t         n_inner;
  unsigned long id;
  dim_t         m_index;
  dim_t         n_index;
  dim_t         n_elem_alloc;
  void*         buffer;
  int           buffer_info;
  FLA_Uplo      uplo;
  /* private: 1 when this library allocated `buffer` in HBM */
  int           b200_owns_device_buffer;
} FLA_Base_obj;

/* View, passed by value: identical layout to
 * src/base/flamec/include/FLA_type_defs.h:168-180. */
typedef struct FLA_Obj_view
{
  dim_t         offm;
  dim_t         offn;
  dim_t         m;
  dim_t         n;
  dim_t         m_inner;
  dim_t         n_inner;
  FLA_Base_obj* base;
} FLA_Obj;

/* ---- constants: src/base/flamec/include/FLA_macro_defs.h:25-150 -------- */
#undef  TRUE
#undef  FALSE
#define TRUE  1
#define FALSE 0

#define FLA_SUCCESS           (-1)
#define FLA_FAILURE           (-2)

#define FLA_FLOAT             100
#define FLA_DOUBLE            101
#define FLA_COMPLEX           102
#define FLA_DOUBLE_COMPLEX    103
#define FLA_INT               104
#define FLA_CONSTANT          105

#define FLA_MATRIX            150
#define FLA_SCALAR            151

#define FLA_TOP               200
#define FLA_BOTTOM            201
#define FLA_LEFT              210
#define FLA_RIGHT             211

#define FLA_LOWER_TRIANGULAR  300
#define FLA_UPPER_TRIANGULAR  301
#define FLA_ZERO_MATRIX       310
#define FLA_FULL_MATRIX       311

#define FLA_NO_TRANSPOSE      400
#define FLA_TRANSPOSE         401
#define FLA_CONJ_TRANSPOSE    402
#define FLA_CONJ_NO_TRANSPOSE 403

#define FLA_NO_CONJUGATE      450
#define FLA_CONJUGATE         451

#define FLA_UNIT_DIAG         500
#define FLA_NONUNIT_DIAG      501
#define FLA_ZERO_DIAG         502

#define FLA_DIMENSION_M       600
#define FLA_DIMENSION_K       601
#define FLA_DIMENSION_N       602
#define FLA_DIMENSION_MIN     603

#define FLA_NATIVE_PIVOTS     700
#define FLA_LAPACK_PIVOTS     701

#define FLA_FORWARD           800
#define FLA_BACKWARD          801

#define FLA_COLUMNWISE        900
#define FLA_ROWWISE           901

#define FLA_FLAT             1000
#define FLA_HIER             1001

#define FLA_FULL_ERROR_CHECKING 2
#define FLA_MIN_ERROR_CHECKING  1
#define FLA_NO_ERROR_CHECKING   0

/* ---- library lifecycle: src/base/flamec/main/FLA_Init.c:47-127 -------- */
/* FLA_Init creates the CUDA context on the current device, the library's
 * streams and its workspace pool; FLA_Finalize releases them.  Both are
 * idempotent like the reference's. */
void          FLA_Init( void );
void          FLA_Finalize( void );
FLA_Bool      FLA_Initialized( void );
void          FLA_Init_safe( FLA_Error* init_result );
void          FLA_Finalize_safe( FLA_Error init_result );

/* ---- error checking: src/base/flamec/main/FLA_Check.c:17-30 ----------- */
unsigned int  FLA_Check_error_level( void );
unsigned int  FLA_Check_error_level_set( unsigned int level );

/* ---- objects: src/base/flamec/main/FLA_Obj.c:55-620 -------------------- */
/* FLA_Obj_create: rs = cs = 0 selects column-major with ld = max(m,1)
 * (FLA_Obj.c:55-70); the buffer is allocated in HBM. */
FLA_Error     FLA_Obj_create( FLA_Datatype datatype, dim_t m, dim_t n, dim_t rs, dim_t cs, FLA_Obj* obj );
FLA_Error     FLA_Obj_create_without_buffer( FLA_Datatype datatype, dim_t m, dim_t n, FLA_Obj* obj );
/* buffer may be host or device memory; it is borrowed, not owned. */
FLA_Error     FLA_Obj_attach_buffer( void* buffer, dim_t rs, dim_t cs, FLA_Obj* obj );
FLA_Error     FLA_Obj_free( FLA_Obj* obj );
FLA_Error     FLA_Obj_free_without_buffer( FLA_Obj* obj );
FLA_Datatype  FLA_Obj_datatype( FLA_Obj obj );
dim_t         FLA_Obj_length( FLA_Obj obj );
dim_t         FLA_Obj_width( FLA_Obj obj );
dim_t         FLA_Obj_min_dim( FLA_Obj obj );
dim_t         FLA_Obj_max_dim( FLA_Obj obj );
dim_t         FLA_Obj_row_stride( FLA_Obj obj );
dim_t         FLA_Obj_col_stride( FLA_Obj obj );
void*         FLA_Obj_buffer_at_view( FLA_Obj obj );

/* ---- factorizations ---------------------------------------------------- */
/* src/lapack/dec/chol/front/flamec/FLA_Chol.c:16-29.  A := chol(A) in place
 * (lower: L with A = L L^T; upper: U with A = U^T U).  Returns FLA_SUCCESS
 * or the zero-based index of the first column whose pivot is <= 0 or NaN.
 * FLA_DOUBLE or FLA_FLOAT. */
FLA_Error     FLA_Chol( FLA_Uplo uplo, FLA_Obj A );

/* src/lapack/dec/lu/piv/front/flamec/FLA_LU_piv.c:16-33.  A := P L U in
 * place; p (FLA_INT, min(m,n) x 1) receives relative zero-based pivots:
 * row i was interchanged with row i + p[i].  Returns FLA_SUCCESS or the
 * zero-based index of the first zero pivot (the factorization completes). */
FLA_Error     FLA_LU_piv( FLA_Obj A, FLA_Obj p );

/* src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT.c:15-28.  A := Q R via the
 * UT transform: Householder vectors (unit diagonal implied) below the
 * diagonal of A, R on and above; T (b x n, from FLA_QR_UT_create_T) holds
 * the upper-triangular b x b block-reflector factors of each block of b
 * columns, with tau = (1 + u^T u)/2 on the diagonal. */
FLA_Error     FLA_QR_UT( FLA_Obj A, FLA_Obj T );

/* src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_create_T.c:13-51:
 * T is min(32, min_dim(A)) x width(A), column-major, in HBM. */
FLA_Error     FLA_QR_UT_create_T( FLA_Obj A, FLA_Obj* T );

/* src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_recover_tau.c: t := diag of
 * each block of T (libflame's tau, the reciprocal of LAPACK's). */
FLA_Error     FLA_QR_UT_recover_tau( FLA_Obj T, FLA_Obj t );

/* src/lapack/util/app/qut/front/flamec/FLA_Apply_Q_UT.c:16-28.  Supported:
 * side = FLA_LEFT, direct = FLA_FORWARD, storev = FLA_COLUMNWISE, trans =
 * FLA_CONJ_TRANSPOSE / FLA_TRANSPOSE (B := Q^T B) or FLA_NO_TRANSPOSE
 * (B := Q B).  W is accepted for interface compatibility; the GPU code
 * uses its own workspace. */
FLA_Error     FLA_Apply_Q_UT( FLA_Side side, FLA_Trans trans, FLA_Direct direct, FLA_Store storev,
                              FLA_Obj A, FLA_Obj T, FLA_Obj W, FLA_Obj B );

/* src/lapack/util/app/qut/front/flamec/FLA_Apply_Q_UT_create_workspace.c:13-25. */
FLA_Error     FLA_Apply_Q_UT_create_workspace( FLA_Obj T, FLA_Obj B, FLA_Obj* W );

/* src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_form_Q.c:13-86.  Q (as many
 * rows as A) := the first width(Q) columns of H(0) H(1) ... from the factor
 * in A and T; Q may be A itself (formed in place). */
FLA_Error     FLA_QR_UT_form_Q( FLA_Obj A, FLA_Obj T, FLA_Obj Q );

/* src/lapack/util/accum/tut/front/flamec/FLA_Accum_T_UT.c:13.  Supported:
 * FLA_FORWARD, FLA_COLUMNWISE.  T (b x k) := striu(U^T U) + diag(t) per
 * block of b reflectors stored below the diagonal of A, t libflame's tau. */
FLA_Error     FLA_Accum_T_UT( FLA_Direct direct, FLA_Store storev, FLA_Obj A, FLA_Obj t, FLA_Obj T );

/* ---- solves ------------------------------------------------------------- */
/* src/lapack/dec/chol/front/flamec/FLA_Chol_solve.c:13-35: X := inv(A) B
 * with A holding the Cholesky factor from FLA_Chol(uplo, .). */
FLA_Error     FLA_Chol_solve( FLA_Uplo uplo, FLA_Obj A, FLA_Obj B, FLA_Obj X );

/* src/lapack/dec/lu/piv/front/flamec/FLA_LU_piv_solve.c:13-29. */
FLA_Error     FLA_LU_piv_solve( FLA_Obj A, FLA_Obj p, FLA_Obj B, FLA_Obj X );

/* src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_solve.c:13-49: least-squares
 * X (n x nrhs) := inv(R) (Q^T B)(0:n-1, :) for the m x n (m >= n) factor
 * from FLA_QR_UT; B is not modified. */
FLA_Error     FLA_QR_UT_solve( FLA_Obj A, FLA_Obj T, FLA_Obj B, FLA_Obj X );

/* ---- inversion ----------------------------------------------------------- */
/* src/lapack/inv/tri/front/flamec/FLA_Trinv.c:17-50: the uplo triangle of A
 * := its inverse (unit: diagonal taken as ones, not referenced).  Returns
 * FLA_SUCCESS (no singularity check, as the reference's variants). */
FLA_Error     FLA_Trinv( FLA_Uplo uplo, FLA_Diag diag, FLA_Obj A );

/* src/lapack/misc/ttmm/front/flamec/FLA_Ttmm.c:17-43: lower: tril(A) :=
 * tril(L^T L), L = tril(A); upper: triu(A) := triu(U U^T). */
FLA_Error     FLA_Ttmm( FLA_Uplo uplo, FLA_Obj A );

/* src/lapack/inv/spd/front/flamec/FLA_SPDinv.c:15-28: the uplo triangle of
 * the SPD matrix A := that triangle of inv(A) (Chol, Trinv, Ttmm). */
FLA_Error     FLA_SPDinv( FLA_Uplo uplo, FLA_Obj A );

/* src/lapack/util/app/piv/front/flamec/FLA_Apply_pivots.c: side FLA_LEFT,
 * trans FLA_NO_TRANSPOSE (P A) or FLA_TRANSPOSE (P^T A). */
FLA_Error     FLA_Apply_pivots( FLA_Side side, FLA_Trans trans, FLA_Obj p, FLA_Obj A );

/* src/base/flamec/util/lapack/FLA_Shift_pivots_to.c:13-42. */
FLA_Error     FLA_Shift_pivots_to( FLA_Pivot_type ptype, FLA_Obj p );

/* ---- LAPACK ABI (lapack2flame): src/map/lapack2flamec ------------------ */
/* Host or device pointers.  ILP32 integers, Fortran calling convention. */
/* src/map/lapack2flamec/FLA_potrf.c:31-83 */
int dpotrf_( char* uplo, int* n, double* a, int* lda, int* info );
/* src/map/lapack2flamec/FLA_getrf.c:32-92 (ipiv is 1-based, LAPACK style) */
int dgetrf_( int* m, int* n, double* a, int* lda, int* ipiv, int* info );
/* src/map/lapack2flamec/FLA_geqrf.c:24-88 (tau is LAPACK's tau) */
int dgeqrf_( int* m, int* n, double* a, int* lda, double* tau, double* work, int* lwork, int* info );
/* src/map/lapack2flamec/FLA_ormqr.c:35-97: C := op(Q) C or C op(Q), Q from
 * dgeqrf_'s k reflectors (A, tau); work only answers the size query. */
int dormqr_( char* side, char* trans, int* m, int* n, int* k, double* a, int* lda, double* tau,
             double* c, int* ldc, double* work, int* lwork, int* info );
/* src/map/lapack2flamec/FLA_orgqr.c:30-80: A (m x n) := the first n columns
 * of Q from dgeqrf_'s first k reflectors in A and tau. */
int dorgqr_( int* m, int* n, int* k, double* a, int* lda, double* tau, double* work, int* lwork, int* info );
/* src/map/lapack2flamec/FLA_potri.c:25-56: the uplo triangle of A (dpotrf_'s
 * factor) := that triangle of inv(A). */
int dpotri_( char* uplo, int* n, double* a, int* lda, int* info );
/* src/map/common/lapacksrc/f2c/dpotrs.c, dgetrs.c */
int dpotrs_( char* uplo, int* n, int* nrhs, double* a, int* lda, double* b, int* ldb, int* info );
int dgetrs_( char* trans, int* n, int* nrhs, double* a, int* lda, int* ipiv, double* b, int* ldb, int* info );
/* src/map/common/lapacksrc/f2c/dposv.c:120-190, dgesv.c:113-175 */
int dposv_( char* uplo, int* n, int* nrhs, double* a, int* lda, double* b, int* ldb, int* info );
int dgesv_( int* n, int* nrhs, double* a, int* lda, int* ipiv, double* b, int* ldb, int* info );
/* src/map/common/lapacksrc/f2c/dsgesv.c:189-412, dsposv.c:250-413: mixed
 * precision with FP64 refinement; iter >= 0 refinement steps, -3 / -31 when
 * the FP64 factorization took over (A then holds its factors).  work and
 * swork are accepted and not referenced. */
int dsgesv_( int* n, int* nrhs, double* a, int* lda, int* ipiv, double* b, int* ldb, double* x, int* ldx,
             double* work, float* swork, int* iter, int* info );
int dsposv_( char* uplo, int* n, int* nrhs, double* a, int* lda, double* b, int* ldb, double* x, int* ldx,
             double* work, float* swork, int* iter, int* info );

/* ---- FLASH hierarchical objects and front-ends ----------------------------
 * Depth-1 hierarchies (storage by blocks, in HBM): the leaves of an m x n
 * object are b_m x b_n blocks (the last row and column smaller); the
 * front-ends gather the blocks into a column-major HBM copy, run the flat
 * entry point and scatter the result back, with the flat entry point's
 * return values.  Depths above 1 are rejected. */
/* src/base/flamec/hierarchy/main/FLASH_Obj.c:20-81, 143-175, 591-700, 765-780 */
dim_t         FLASH_Obj_depth( FLA_Obj H );
dim_t         FLASH_Obj_blocksizes( FLA_Obj H, dim_t* b_m, dim_t* b_n );
FLA_Error     FLASH_Obj_create( FLA_Datatype datatype, dim_t m, dim_t n, dim_t depth, dim_t* b_mn, FLA_Obj* H );
FLA_Error     FLASH_Obj_create_ext( FLA_Datatype datatype, dim_t m, dim_t n, dim_t depth, dim_t* b_m, dim_t* b_n,
                                    FLA_Obj* H );
FLA_Error     FLASH_Obj_create_hier_copy_of_flat( FLA_Obj F, dim_t depth, dim_t* b_mn, FLA_Obj* H );
FLA_Error     FLASH_Obj_create_hier_copy_of_flat_ext( FLA_Obj F, dim_t depth, dim_t* b_m, dim_t* b_n, FLA_Obj* H );
FLA_Error     FLASH_Obj_create_flat_copy_of_hier( FLA_Obj H, FLA_Obj* F );
void          FLASH_Obj_free( FLA_Obj* H );
FLA_Error     FLASH_Obj_flatten( FLA_Obj H, FLA_Obj F );
FLA_Error     FLASH_Obj_hierarchify( FLA_Obj F, FLA_Obj H );
/* src/base/flamec/hierarchy/main/FLASH_Copy_other.c:81-136 */
FLA_Error     FLASH_Copy_flat_to_hier( FLA_Obj F, dim_t i, dim_t j, FLA_Obj H );
FLA_Error     FLASH_Copy_hier_to_flat( dim_t i, dim_t j, FLA_Obj H, FLA_Obj F );
/* src/base/flamec/hierarchy/main/FLASH_View.c:600-690 */
dim_t         FLASH_Obj_scalar_length( FLA_Obj H );
dim_t         FLASH_Obj_scalar_width( FLA_Obj H );
dim_t         FLASH_Obj_scalar_min_dim( FLA_Obj H );
dim_t         FLASH_Obj_scalar_max_dim( FLA_Obj H );
/* src/lapack/dec/chol/front/flamec/FLASH_Chol.c:15-30, FLASH_Chol_solve.c */
FLA_Error     FLASH_Chol( FLA_Uplo uplo, FLA_Obj A );
FLA_Error     FLASH_Chol_solve( FLA_Uplo uplo, FLA_Obj A, FLA_Obj B, FLA_Obj X );
/* src/lapack/dec/lu/piv/front/flamec/FLASH_LU_piv.c:15-41, FLASH_LU_piv_solve.c;
 * p hierarchical (one column of blocks) or flat, relative pivots as FLA_LU_piv */
FLA_Error     FLASH_LU_piv( FLA_Obj A, FLA_Obj p );
FLA_Error     FLASH_LU_piv_solve( FLA_Obj A, FLA_Obj p, FLA_Obj B, FLA_Obj X );
/* src/lapack/dec/q/qrut/front/flamec/FLASH_QR_UT.c, FLASH_QR_UT_create_hier_matrices.c,
 * FLASH_QR_UT_solve.c: TW min_dim x min_dim with square b_flash blocks
 * (b_alg == b_flash, min_dim(A) % b_flash == 0); block column q's T in TW's
 * diagonal block (q, q), as the reference's algorithm-by-blocks stores it */
FLA_Error     FLASH_QR_UT_create_hier_matrices( FLA_Obj A_flat, dim_t depth, dim_t* b_flash, FLA_Obj* A,
                                                FLA_Obj* TW );
FLA_Error     FLASH_QR_UT( FLA_Obj A, FLA_Obj TW );
FLA_Error     FLASH_QR_UT_solve( FLA_Obj A, FLA_Obj TW, FLA_Obj B, FLA_Obj X );
/* src/lapack/util/app/qut/front/flamec/FLASH_Apply_Q_UT.c, FLASH_Apply_Q_UT_create_workspace.c */
FLA_Error     FLASH_Apply_Q_UT( FLA_Side side, FLA_Trans trans, FLA_Direct direct, FLA_Store storev,
                                FLA_Obj A, FLA_Obj TW, FLA_Obj W, FLA_Obj B );
FLA_Error     FLASH_Apply_Q_UT_create_workspace( FLA_Obj TW, FLA_Obj B, FLA_Obj* W );

#ifdef __cplusplus
}
#endif

#include "FLAME_b200.h"

#endif
