"""libflame_b200: B200-native dense factorizations behind libflame's FLA_Obj API.

The product is the C-ABI shared library ``libflame_b200/libflame_b200.so``
(built by ``libflame_b200.build``) whose entry points are declared in
``include/FLAME.h``.  This module is the ctypes binding a Python caller uses
to reach it: it mirrors the reference FLA_Obj interface (same names,
argument meaning and return codes) and adds helpers that wrap torch CUDA
tensors or NumPy arrays as FLA_Obj views.

There is no CPU fallback: importing the binding fails loudly when the shared
library has not been built.
"""
import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libflame_b200.so")

# Constants: the reference's values (src/base/flamec/include/FLA_macro_defs.h).
FLA_SUCCESS, FLA_FAILURE = -1, -2
FLA_FLOAT, FLA_DOUBLE, FLA_INT = 100, 101, 104
FLA_LEFT, FLA_RIGHT = 210, 211
FLA_LOWER_TRIANGULAR, FLA_UPPER_TRIANGULAR = 300, 301
FLA_NO_TRANSPOSE, FLA_TRANSPOSE, FLA_CONJ_TRANSPOSE = 400, 401, 402
FLA_UNIT_DIAG, FLA_NONUNIT_DIAG = 500, 501
FLA_NATIVE_PIVOTS, FLA_LAPACK_PIVOTS = 700, 701
FLA_FORWARD, FLA_BACKWARD = 800, 801
FLA_COLUMNWISE, FLA_ROWWISE = 900, 901
FLA_NO_ERROR_CHECKING, FLA_MIN_ERROR_CHECKING, FLA_FULL_ERROR_CHECKING = 0, 1, 2


class FLA_Obj(C.Structure):
    """FLA_Obj view, passed by value (include/FLAME.h; reference layout
    src/base/flamec/include/FLA_type_defs.h:168-180)."""
    _fields_ = [("offm", C.c_ulong), ("offn", C.c_ulong), ("m", C.c_ulong), ("n", C.c_ulong),
                ("m_inner", C.c_ulong), ("n_inner", C.c_ulong), ("base", C.c_void_p)]


_lib = None

_SIGS = {
    # name: (restype, argtypes)
    "FLA_Init": (None, []),
    "FLA_Finalize": (None, []),
    "FLA_Initialized": (C.c_int, []),
    "FLA_Check_error_level": (C.c_uint, []),
    "FLA_Check_error_level_set": (C.c_uint, [C.c_uint]),
    "FLA_Obj_create": (C.c_int, [C.c_int, C.c_ulong, C.c_ulong, C.c_ulong, C.c_ulong, C.POINTER(FLA_Obj)]),
    "FLA_Obj_create_without_buffer": (C.c_int, [C.c_int, C.c_ulong, C.c_ulong, C.POINTER(FLA_Obj)]),
    "FLA_Obj_attach_buffer": (C.c_int, [C.c_void_p, C.c_ulong, C.c_ulong, C.POINTER(FLA_Obj)]),
    "FLA_Obj_free": (C.c_int, [C.POINTER(FLA_Obj)]),
    "FLA_Obj_free_without_buffer": (C.c_int, [C.POINTER(FLA_Obj)]),
    "FLA_Obj_length": (C.c_ulong, [FLA_Obj]),
    "FLA_Obj_width": (C.c_ulong, [FLA_Obj]),
    "FLA_Obj_buffer_at_view": (C.c_void_p, [FLA_Obj]),
    "FLA_Chol": (C.c_int, [C.c_int, FLA_Obj]),
    "FLA_LU_piv": (C.c_int, [FLA_Obj, FLA_Obj]),
    "FLA_Apply_pivots": (C.c_int, [C.c_int, C.c_int, FLA_Obj, FLA_Obj]),
    "FLA_Shift_pivots_to": (C.c_int, [C.c_int, FLA_Obj]),
    "FLA_Chol_solve": (C.c_int, [C.c_int, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLA_QR_UT": (C.c_int, [FLA_Obj, FLA_Obj]),
    "FLA_QR_UT_create_T": (C.c_int, [FLA_Obj, C.POINTER(FLA_Obj)]),
    "FLA_QR_UT_recover_tau": (C.c_int, [FLA_Obj, FLA_Obj]),
    "FLA_Apply_Q_UT": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, FLA_Obj, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLA_Apply_Q_UT_create_workspace": (C.c_int, [FLA_Obj, FLA_Obj, C.POINTER(FLA_Obj)]),
    "FLA_LU_piv_solve": (C.c_int, [FLA_Obj, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLA_QR_UT_solve": (C.c_int, [FLA_Obj, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLA_QR_UT_form_Q": (C.c_int, [FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLA_Accum_T_UT": (C.c_int, [C.c_int, C.c_int, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLA_Trinv": (C.c_int, [C.c_int, C.c_int, FLA_Obj]),
    "FLA_Ttmm": (C.c_int, [C.c_int, FLA_Obj]),
    "FLA_SPDinv": (C.c_int, [C.c_int, FLA_Obj]),
    "dormqr_": (C.c_int, [C.c_char_p, C.c_char_p] + [C.c_void_p] * 11),
    "dorgqr_": (C.c_int, [C.c_void_p] * 9),
    "dpotri_": (C.c_int, [C.c_char_p] + [C.c_void_p] * 4),
    "FLA_B200_kernel_launches": (C.c_ulonglong, []),
    "FLA_B200_last_error": (C.c_char_p, []),
    "FLA_B200_num_sms": (C.c_int, []),
    "FLA_B200_last_op_ms": (C.c_double, []),
    "FLA_B200_profile": (None, [C.c_int]),
    "FLA_B200_profile_read": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                        C.POINTER(C.c_ulonglong)]),
    "FLA_B200_dgemm": (C.c_int, [C.c_int, C.c_int, C.c_long, C.c_long, C.c_long, C.c_double,
                                 C.c_void_p, C.c_long, C.c_void_p, C.c_long, C.c_double,
                                 C.c_void_p, C.c_long, C.c_int]),
    "FLA_B200_gemm_concurrency_check": (C.c_int, [C.c_long, C.c_long, C.c_long, C.c_int,
                                                  C.POINTER(C.c_ulonglong)]),
    "FLA_B200_LU_piv_solve_mixed": (C.c_int, [FLA_Obj, FLA_Obj, FLA_Obj, C.c_int, C.c_int,
                                              C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "FLA_B200_Chol_solve_mixed": (C.c_int, [C.c_int, FLA_Obj, FLA_Obj, FLA_Obj, C.c_int, C.c_int,
                                            C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "FLA_Chol_batched": (C.c_int, [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                   C.c_void_p, C.c_void_p]),
    "FLA_LU_piv_batched": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                     C.c_void_p, C.c_void_p]),
    "FLA_B200_Chol_batched_f32": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                            C.c_void_p, C.c_void_p]),
    "FLA_B200_LU_piv_batched_f32": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                              C.c_void_p, C.c_void_p, C.c_void_p]),
    "FLA_B200_Chol_batched_logdet": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p]),
    "FLA_Chol_adjoint_batched": (C.c_int, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double]),
    "FLA_B200_batched_tune": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_void_p]),
    "FLASH_Obj_depth": (C.c_ulong, [FLA_Obj]),
    "FLASH_Obj_blocksizes": (C.c_ulong, [FLA_Obj, C.POINTER(C.c_ulong), C.POINTER(C.c_ulong)]),
    "FLASH_Obj_create": (C.c_int, [C.c_int, C.c_ulong, C.c_ulong, C.c_ulong, C.POINTER(C.c_ulong),
                                   C.POINTER(FLA_Obj)]),
    "FLASH_Obj_create_ext": (C.c_int, [C.c_int, C.c_ulong, C.c_ulong, C.c_ulong, C.POINTER(C.c_ulong),
                                       C.POINTER(C.c_ulong), C.POINTER(FLA_Obj)]),
    "FLASH_Obj_create_hier_copy_of_flat": (C.c_int, [FLA_Obj, C.c_ulong, C.POINTER(C.c_ulong), C.POINTER(FLA_Obj)]),
    "FLASH_Obj_create_hier_copy_of_flat_ext": (C.c_int, [FLA_Obj, C.c_ulong, C.POINTER(C.c_ulong),
                                                         C.POINTER(C.c_ulong), C.POINTER(FLA_Obj)]),
    "FLASH_Obj_create_flat_copy_of_hier": (C.c_int, [FLA_Obj, C.POINTER(FLA_Obj)]),
    "FLASH_Obj_free": (None, [C.POINTER(FLA_Obj)]),
    "FLASH_Obj_flatten": (C.c_int, [FLA_Obj, FLA_Obj]),
    "FLASH_Obj_hierarchify": (C.c_int, [FLA_Obj, FLA_Obj]),
    "FLASH_Copy_flat_to_hier": (C.c_int, [FLA_Obj, C.c_ulong, C.c_ulong, FLA_Obj]),
    "FLASH_Copy_hier_to_flat": (C.c_int, [C.c_ulong, C.c_ulong, FLA_Obj, FLA_Obj]),
    "FLASH_Obj_scalar_length": (C.c_ulong, [FLA_Obj]),
    "FLASH_Obj_scalar_width": (C.c_ulong, [FLA_Obj]),
    "FLASH_Obj_scalar_min_dim": (C.c_ulong, [FLA_Obj]),
    "FLASH_Obj_scalar_max_dim": (C.c_ulong, [FLA_Obj]),
    "FLASH_Chol": (C.c_int, [C.c_int, FLA_Obj]),
    "FLASH_Chol_solve": (C.c_int, [C.c_int, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLASH_LU_piv": (C.c_int, [FLA_Obj, FLA_Obj]),
    "FLASH_LU_piv_solve": (C.c_int, [FLA_Obj, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLASH_QR_UT_create_hier_matrices": (C.c_int, [FLA_Obj, C.c_ulong, C.POINTER(C.c_ulong), C.POINTER(FLA_Obj),
                                                   C.POINTER(FLA_Obj)]),
    "FLASH_QR_UT": (C.c_int, [FLA_Obj, FLA_Obj]),
    "FLASH_QR_UT_solve": (C.c_int, [FLA_Obj, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLASH_Apply_Q_UT": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, FLA_Obj, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLASH_Apply_Q_UT_create_workspace": (C.c_int, [FLA_Obj, FLA_Obj, C.POINTER(FLA_Obj)]),
    "FLA_B200_batched_nb": (C.c_int, [C.c_int, C.c_int, C.c_int]),
    "FLA_Chol_adjoint": (C.c_int, [C.c_int, FLA_Obj, FLA_Obj]),
    "FLA_B200_Chol_logdet_adjoint": (C.c_int, [FLA_Obj, FLA_Obj, C.c_double, C.POINTER(C.c_double)]),
    "FLA_B200_Trsm_llnn_adjoint": (C.c_int, [FLA_Obj, FLA_Obj, FLA_Obj, FLA_Obj]),
    "FLA_B200_lp_gemm": (C.c_int, [C.c_int, C.c_long, C.c_long, C.c_long, C.c_float, C.c_void_p, C.c_long,
                                   C.c_void_p, C.c_long, C.c_float, C.c_void_p, C.c_long]),
}

_OPTIONAL = set()


def lib():
    """Load the shared library (raises when it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libflame_b200.so is not built; run `python -m libflame_b200.build` "
                              "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            try:
                f = getattr(L, name)
            except AttributeError:
                if name in _OPTIONAL:
                    continue
                raise
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    """Names of the C entry points the binding declares."""
    return list(_SIGS.keys())


# ---------------------------------------------------------------------------
# Wrapping buffers as FLA_Obj views.
# ---------------------------------------------------------------------------
class View:
    """An FLA_Obj view over a caller-owned buffer (torch tensor or NumPy
    array), column-major.  Keeps the buffer alive; frees the base object on
    deletion (never the buffer, which is borrowed)."""

    def __init__(self, buf, dt=None):
        import numpy as np
        self.buf = buf
        if hasattr(buf, "data_ptr"):  # torch tensor
            import torch
            t = buf
            if t.dim() == 1:
                m, n, ld = t.shape[0], 1, max(t.shape[0], 1)
                assert t.stride(0) == 1
            else:
                m, n = t.shape
                assert t.stride(0) == 1, "tensor must be column-major (stride(0) == 1)"
                ld = max(t.stride(1), 1)
            ptr = t.data_ptr()
            if dt is None:
                dt = {torch.float64: FLA_DOUBLE, torch.float32: FLA_FLOAT, torch.int32: FLA_INT}[t.dtype]
        else:
            a = buf
            if a.ndim == 1:
                m, n, ld = a.shape[0], 1, max(a.shape[0], 1)
            else:
                assert a.flags["F_CONTIGUOUS"], "array must be Fortran-ordered"
                m, n = a.shape
                ld = max(m, 1)
            ptr = a.ctypes.data
            if dt is None:
                dt = {np.dtype(np.float64): FLA_DOUBLE, np.dtype(np.float32): FLA_FLOAT,
                      np.dtype(np.int32): FLA_INT}[a.dtype]
        self.obj = FLA_Obj()
        L = lib()
        L.FLA_Obj_create_without_buffer(dt, m, n, C.byref(self.obj))
        L.FLA_Obj_attach_buffer(C.c_void_p(ptr), 1, ld, C.byref(self.obj))

    def __del__(self):
        try:
            lib().FLA_Obj_free_without_buffer(C.byref(self.obj))
        except Exception:
            pass


def init():
    lib().FLA_Init()


def last_error():
    return lib().FLA_B200_last_error().decode()


def kernel_launches():
    return int(lib().FLA_B200_kernel_launches())


def num_sms():
    """SM count of the device bound at FLA_Init."""
    return int(lib().FLA_B200_num_sms())


def last_op_ms():
    """Device time of the last factorization/solve call (CUDA events)."""
    return float(lib().FLA_B200_last_op_ms())


PROF_GEMM, PROF_PANEL, PROF_TRSM, PROF_SWAP, PROF_DIAG, PROF_OTHER = range(6)


def profile(on=True):
    lib().FLA_B200_profile(1 if on else 0)


def profile_read(cls):
    ms, fl, n = C.c_double(), C.c_double(), C.c_ulonglong()
    lib().FLA_B200_profile_read(cls, C.byref(ms), C.byref(fl), C.byref(n))
    return ms.value, fl.value, n.value


# Thin Python mirrors of the reference calls on buffers (return codes as in
# C).  The views are held in locals for the duration of the call: a View
# frees its FLA_Obj base when it is collected.
def chol(A, uplo=FLA_LOWER_TRIANGULAR):
    """FLA_Chol(uplo, A) on a column-major buffer, in place."""
    va = View(A)
    return lib().FLA_Chol(uplo, va.obj)


def lu_piv(A, p):
    """FLA_LU_piv(A, p) in place; p int32 vector of length >= min(m, n)."""
    va, vp = View(A), View(p)
    return lib().FLA_LU_piv(va.obj, vp.obj)


def apply_pivots(p, A, trans=FLA_NO_TRANSPOSE):
    vp, va = View(p), View(A)
    return lib().FLA_Apply_pivots(FLA_LEFT, trans, vp.obj, va.obj)


def chol_solve(A, B, X, uplo=FLA_LOWER_TRIANGULAR):
    va, vb, vx = View(A), View(B), View(X)
    return lib().FLA_Chol_solve(uplo, va.obj, vb.obj, vx.obj)


def lu_piv_solve(A, p, B, X):
    va, vp, vb, vx = View(A), View(p), View(B), View(X)
    return lib().FLA_LU_piv_solve(va.obj, vp.obj, vb.obj, vx.obj)


def qr_ut(A, T):
    """FLA_QR_UT(A, T) in place; T is b_alg x n (b_alg = min(32, min(m, n)))."""
    va, vt = View(A), View(T)
    return lib().FLA_QR_UT(va.obj, vt.obj)


def apply_q_ut(A, T, B, trans=FLA_CONJ_TRANSPOSE):
    """FLA_Apply_Q_UT(LEFT, trans, FORWARD, COLUMNWISE, A, T, W, B): B := Q^T B
    (trans = FLA_CONJ_TRANSPOSE / FLA_TRANSPOSE) or Q B (FLA_NO_TRANSPOSE)."""
    va, vt, vb = View(A), View(T), View(B)
    return lib().FLA_Apply_Q_UT(FLA_LEFT, trans, FLA_FORWARD, FLA_COLUMNWISE, va.obj, vt.obj, vt.obj, vb.obj)


def qr_ut_recover_tau(T, t):
    vt, vv = View(T), View(t)
    return lib().FLA_QR_UT_recover_tau(vt.obj, vv.obj)


def shift_pivots_to(ptype, p):
    vp = View(p)
    return lib().FLA_Shift_pivots_to(ptype, vp.obj)


def lu_piv_solve_mixed(A, B, X, prec=-1, solver=-1):
    """X := A^-1 B, low-precision LU + FP64 refinement (A unchanged).
    Returns (FLA error code, refinement steps, GMRES iterations)."""
    vA, vB, vX = View(A), View(B), View(X)
    it, inner = C.c_int(0), C.c_int(0)
    r = lib().FLA_B200_LU_piv_solve_mixed(vA.obj, vB.obj, vX.obj, prec, solver, C.byref(it), C.byref(inner))
    return r, it.value, inner.value


def chol_solve_mixed(A, B, X, uplo=FLA_LOWER_TRIANGULAR, prec=-1, solver=-1):
    """X := A^-1 B for SPD A, low-precision Cholesky + FP64 refinement."""
    vA, vB, vX = View(A), View(B), View(X)
    it, inner = C.c_int(0), C.c_int(0)
    r = lib().FLA_B200_Chol_solve_mixed(uplo, vA.obj, vB.obj, vX.obj, prec, solver, C.byref(it), C.byref(inner))
    return r, it.value, inner.value


def _ptr_array(tensors):
    return (C.c_void_p * len(tensors))(*[t.data_ptr() for t in tensors])


def batched(kind, mats, pivs=None, rhs=None, f32=False):
    """Batched factorization (+ solve) of column-major CUDA tensors.
    kind: "chol" or "lu".  mats: list of n x n tensors (column-major views);
    pivs: list of int32 CUDA tensors (LU); rhs: list of n x nrhs tensors
    overwritten with the solutions.  Returns (error code, info list)."""
    import numpy as _np
    cnt = len(mats)
    n = _np.array([m.shape[0] for m in mats], dtype=_np.int32)
    lda = _np.array([max(1, m.stride(1)) for m in mats], dtype=_np.int32)
    A = _ptr_array(mats)
    nrhs = 0 if rhs is None else rhs[0].shape[1]
    B = _ptr_array(rhs) if rhs is not None else None
    ldb = _np.array([max(1, b.stride(1)) for b in rhs], dtype=_np.int32) if rhs is not None else None
    info = _np.zeros(cnt, dtype=_np.int32)
    P = (lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None)
    L = lib()
    if kind == "chol":
        if f32:
            r = L.FLA_B200_Chol_batched_f32(cnt, P(n), A, P(lda), nrhs, B, P(ldb), P(info))
        else:
            r = L.FLA_Chol_batched(FLA_LOWER_TRIANGULAR, cnt, P(n), A, P(lda), nrhs, B, P(ldb), P(info))
    else:
        pv = _ptr_array(pivs)
        if f32:
            r = L.FLA_B200_LU_piv_batched_f32(cnt, P(n), A, P(lda), pv, nrhs, B, P(ldb), P(info))
        else:
            r = L.FLA_LU_piv_batched(cnt, P(n), A, P(lda), pv, nrhs, B, P(ldb), P(info))
    return r, info.tolist()


def chol_batched_logdet(mats, rhs=None):
    """FLA_B200_Chol_batched_logdet on column-major CUDA tensors: lower
    Cholesky of every matrix in place (+ solves of rhs), per-matrix
    log-determinants.  Returns (error code, info list, logdet list)."""
    import numpy as _np
    cnt = len(mats)
    n = _np.array([m.shape[0] for m in mats], dtype=_np.int32)
    lda = _np.array([max(1, m.stride(1)) for m in mats], dtype=_np.int32)
    nrhs = 0 if rhs is None else rhs[0].shape[1]
    B = _ptr_array(rhs) if rhs is not None else None
    ldb = _np.array([max(1, b.stride(1)) for b in rhs], dtype=_np.int32) if rhs is not None else None
    info = _np.zeros(cnt, dtype=_np.int32)
    logdet = _np.zeros(cnt, dtype=_np.float64)
    P = (lambda a: a.ctypes.data_as(C.c_void_p) if a is not None else None)
    r = lib().FLA_B200_Chol_batched_logdet(cnt, P(n), _ptr_array(mats), P(lda), nrhs, B, P(ldb), P(logdet), P(info))
    return r, info.tolist(), logdet.tolist()


def chol_adjoint_batched(Ls, Lbars, logdet_scale=0.0):
    """FLA_Chol_adjoint_batched over lists of column-major CUDA tensors (each
    L[i] and Lbar[i] with the same leading dimension)."""
    import numpy as _np
    n = _np.array([m.shape[0] for m in Ls], dtype=_np.int32)
    ld = _np.array([max(1, m.stride(1)) for m in Ls], dtype=_np.int32)
    assert all(max(1, b.stride(1)) == l for b, l in zip(Lbars, ld))
    P = (lambda a: a.ctypes.data_as(C.c_void_p))
    return lib().FLA_Chol_adjoint_batched(len(Ls), P(n), _ptr_array(Ls), P(ld), _ptr_array(Lbars), logdet_scale)


def chol_adjoint(L, Lbar):
    """Lbar (lower) := Abar, the adjoint of the lower entries of A = L L^T."""
    vL, vB = View(L), View(Lbar)
    return lib().FLA_Chol_adjoint(FLA_LOWER_TRIANGULAR, vL.obj, vB.obj)


def chol_logdet_adjoint(L, Lbar, scale):
    vL, vB = View(L), View(Lbar)
    ld = C.c_double(0.0)
    r = lib().FLA_B200_Chol_logdet_adjoint(vL.obj, vB.obj, scale, C.byref(ld))
    return r, ld.value


def trsm_llnn_adjoint(L, X, Xbar, Lbar):
    vL, vX, vXb, vLb = View(L), View(X), View(Xbar), View(Lbar)
    return lib().FLA_B200_Trsm_llnn_adjoint(vL.obj, vX.obj, vXb.obj, vLb.obj)


def qr_ut_solve(A, T, B, X):
    """FLA_QR_UT_solve(A, T, B, X): least-squares X from the QR_UT factor."""
    va, vt, vb, vx = View(A), View(T), View(B), View(X)
    return lib().FLA_QR_UT_solve(va.obj, vt.obj, vb.obj, vx.obj)


def qr_ut_form_q(A, T, Q):
    """FLA_QR_UT_form_Q(A, T, Q); Q may be A itself (in place)."""
    va, vt = View(A), View(T)
    vq = va if Q is A else View(Q)
    return lib().FLA_QR_UT_form_Q(va.obj, vt.obj, vq.obj)


def accum_t_ut(A, t, T):
    """FLA_Accum_T_UT(FORWARD, COLUMNWISE, A, t, T)."""
    va, vt, vT = View(A), View(t), View(T)
    return lib().FLA_Accum_T_UT(FLA_FORWARD, FLA_COLUMNWISE, va.obj, vt.obj, vT.obj)


def trinv(A, uplo=FLA_LOWER_TRIANGULAR, diag=FLA_NONUNIT_DIAG):
    va = View(A)
    return lib().FLA_Trinv(uplo, diag, va.obj)


def ttmm(A, uplo=FLA_LOWER_TRIANGULAR):
    va = View(A)
    return lib().FLA_Ttmm(uplo, va.obj)


def spdinv(A, uplo=FLA_LOWER_TRIANGULAR):
    va = View(A)
    return lib().FLA_SPDinv(uplo, va.obj)


def _buf(x):
    """Raw pointer of a torch tensor or NumPy array (LAPACK entry points)."""
    return C.c_void_p(x.data_ptr() if hasattr(x, "data_ptr") else x.ctypes.data)


def _ld(x):
    return max(1, x.stride(1) if hasattr(x, "stride") and x.dim() == 2 else x.shape[0])


def dormqr(side, trans, a, tau, c):
    """dormqr_ on column-major buffers (host or device); returns info."""
    m, n = c.shape
    k = tau.shape[0]
    info = C.c_int(0)
    nw = n if side == "L" else m
    work = (C.c_double * max(1, nw))()
    lw = C.c_int(len(work))
    ints = [C.c_int(v) for v in (m, n, k, _ld(a), _ld(c))]
    lib().dormqr_(side.encode(), trans.encode(), C.byref(ints[0]), C.byref(ints[1]), C.byref(ints[2]), _buf(a),
                  C.byref(ints[3]), _buf(tau), _buf(c), C.byref(ints[4]), work, C.byref(lw), C.byref(info))
    return info.value


def dorgqr(a, tau):
    """dorgqr_ in place on the m x n buffer a with k = len(tau); returns info."""
    m, n = a.shape
    k = tau.shape[0]
    info = C.c_int(0)
    work = (C.c_double * max(1, n))()
    ints = [C.c_int(v) for v in (m, n, k, _ld(a), len(work))]
    lib().dorgqr_(C.byref(ints[0]), C.byref(ints[1]), C.byref(ints[2]), _buf(a), C.byref(ints[3]), _buf(tau),
                  work, C.byref(ints[4]), C.byref(info))
    return info.value


def dpotri(uplo, a):
    n = a.shape[0]
    info = C.c_int(0)
    ni, ld = C.c_int(n), C.c_int(_ld(a))
    lib().dpotri_(uplo.encode(), C.byref(ni), _buf(a), C.byref(ld), C.byref(info))
    return info.value


def dgeqrf(a, tau):
    m, n = a.shape
    info = C.c_int(0)
    work = (C.c_double * max(1, n * 32))()
    ints = [C.c_int(v) for v in (m, n, _ld(a), len(work))]
    lib().dgeqrf_(C.byref(ints[0]), C.byref(ints[1]), _buf(a), C.byref(ints[2]), _buf(tau), work,
                  C.byref(ints[3]), C.byref(info))
    return info.value
