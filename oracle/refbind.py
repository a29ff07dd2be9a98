"""ctypes binding to the reference libflame built from source by
oracle/build_ref.py (oracle/_ref/libflame_ref.so).

Test infrastructure only: used by tests/, by tests/golden/make_golden.py and
by the CPU-baseline leg of bench.py, never by the product path.

Every wrapper takes NumPy arrays, copies them into Fortran-ordered float64
buffers, attaches them to FLA_Obj views exactly as lapack2flame does
(FLA_Obj_create_without_buffer + FLA_Obj_attach_buffer(buf, 1, ld),
src/map/lapack2flamec/FLA_potrf.c:48-49) and calls the reference entry point.
"""
import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

# Constants, values from src/base/flamec/include/FLA_macro_defs.h:32-120.
FLA_SUCCESS = -1
FLA_DOUBLE = 101
FLA_FLOAT = 100
FLA_INT = 104
FLA_LEFT, FLA_RIGHT = 210, 211
FLA_LOWER_TRIANGULAR, FLA_UPPER_TRIANGULAR = 300, 301
FLA_NO_TRANSPOSE, FLA_TRANSPOSE, FLA_CONJ_TRANSPOSE = 400, 401, 402
FLA_UNIT_DIAG, FLA_NONUNIT_DIAG = 500, 501
FLA_NATIVE_PIVOTS, FLA_LAPACK_PIVOTS = 700, 701
FLA_FORWARD, FLA_BACKWARD = 800, 801
FLA_COLUMNWISE, FLA_ROWWISE = 900, 901


class FLA_Obj(C.Structure):
    """View struct, layout of src/base/flamec/include/FLA_type_defs.h:168-180."""
    _fields_ = [("offm", C.c_ulong), ("offn", C.c_ulong), ("m", C.c_ulong),
                ("n", C.c_ulong), ("m_inner", C.c_ulong), ("n_inner", C.c_ulong),
                ("base", C.c_void_p)]


_lib = {}


LIB_FILES = {"serial": "libflame_ref.so", "smp": "libflame_ref_smp.so",
             "openblas": "libflame_ref_openblas.so"}


def lib(smp=False, kind=None):
    """The reference library: "serial" (f2c built-in BLAS, the parity
    oracle), "smp" (+ SuperMatrix/OpenMP) or "openblas" (flat FLA_* over
    SciPy's bundled OpenBLAS, the fast CPU baseline)."""
    key = kind or ("smp" if smp else "serial")
    if key not in _lib:
        path = os.path.join(REF_DIR, LIB_FILES[key])
        if not os.path.exists(path):
            raise FileNotFoundError(path + " missing: run python oracle/build_ref.py")
        L = C.CDLL(path)
        L.FLA_Init.restype = None
        L.FLA_Init()
        for name in ["FLA_Chol", "FLA_LU_piv", "FLA_QR_UT", "FLA_Apply_Q_UT",
                     "FLA_Chol_solve", "FLA_LU_piv_solve", "FLA_Apply_pivots",
                     "FLA_Shift_pivots_to", "FLA_Obj_create_without_buffer",
                     "FLA_Obj_attach_buffer", "FLA_Obj_free_without_buffer",
                     "FLA_Trsm", "FLA_Set", "FLA_QR_UT_solve", "FLA_QR_UT_form_Q",
                     "FLA_SPDinv", "FLA_Trinv", "FLA_Ttmm", "FLA_Accum_T_UT"]:
            getattr(L, name).restype = C.c_int
        _lib[key] = L
    return _lib[key]


class _Mat:
    """A Fortran-ordered buffer attached to an FLA_Obj view."""

    def __init__(self, L, arr, dtype=np.float64, dt=FLA_DOUBLE):
        self.a = np.array(arr, dtype=dtype, order="F", copy=True)
        if self.a.ndim == 1:
            self.a = self.a.reshape(-1, 1, order="F")
        m, n = self.a.shape
        self.obj = FLA_Obj()
        L.FLA_Obj_create_without_buffer(dt, C.c_ulong(m), C.c_ulong(n), C.byref(self.obj))
        ld = max(m, 1)
        L.FLA_Obj_attach_buffer(self.a.ctypes.data_as(C.c_void_p), C.c_ulong(1),
                                C.c_ulong(ld), C.byref(self.obj))
        self.L = L

    def __del__(self):
        try:
            self.L.FLA_Obj_free_without_buffer(C.byref(self.obj))
        except Exception:
            pass


def _dt(a):
    return (np.float32, FLA_FLOAT) if np.asarray(a).dtype == np.float32 else (np.float64, FLA_DOUBLE)


def chol(A, uplo=FLA_LOWER_TRIANGULAR, smp=False, kind=None):
    """FLA_Chol (src/lapack/dec/chol/front/flamec/FLA_Chol.c:16-29).
    Returns (factored copy of A, return value)."""
    L = lib(smp, kind)
    npdt, dt = _dt(A)
    M = _Mat(L, A, npdt, dt)
    r = L.FLA_Chol(uplo, M.obj)
    return M.a, r


def lu_piv(A, smp=False, kind=None):
    """FLA_LU_piv (src/lapack/dec/lu/piv/front/flamec/FLA_LU_piv.c:16-33).
    Returns (LU, relative zero-based pivots, return value)."""
    L = lib(smp, kind)
    npdt, dt = _dt(A)
    M = _Mat(L, A, npdt, dt)
    k = min(M.a.shape)
    P = _Mat(L, np.zeros(k, dtype=np.int32), np.int32, FLA_INT)
    r = L.FLA_LU_piv(M.obj, P.obj)
    return M.a, P.a.ravel().copy(), r


def qr_ut(A, b_alg=None, kind=None):
    """FLA_QR_UT_create_T + FLA_QR_UT (src/lapack/dec/q/qrut/front/flamec/
    FLA_QR_UT_create_T.c:13-51, FLA_QR_UT.c:15-28).  Returns (A, T, rval)."""
    L = lib(kind=kind)
    M = _Mat(L, A)
    m, n = M.a.shape
    if b_alg is None:
        b_alg = min(32, min(m, n))
    T = _Mat(L, np.zeros((b_alg, n)))
    r = L.FLA_QR_UT(M.obj, T.obj)
    return M.a, T.a, r


def apply_q_ut(A, T, B, trans=FLA_CONJ_TRANSPOSE):
    """FLA_Apply_Q_UT(LEFT, trans, FORWARD, COLUMNWISE, A, T, W, B)
    (src/lapack/util/app/qut/front/flamec/FLA_Apply_Q_UT.c:16-28) with
    W from FLA_Apply_Q_UT_create_workspace (b_alg x max_dim(B))."""
    L = lib()
    MA = _Mat(L, A)
    MT = _Mat(L, T)
    MB = _Mat(L, B)
    W = _Mat(L, np.zeros((T.shape[0], max(MB.a.shape))))
    r = L.FLA_Apply_Q_UT(FLA_LEFT, trans, FLA_FORWARD, FLA_COLUMNWISE,
                         MA.obj, MT.obj, W.obj, MB.obj)
    return MB.a, r


def chol_solve(Afac, B, uplo=FLA_LOWER_TRIANGULAR):
    """FLA_Chol_solve (src/lapack/dec/chol/front/flamec/FLA_Chol_solve.c:13-35)."""
    L = lib()
    MA = _Mat(L, Afac)
    MB = _Mat(L, B)
    MX = _Mat(L, np.zeros_like(MB.a))
    r = L.FLA_Chol_solve(uplo, MA.obj, MB.obj, MX.obj)
    return MX.a, r


def lu_piv_solve(LU, p, B):
    """FLA_LU_piv_solve (src/lapack/dec/lu/piv/front/flamec/FLA_LU_piv_solve.c:13-29)."""
    L = lib()
    MA = _Mat(L, LU)
    P = _Mat(L, np.asarray(p, dtype=np.int32), np.int32, FLA_INT)
    MB = _Mat(L, B)
    MX = _Mat(L, np.zeros_like(MB.a))
    r = L.FLA_LU_piv_solve(MA.obj, P.obj, MB.obj, MX.obj)
    return MX.a, r


def apply_pivots(p, A, trans=FLA_NO_TRANSPOSE):
    L = lib()
    P = _Mat(L, np.asarray(p, dtype=np.int32), np.int32, FLA_INT)
    M = _Mat(L, A)
    r = L.FLA_Apply_pivots(FLA_LEFT, trans, P.obj, M.obj)
    return M.a, r


def qr_ut_solve(QR, T, B):
    """FLA_QR_UT_solve (src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_solve.c:13-49)."""
    L = lib()
    MA, MT, MB = _Mat(L, QR), _Mat(L, T), _Mat(L, B)
    MX = _Mat(L, np.zeros((MA.a.shape[1], MB.a.shape[1])))
    r = L.FLA_QR_UT_solve(MA.obj, MT.obj, MB.obj, MX.obj)
    return MX.a, r


def qr_ut_form_q(QR, T, ncols):
    """FLA_QR_UT_form_Q (src/lapack/dec/q/qrut/front/flamec/FLA_QR_UT_form_Q.c:13-86)
    into a separate m x ncols Q."""
    L = lib()
    MA, MT = _Mat(L, QR), _Mat(L, T)
    MQ = _Mat(L, np.zeros((MA.a.shape[0], ncols)))
    r = L.FLA_QR_UT_form_Q(MA.obj, MT.obj, MQ.obj)
    return MQ.a, r


def accum_t_ut(QR, t, b):
    """FLA_Accum_T_UT(FORWARD, COLUMNWISE) (src/lapack/util/accum/tut/front/flamec/FLA_Accum_T_UT.c:13)."""
    L = lib()
    MA = _Mat(L, QR)
    Mt = _Mat(L, np.asarray(t, dtype=np.float64))
    MT = _Mat(L, np.zeros((b, min(MA.a.shape))))
    r = L.FLA_Accum_T_UT(FLA_FORWARD, FLA_COLUMNWISE, MA.obj, Mt.obj, MT.obj)
    return MT.a, r


def spdinv(A, uplo=FLA_LOWER_TRIANGULAR):
    """FLA_SPDinv (src/lapack/inv/spd/front/flamec/FLA_SPDinv.c:15-28)."""
    L = lib()
    M = _Mat(L, A)
    r = L.FLA_SPDinv(uplo, M.obj)
    return M.a, r


def trinv(A, uplo=FLA_LOWER_TRIANGULAR, diag=FLA_NONUNIT_DIAG):
    """FLA_Trinv (src/lapack/inv/tri/front/flamec/FLA_Trinv.c:17-50)."""
    L = lib()
    M = _Mat(L, A)
    r = L.FLA_Trinv(uplo, diag, M.obj)
    return M.a, r


def ttmm(A, uplo=FLA_LOWER_TRIANGULAR):
    """FLA_Ttmm (src/lapack/misc/ttmm/front/flamec/FLA_Ttmm.c:17-43)."""
    L = lib()
    M = _Mat(L, A)
    r = L.FLA_Ttmm(uplo, M.obj)
    return M.a, r


# ---- LAPACK ABI through lapack2flame / f2c drivers ------------------------

def _ip(x):
    return C.byref(C.c_int(x))


def dpotrf(A, uplo="L"):
    L = lib()
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    n = a.shape[0]
    info = C.c_int(0)
    L.dpotrf_(C.c_char_p(uplo.encode()), _ip(n), a.ctypes.data_as(C.c_void_p), _ip(max(n, 1)), C.byref(info))
    return a, info.value


def dgetrf(A):
    L = lib()
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    m, n = a.shape
    ipiv = np.zeros(min(m, n), dtype=np.int32)
    info = C.c_int(0)
    L.dgetrf_(_ip(m), _ip(n), a.ctypes.data_as(C.c_void_p), _ip(max(m, 1)),
              ipiv.ctypes.data_as(C.c_void_p), C.byref(info))
    return a, ipiv, info.value


def dgeqrf(A):
    L = lib()
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    m, n = a.shape
    tau = np.zeros(min(m, n))
    lwork = max(1, n * 32)
    work = np.zeros(lwork)
    info = C.c_int(0)
    L.dgeqrf_(_ip(m), _ip(n), a.ctypes.data_as(C.c_void_p), _ip(max(m, 1)),
              tau.ctypes.data_as(C.c_void_p), work.ctypes.data_as(C.c_void_p),
              _ip(lwork), C.byref(info))
    return a, tau, info.value


last_secs = 0.0  # seconds of the last dsposv / dsgesv / dposv / dgesv call itself


def dposv(A, B, uplo="L", kind=None):
    global last_secs
    import time
    L = lib(kind=kind)
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    n, nrhs = b.shape
    info = C.c_int(0)
    t0 = time.perf_counter()
    L.dposv_(C.c_char_p(uplo.encode()), _ip(n), _ip(nrhs), a.ctypes.data_as(C.c_void_p),
             _ip(max(n, 1)), b.ctypes.data_as(C.c_void_p), _ip(max(n, 1)), C.byref(info))
    last_secs = time.perf_counter() - t0
    return a, b, info.value


def dgesv(A, B, kind=None):
    global last_secs
    import time
    L = lib(kind=kind)
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    n, nrhs = b.shape
    ipiv = np.zeros(n, dtype=np.int32)
    info = C.c_int(0)
    t0 = time.perf_counter()
    L.dgesv_(_ip(n), _ip(nrhs), a.ctypes.data_as(C.c_void_p), _ip(max(n, 1)),
             ipiv.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), _ip(max(n, 1)),
             C.byref(info))
    last_secs = time.perf_counter() - t0
    return a, ipiv, b, info.value


def dsposv(A, B, uplo="L", kind=None):
    """The reference's FP32-factor/FP64-refine driver
    (src/map/common/lapacksrc/f2c/dsposv.c:250-413)."""
    global last_secs
    import time
    L = lib(kind=kind)
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    n, nrhs = b.shape
    x = np.zeros_like(b, order="F")
    work = np.zeros(n * nrhs)
    swork = np.zeros(n * (n + nrhs), dtype=np.float32)
    it = C.c_int(0)
    info = C.c_int(0)
    t0 = time.perf_counter()
    L.dsposv_(C.c_char_p(uplo.encode()), _ip(n), _ip(nrhs), a.ctypes.data_as(C.c_void_p), _ip(n),
              b.ctypes.data_as(C.c_void_p), _ip(n), x.ctypes.data_as(C.c_void_p), _ip(n),
              work.ctypes.data_as(C.c_void_p), swork.ctypes.data_as(C.c_void_p),
              C.byref(it), C.byref(info))
    last_secs = time.perf_counter() - t0
    return x, it.value, info.value


def dsgesv(A, B, kind=None):
    """src/map/common/lapacksrc/f2c/dsgesv.c:246-405."""
    global last_secs
    import time
    L = lib(kind=kind)
    a = np.array(A, dtype=np.float64, order="F", copy=True)
    b = np.array(B, dtype=np.float64, order="F", copy=True)
    if b.ndim == 1:
        b = b.reshape(-1, 1, order="F")
    n, nrhs = b.shape
    x = np.zeros_like(b, order="F")
    ipiv = np.zeros(n, dtype=np.int32)
    work = np.zeros(n * nrhs)
    swork = np.zeros(n * (n + nrhs), dtype=np.float32)
    it = C.c_int(0)
    info = C.c_int(0)
    t0 = time.perf_counter()
    L.dsgesv_(_ip(n), _ip(nrhs), a.ctypes.data_as(C.c_void_p), _ip(n),
              ipiv.ctypes.data_as(C.c_void_p), b.ctypes.data_as(C.c_void_p), _ip(n),
              x.ctypes.data_as(C.c_void_p), _ip(n), work.ctypes.data_as(C.c_void_p),
              swork.ctypes.data_as(C.c_void_p), C.byref(it), C.byref(info))
    last_secs = time.perf_counter() - t0
    return x, it.value, info.value


# ---- SuperMatrix (FLASH) front ends, the reference's multithreaded path --

def _flash_run(kind, A, nthreads, block=256):
    """Run FLASH_LU_piv / FLASH_Chol on a hierarchical copy of A (one level,
    block x block blocks) with SuperMatrix on `nthreads` OpenMP threads
    (src/lapack/dec/lu/piv/front/flamec/FLASH_LU_piv.c,
    src/base/flamec/supermatrix/main/FLASH_Queue.c:187-600).
    Returns (result, seconds of the factorization call)."""
    import time
    L = lib(smp=True)
    M = _Mat(L, A)
    b = C.c_ulong(block)
    H = FLA_Obj()
    L.FLASH_Queue_set_num_threads(C.c_uint(nthreads))
    L.FLASH_Obj_create_hier_copy_of_flat(M.obj, C.c_ulong(1), C.byref(b), C.byref(H))
    if kind == "lu":
        k = min(M.a.shape)
        P = _Mat(L, np.zeros(k, dtype=np.int32), np.int32, FLA_INT)
        PH = FLA_Obj()
        L.FLASH_Obj_create_hier_copy_of_flat(P.obj, C.c_ulong(1), C.byref(b), C.byref(PH))
        t0 = time.perf_counter()
        r = L.FLASH_LU_piv(H, PH)
        dt = time.perf_counter() - t0
        L.FLASH_Obj_flatten(PH, P.obj)
        L.FLASH_Obj_free(C.byref(PH))
        extra = P.a.ravel().copy()
    else:
        t0 = time.perf_counter()
        r = L.FLASH_Chol(FLA_LOWER_TRIANGULAR, H)
        dt = time.perf_counter() - t0
        extra = None
    L.FLASH_Obj_flatten(H, M.obj)
    L.FLASH_Obj_free(C.byref(H))
    return M.a, extra, r, dt


def lu_piv_flash(A, nthreads, block=256):
    a, p, r, dt = _flash_run("lu", A, nthreads, block)
    return a, p, r, dt


def chol_flash(A, nthreads, block=256):
    a, _, r, dt = _flash_run("chol", A, nthreads, block)
    return a, r, dt


def dormqr(side, trans, QR, tau, Cm):
    """dormqr_ (src/map/lapack2flamec/FLA_ormqr.c:35-97)."""
    L = lib()
    a = np.array(QR, dtype=np.float64, order="F", copy=True)
    c = np.array(Cm, dtype=np.float64, order="F", copy=True)
    t = np.array(tau, dtype=np.float64, copy=True)
    m, n = c.shape
    k = len(t)
    nw = n if side == "L" else m
    work = np.zeros(max(1, nw) * 64)
    info = C.c_int(0)
    L.dormqr_(C.c_char_p(side.encode()), C.c_char_p(trans.encode()), _ip(m), _ip(n), _ip(k),
              a.ctypes.data_as(C.c_void_p), _ip(max(a.shape[0], 1)), t.ctypes.data_as(C.c_void_p),
              c.ctypes.data_as(C.c_void_p), _ip(max(m, 1)), work.ctypes.data_as(C.c_void_p),
              _ip(len(work)), C.byref(info))
    return c, info.value


def dorgqr(QR, tau, n):
    """dorgqr_ (src/map/lapack2flamec/FLA_orgqr.c:30-80) on the first n columns."""
    L = lib()
    a = np.array(QR[:, :n], dtype=np.float64, order="F", copy=True)
    t = np.array(tau, dtype=np.float64, copy=True)
    m = a.shape[0]
    k = len(t)
    work = np.zeros(max(1, n) * 64)
    info = C.c_int(0)
    L.dorgqr_(_ip(m), _ip(n), _ip(k), a.ctypes.data_as(C.c_void_p), _ip(max(m, 1)),
              t.ctypes.data_as(C.c_void_p), work.ctypes.data_as(C.c_void_p), _ip(len(work)), C.byref(info))
    return a, info.value


def dpotri(Afac, uplo="L"):
    """dpotri_ (src/map/lapack2flamec/FLA_potri.c:25-56)."""
    L = lib()
    a = np.array(Afac, dtype=np.float64, order="F", copy=True)
    n = a.shape[0]
    info = C.c_int(0)
    L.dpotri_(C.c_char_p(uplo.encode()), _ip(n), a.ctypes.data_as(C.c_void_p), _ip(max(n, 1)), C.byref(info))
    return a, info.value


def openblas_threads(n):
    """Thread count of the OpenBLAS behind the "openblas" build."""
    L = lib(kind="openblas")
    f = getattr(L, "scipy_openblas_set_num_threads", None)
    if f is None:
        import glob
        import scipy
        d = os.path.realpath(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs"))
        f = C.CDLL(sorted(glob.glob(os.path.join(d, "libscipy_openblas*.so")))[0]).scipy_openblas_set_num_threads
    f(int(n))


def timed_call(op, A, kind="openblas"):
    """Seconds taken by one reference FLA_LU_piv (op "lu") or lower FLA_Chol
    (op "chol") on a copy of A, the copy into the reference's buffer
    excluded.  Returns (seconds, return value)."""
    import time
    L = lib(kind=kind)
    M = _Mat(L, A)
    if op == "lu":
        P = _Mat(L, np.zeros(min(M.a.shape), dtype=np.int32), np.int32, FLA_INT)
        t0 = time.perf_counter()
        r = L.FLA_LU_piv(M.obj, P.obj)
    else:
        t0 = time.perf_counter()
        r = L.FLA_Chol(FLA_LOWER_TRIANGULAR, M.obj)
    return time.perf_counter() - t0, r
