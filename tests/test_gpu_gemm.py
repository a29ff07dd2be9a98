"""The FP64 DMMA GEMM engine against a plain torch fp64 reference
(C := alpha op(A) op(B) + beta C, the four transposition cases, the
lower-triangle mode used by the Cholesky update, ragged sizes)."""
import ctypes as C

import numpy as np
import pytest

from conftest import seeded

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (128, 64, 16), (130, 70, 33), (300, 257, 128), (513, 190, 200),
                                   # few output tiles, long K: split-K slices and their ordered reduction
                                   (32, 64, 16384), (64, 130, 5000), (33, 7, 3001),
                                   # at most 32 columns, long K: 128 x 32 tiles, split K (refinement residuals)
                                   (4099, 32, 8192), (1000, 17, 2048)])
def test_dgemm_matches_torch(cuda, flame, ta, tb, m, n, k):
    torch = cuda
    g = torch.Generator(device="cuda").manual_seed(m * 1000 + n * 10 + k + 7 * ta + 3 * tb)
    A = torch.randn((k, m) if ta else (m, k), dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn((n, k) if tb else (k, n), dtype=torch.float64, device="cuda", generator=g)
    Cm = torch.randn((m, n), dtype=torch.float64, device="cuda", generator=g)
    # column-major copies with an even leading dimension
    def cm(t):
        r, c = t.shape
        ld = r + (r & 1)
        buf = torch.zeros((c, ld), dtype=torch.float64, device="cuda")
        buf[:, :r] = t.t()
        return buf, ld
    Ab, lda = cm(A)
    Bb, ldb = cm(B)
    Cb, ldc = cm(Cm)
    alpha, beta = -1.0, 1.0
    rc = flame.lib().FLA_B200_dgemm(ta, tb, m, n, k, alpha, C.c_void_p(Ab.data_ptr()), lda,
                                    C.c_void_p(Bb.data_ptr()), ldb, beta, C.c_void_p(Cb.data_ptr()), ldc, 0)
    assert rc == flame.FLA_SUCCESS, flame.last_error()
    opA = A.t() if ta else A
    opB = B.t() if tb else B
    ref = alpha * (opA @ opB) + beta * Cm
    got = Cb[:, :m].t()
    err = (got - ref).abs().max().item() / max(1.0, ref.abs().max().item())
    assert err < 1e-13 * max(1, k) ** 0.5


def test_dgemm_lower_mode_leaves_upper_untouched(cuda, flame):
    torch = cuda
    n, k = 300, 128
    g = torch.Generator(device="cuda").manual_seed(5)
    A = torch.randn((n, k), dtype=torch.float64, device="cuda", generator=g)
    Cm = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
    Ab = A.t().contiguous()  # column-major n x k storage, ld = n
    Cb = Cm.t().contiguous()
    rc = flame.lib().FLA_B200_dgemm(0, 1, n, n, k, -1.0, C.c_void_p(Ab.data_ptr()), n,
                                    C.c_void_p(Ab.data_ptr()), n, 1.0, C.c_void_p(Cb.data_ptr()), n, 1)
    assert rc == flame.FLA_SUCCESS
    got = Cb.t()
    ref = Cm - A @ A.t()
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device="cuda"))
    assert (got[low] - ref[low]).abs().max().item() < 1e-12
    assert torch.equal(got[~low], Cm[~low])


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0)])
@pytest.mark.parametrize("alpha,beta", [(-1.0, 1.0), (0.5, 2.0), (1.0, 0.0)])
def test_dgemm_many_tiles(cuda, flame, ta, tb, alpha, beta):
    """More tiles than resident CTAs (several waves), general alpha/beta."""
    torch = cuda
    m, n, k = 2000, 3000, 144
    g = torch.Generator(device="cuda").manual_seed(11 + ta + 2 * tb)
    A = torch.randn((k, m) if ta else (m, k), dtype=torch.float64, device="cuda", generator=g)
    B = torch.randn((n, k) if tb else (k, n), dtype=torch.float64, device="cuda", generator=g)
    Cm = torch.randn((m, n), dtype=torch.float64, device="cuda", generator=g)
    Ab, Bb, Cb = A.t().contiguous(), B.t().contiguous(), Cm.t().contiguous()
    rc = flame.lib().FLA_B200_dgemm(ta, tb, m, n, k, alpha, C.c_void_p(Ab.data_ptr()), A.shape[0],
                                    C.c_void_p(Bb.data_ptr()), B.shape[0], beta,
                                    C.c_void_p(Cb.data_ptr()), m, 0)
    assert rc == flame.FLA_SUCCESS, flame.last_error()
    opA = A.t() if ta else A
    opB = B.t() if tb else B
    ref = alpha * (opA @ opB) + beta * Cm
    err = (Cb.t() - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-14 * k


def test_dgemm_lower_mode_many_tiles(cuda, flame):
    torch = cuda
    n, k = 2500, 128
    g = torch.Generator(device="cuda").manual_seed(6)
    A = torch.randn((n, k), dtype=torch.float64, device="cuda", generator=g)
    Cm = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
    Ab = A.t().contiguous()
    Cb = Cm.t().contiguous()
    rc = flame.lib().FLA_B200_dgemm(0, 1, n, n, k, -1.0, C.c_void_p(Ab.data_ptr()), n,
                                    C.c_void_p(Ab.data_ptr()), n, 1.0, C.c_void_p(Cb.data_ptr()), n, 1)
    assert rc == flame.FLA_SUCCESS
    got = Cb.t()
    ref = Cm - A @ A.t()
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device="cuda"))
    assert (got[low] - ref[low]).abs().max().item() < 1e-12
    assert torch.equal(got[~low], Cm[~low])


def test_gemm_concurrent_with_panel_work(flame):
    """The trailing-update GEMM with Cholesky-panel kernels beside it on the
    library's second stream (the factorizations' lookahead): 3000 updates of
    8192 x 8192 x 128, each bitwise equal to the update computed alone.  A
    stage-release race in the GEMM's shared-memory pipeline once gave, on
    some B200s, about one wrong tile per 3000 such updates (8 rows x 32
    columns fed by one warp's A fragment)."""
    bad = C.c_ulonglong(12345)
    rc = flame.lib().FLA_B200_gemm_concurrency_check(8192, 8192, 128, 3000, C.byref(bad))
    assert rc == flame.FLA_SUCCESS, flame.last_error()
    assert bad.value == 0


def test_gemm_concurrency_check_rejects_bad_arguments(flame):
    bad = C.c_ulonglong(0)
    assert flame.lib().FLA_B200_gemm_concurrency_check(0, 8, 8, 1, C.byref(bad)) == flame.FLA_FAILURE
    assert flame.lib().FLA_B200_gemm_concurrency_check(8, 8, 8, 1, None) == flame.FLA_FAILURE
