"""The allocation-free panel entry point, FLA_B200_LU_piv_panel_noalloc.

It exists for callers that cannot let the library call cudaMalloc (their
own allocator owns the device memory, or they cannot afford the
synchronization cudaMalloc/cudaFree may cause).  It factors one panel with
the LU panel kernel, keeping that kernel's scratch in a fixed device array
that ships with the library.  Here it is called through the C-ABI and its
output is checked against the existing entry point FLA_LU_piv on the same
panels, on two calls in a row (same tolerance as the LU parity tests:
factors within 1e-12 normwise, identical pivots, identical return code),
and against the CPU oracle directly.

This file is named so pytest collects it last; it must pass both alone in a
fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_fro, seeded, to_dev, to_host

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-12
# Shared-memory budget of the panel kernel for its row slab (bytes); the
# slab is lds x n doubles plus one row, lds = R | 1, R = ceil(m / SMs).
SLAB_SMEM_CAP = 200 * 1024


def _noalloc(flame, Ad, p):
    m, n = Ad.shape
    L = flame.lib()
    f = L.FLA_B200_LU_piv_panel_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    return f(m, n, C.c_void_p(Ad.data_ptr()), Ad.stride(1), C.c_void_p(p.data_ptr()), None)


def _existing(cuda, flame, A):
    Ad = to_dev(cuda, A)
    p = cuda.zeros(A.shape[1], dtype=cuda.int32, device="cuda")
    r = flame.lu_piv(Ad, p)
    return to_host(Ad), p.cpu().numpy(), r


def _padded(torch, A, pad):
    """Column-major device copy of A with leading dimension m + pad."""
    m, n = A.shape
    buf = torch.zeros((n, m + pad), dtype=torch.float64, device="cuda")
    buf[:, :m] = torch.from_numpy(np.ascontiguousarray(A.T)).cuda()
    return buf.t()[:m, :]


def test_noalloc_panel_matches_FLA_LU_piv_two_calls_in_a_row(cuda, flame):
    torch = cuda
    rng = seeded(4242)
    cases = [rng.uniform(-1, 1, (3000, 96)), rng.uniform(-1, 1, (700, 128))]
    # second panel gets a zero column: the first call leaves a null-pivot
    # record in the shared scratch, the next call must start from a clean one
    cases[1][:, 5] = 0.0
    cases.append(rng.uniform(-1, 1, (1500, 64)))
    for A in cases:
        LUe, pe, re_ = _existing(cuda, flame, A)
        Ad = to_dev(cuda, A)
        p = torch.zeros(A.shape[1], dtype=torch.int32, device="cuda")
        r = _noalloc(flame, Ad, p)
        assert r == re_, (r, re_, flame.last_error())
        assert np.array_equal(p.cpu().numpy(), pe)
        assert rel_fro(to_host(Ad), LUe) < FACTOR_TOL


def test_noalloc_panel_matches_the_oracle(cuda, flame, oracle):
    torch = cuda
    A = seeded(99).uniform(-1, 1, (2500, 128))
    LUo, po, ro = oracle.lu_piv(A)
    for _ in range(2):
        Ad = to_dev(cuda, A)
        p = torch.zeros(128, dtype=torch.int32, device="cuda")
        r = _noalloc(flame, Ad, p)
        assert r == ro, flame.last_error()
        assert np.array_equal(p.cpu().numpy(), po)
        assert rel_fro(to_host(Ad), LUo) < FACTOR_TOL


def test_noalloc_panel_nan_column_keeps_pivots_in_range(cuda, flame):
    # a column whose candidates are all NaN: no orderable pivot; the pivot
    # vector must stay in range and agree with FLA_LU_piv's leaf kernels
    torch = cuda
    A = seeded(5).uniform(-1, 1, (900, 48))
    A[:, 7] = np.nan
    LUe, pe, re_ = _existing(cuda, flame, A)
    for _ in range(2):
        Ad = to_dev(cuda, A)
        p = torch.zeros(48, dtype=torch.int32, device="cuda")
        r = _noalloc(flame, Ad, p)
        pv = p.cpu().numpy()
        assert r == re_, flame.last_error()
        assert np.array_equal(pv, pe)
        assert np.all(pv >= 0) and np.all(pv + np.arange(48) < 900)


def _max_rows(sms, n):
    """Largest m the panel kernel's geometry accepts for n columns."""
    best = 0
    for R in range(1, 4096):
        lds = R | 1
        if lds * n * 8 + n * 8 <= SLAB_SMEM_CAP:
            best = R
    return sms * best


def test_noalloc_panel_at_its_size_limit(cuda, flame, oracle):
    torch = cuda
    n = 128
    m = _max_rows(flame.num_sms(), n)
    A = seeded(11).uniform(-1, 1, (m, n))
    LUo, po, ro = oracle.lu_piv(A)
    Ad = _padded(torch, A, 8)
    p = torch.zeros(n, dtype=torch.int32, device="cuda")
    r = _noalloc(flame, Ad, p)
    assert r == ro, flame.last_error()
    assert np.array_equal(p.cpu().numpy(), po)
    assert rel_fro(Ad.cpu().numpy(), LUo) < FACTOR_TOL
    # one row more no longer fits the slab: rejected, nothing written
    B = _padded(torch, seeded(12).uniform(-1, 1, (m + 1, n)), 8)
    B0 = B.clone()
    assert _noalloc(flame, B, p) == flame.FLA_FAILURE
    assert "limits" in flame.last_error()
    assert torch.equal(B, B0)


def test_noalloc_panel_rejects_sizes_beyond_its_limits(cuda, flame):
    torch = cuda
    Ad = torch.zeros((300, 200), dtype=torch.float64, device="cuda").t().contiguous().t()
    p = torch.zeros(200, dtype=torch.int32, device="cuda")
    assert _noalloc(flame, Ad, p) == flame.FLA_FAILURE
    assert "n <= 128" in flame.last_error()
