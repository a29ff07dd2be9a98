"""The allocation-free panel entry point, FLA_B200_LU_piv_panel_noalloc.

It exists for callers that cannot let the library call cudaMalloc (their
own allocator owns the device memory, or they cannot afford the
synchronization cudaMalloc/cudaFree may cause).  It factors one panel with
the LU panel kernel, keeping that kernel's scratch in a fixed device array
that ships with the library.  Here it is called through the C-ABI and its
output is checked against the existing entry point FLA_LU_piv on the same
panels, on two calls in a row (same tolerance as the LU parity tests:
factors within 1e-12 normwise, identical pivots, identical return code).

This file is named so pytest collects it last; it must pass both alone in a
fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_fro, seeded, to_dev, to_host

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-12


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


def test_noalloc_panel_rejects_sizes_beyond_its_limits(cuda, flame):
    torch = cuda
    Ad = torch.zeros((300, 200), dtype=torch.float64, device="cuda").t().contiguous().t()
    p = torch.zeros(200, dtype=torch.int32, device="cuda")
    assert _noalloc(flame, Ad, p) == flame.FLA_FAILURE
    assert "n <= 128" in flame.last_error()
