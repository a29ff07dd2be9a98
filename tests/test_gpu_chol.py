"""FLA_Chol on the GPU against the CPU oracle (the reference's algorithm,
pinned bit for bit to the reference library).

Tolerances (stated by the FP64 plain form): factors agree with the oracle
within 1e-12 normwise (relative Frobenius); the backward error
||A - L L^T||_F / (n eps ||A||_F) is at most the oracle's own plus 1.0
(the oracle's is already O(1), and both are computed in FP64 with
different summation orders); the failing column of a non-SPD matrix is
identical."""
import numpy as np
import pytest

from conftest import rel_fro, seeded, spd, to_dev, to_host

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-12


@pytest.mark.parametrize("n", [1, 2, 5, 31, 32, 33, 127, 128, 129, 200, 257, 500, 1024])
def test_chol_lower_matches_oracle(cuda, flame, oracle, n):
    rng = seeded(1000 + n)
    A = spd(rng, n)
    Ad = to_dev(cuda, A)
    r = flame.chol(Ad)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    L = to_host(Ad)
    Lo, ro = oracle.chol(A)
    assert ro == -1
    assert rel_fro(np.tril(L), np.tril(Lo)) < FACTOR_TOL
    # strictly upper part untouched
    assert np.array_equal(np.triu(L, 1), np.triu(A, 1))
    be, be_o = oracle.chol_backward_error(A, L), oracle.chol_backward_error(A, Lo)
    assert be <= be_o + 1.0, (be, be_o)


@pytest.mark.parametrize("n", [3, 130, 300])
def test_chol_upper_matches_oracle(cuda, flame, oracle, n):
    rng = seeded(2000 + n)
    A = spd(rng, n)
    Ad = to_dev(cuda, A)
    assert flame.chol(Ad, flame.FLA_UPPER_TRIANGULAR) == flame.FLA_SUCCESS
    U = to_host(Ad)
    Lo, _ = oracle.chol(A)
    assert rel_fro(np.triu(U), np.tril(Lo).T) < FACTOR_TOL
    assert np.array_equal(np.tril(U, -1), np.tril(A, -1))


def test_chol_golden_fixtures(cuda, flame, golden):
    for n in [1, 17, 64, 130]:
        A = golden["chol_l_%d_A" % n]
        Ad = to_dev(cuda, A)
        assert flame.chol(Ad) == flame.FLA_SUCCESS
        assert rel_fro(np.tril(to_host(Ad)), np.tril(golden["chol_l_%d_L" % n])) < FACTOR_TOL
    for n in [33, 150]:
        Ad = to_dev(cuda, golden["chol_u_%d_A" % n])
        assert flame.chol(Ad, flame.FLA_UPPER_TRIANGULAR) == flame.FLA_SUCCESS
        assert rel_fro(np.triu(to_host(Ad)), np.triu(golden["chol_u_%d_U" % n])) < FACTOR_TOL


@pytest.mark.parametrize("bad", [0, 37, 127, 128, 200])
def test_chol_reports_failing_column(cuda, flame, oracle, bad):
    rng = seeded(3000 + bad)
    A = spd(rng, 260)
    A[bad, bad] = -1.0
    Ad = to_dev(cuda, A)
    r = flame.chol(Ad)
    _, ro = oracle.chol(A)
    assert r == ro == bad


def test_chol_golden_failure(cuda, flame, golden):
    Ad = to_dev(cuda, golden["chol_fail_A"])
    assert flame.chol(Ad) == int(golden["chol_fail_r"])


def test_chol_host_buffer_and_odd_ld(cuda, flame, oracle):
    rng = seeded(77)
    n = 301
    A = spd(rng, n)
    # host buffer (staged through HBM)
    H = np.asfortranarray(A.copy())
    assert flame.chol(H) == flame.FLA_SUCCESS
    Lo, _ = oracle.chol(A)
    assert rel_fro(np.tril(H), np.tril(Lo)) < FACTOR_TOL
    # device view with an odd leading dimension (repacked for TMA)
    torch = cuda
    store = torch.zeros((n, n + 2), dtype=torch.float64, device="cuda")
    store[:, :n] = torch.from_numpy(A.T.copy()).cuda()
    view = store[:, :n].t()  # n x n column-major view, ld = n + 2 = 303 (odd)
    assert view.stride() == (1, n + 2)
    assert flame.chol(view) == flame.FLA_SUCCESS
    assert rel_fro(np.tril(view.cpu().numpy()), np.tril(Lo)) < FACTOR_TOL


def test_dpotrf_lapack_abi(cuda, flame, golden):
    import ctypes as C
    A = golden["dpotrf_A"]
    a = np.asfortranarray(A.copy())
    n = C.c_int(a.shape[0])
    info = C.c_int(99)
    flame.lib().dpotrf_(C.c_char_p(b"U"), C.byref(n), a.ctypes.data_as(C.c_void_p), C.byref(n), C.byref(info))
    assert info.value == 0
    assert rel_fro(np.triu(a), np.triu(golden["dpotrf_U"])) < FACTOR_TOL
    # non-SPD: info = failing column + 1
    B = golden["chol_fail_A"]
    b = np.asfortranarray(B.copy())
    n = C.c_int(b.shape[0])
    flame.lib().dpotrf_(C.c_char_p(b"L"), C.byref(n), b.ctypes.data_as(C.c_void_p), C.byref(n), C.byref(info))
    assert info.value == int(golden["chol_fail_r"]) + 1


def test_chol_bitwise_repeatable(cuda, flame):
    """Five factorizations of one SPD matrix (n = 4096, several outer
    panels and trailing updates) give bitwise identical factors: no
    ordering-dependent work between the panel and the updates."""
    torch = cuda
    n = 4096
    g = torch.Generator(device="cuda").manual_seed(3)
    G = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g) / n ** 0.5
    S = G @ G.t() + torch.eye(n, dtype=torch.float64, device="cuda")
    W = torch.empty_like(S).t()
    ref = None
    for _ in range(5):
        W.copy_(S)
        torch.cuda.synchronize()
        assert flame.chol(W) == flame.FLA_SUCCESS
        L = torch.tril(W)
        if ref is None:
            ref = L.clone()
        else:
            assert torch.equal(L, ref)
