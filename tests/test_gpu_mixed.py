"""Mixed-precision solvers (16-bit tensor-core factorization, FP64
refinement) against the FP64 oracle.

Bars (the mixed solution must reach the FP64 form's backward error): the normwise
backward error max_c ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) of
the mixed solution is at most 4x that of the oracle's FP64 LU/Cholesky
solution on the same system (and below 1e-15 absolute slack), and the
forward error against the oracle's solution is within kappa * 1e-14.  The
16-bit GEMM itself is checked against a float64 product of the rounded
operands (relative 1e-5: FP32 accumulation)."""
import ctypes as C

import numpy as np
import pytest

from conftest import rel_fro, seeded, to_dev, to_host

pytestmark = pytest.mark.gpu


def conditioned(rng, n, kappa, spd):
    """A = Q diag(s) Q^T (SPD) or U diag(s) V^T, s log-spaced 1 .. 1/kappa."""
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    s = np.logspace(0, -np.log10(kappa), n)
    if spd:
        A = (Q * s) @ Q.T
        return (A + A.T) / 2
    V, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * s) @ V.T


def backward_error(A, X, B):
    R = B - A @ X
    an = np.abs(A).sum(axis=1).max()
    return max(np.abs(R[:, c]).max() / (an * np.abs(X[:, c]).max() + np.abs(B[:, c]).max())
               for c in range(B.shape[1]))


@pytest.mark.parametrize("prec,name", [(0, "bfloat16"), (1, "float16"), (2, None), (3, None)])
@pytest.mark.parametrize("m,n,k", [(300, 200, 128), (1000, 700, 256), (64, 64, 40), (2049, 513, 1000),
                                   (128, 128, 64), (257, 129, 8)])
def test_lp_gemm_matches_rounded_product(cuda, flame, prec, name, m, n, k):
    torch = cuda
    g = torch.Generator(device="cuda").manual_seed(m + n + k + prec)
    A = torch.randn((k, m), dtype=torch.float32, device="cuda", generator=g).t()  # column-major m x k
    B = torch.randn((k, n), dtype=torch.float32, device="cuda", generator=g).t()
    Cm = torch.randn((n, m), dtype=torch.float32, device="cuda", generator=g).t()
    C0 = Cm.clone()
    rc = flame.lib().FLA_B200_lp_gemm(prec, m, n, k, -1.0, C.c_void_p(A.data_ptr()), m, C.c_void_p(B.data_ptr()), n,
                                      1.0, C.c_void_p(Cm.data_ptr()), m)
    assert rc == flame.FLA_SUCCESS, flame.last_error()
    if name is None:  # 3xTF32 / split FP16: FP32-accurate products of the FP32 operands
        ref = C0.double() - A.double() @ B.double().t()
    else:
        dt = getattr(torch, name)
        ref = C0.double() - A.to(dt).double() @ B.to(dt).double().t()
    err = ((Cm.double() - ref).abs().max() / ref.abs().max()).item()
    assert err < 1e-5, err


def _oracle_lu_solution(oracle, A, B):
    LU, p, r = oracle.lu_piv(A)
    assert r == -1
    return oracle.lu_piv_solve(LU, p, B)


@pytest.mark.parametrize("n,kappa", [(300, 1e2), (1000, 1e5)])
@pytest.mark.parametrize("prec", [0, 1, 2, 3])
@pytest.mark.parametrize("solver", [0, 1])
def test_lu_solve_mixed_matches_oracle(cuda, flame, oracle, n, kappa, prec, solver):
    rng = seeded(n + int(np.log10(kappa)) + 10 * prec + 100 * solver)
    A = conditioned(rng, n, kappa, spd=False)
    B = rng.standard_normal((n, 4))
    Ad, Bd = to_dev(cuda, A), to_dev(cuda, B)
    Xd = to_dev(cuda, np.zeros_like(B))
    r, it, inner = flame.lu_piv_solve_mixed(Ad, Bd, Xd, prec, solver)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    assert np.array_equal(to_host(Ad), A)  # A unchanged
    X = to_host(Xd)
    Xo = _oracle_lu_solution(oracle, A, B)
    be, be_o = backward_error(A, X, B), backward_error(A, Xo, B)
    assert be <= max(4 * be_o, 1e-15), (be, be_o, it)
    assert rel_fro(X, Xo) <= kappa * 1e-14, (rel_fro(X, Xo), it)
    # converges (after escalating to 3xTF32 when the 16-bit factors stall)
    assert it >= 0, "refinement should converge here (iter=%d)" % it


@pytest.mark.parametrize("n,kappa", [(300, 1e2), (1000, 1e8)])
@pytest.mark.parametrize("spd", [False, True])
def test_adaptive_solver(cuda, flame, oracle, n, kappa, spd):
    """solver 2: classic refinement while it contracts fast, else the FP64
    factorization (iter < 0); either way the FP64 form's accuracy."""
    rng = seeded(n + int(np.log10(kappa)) + (5 if spd else 0))
    A = conditioned(rng, n, kappa, spd=spd)
    B = rng.standard_normal((n, 4))
    Ad, Bd = to_dev(cuda, A), to_dev(cuda, B)
    Xd = to_dev(cuda, np.zeros_like(B))
    if spd:
        r, it, inner = flame.chol_solve_mixed(Ad, Bd, Xd, flame.FLA_LOWER_TRIANGULAR, 1, 2)
        Lo, ro = oracle.chol(A)
        Xo = oracle.chol_solve(Lo, B)
    else:
        r, it, inner = flame.lu_piv_solve_mixed(Ad, Bd, Xd, 1, 2)
        Xo = _oracle_lu_solution(oracle, A, B)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    assert inner == 0
    X = to_host(Xd)
    be, be_o = backward_error(A, X, B), backward_error(A, Xo, B)
    assert be <= max(4 * be_o, 1e-15), (be, be_o, it)
    if kappa <= 1e2:
        assert it >= 0, "fast contraction: the 16-bit factors suffice (iter=%d)" % it


@pytest.mark.parametrize("n,kappa", [(300, 1e2), (1000, 1e5), (1000, 1e8)])
@pytest.mark.parametrize("uplo", ["L", "U"])
def test_chol_solve_mixed_matches_oracle(cuda, flame, oracle, n, kappa, uplo):
    rng = seeded(n + int(np.log10(kappa)) + (7 if uplo == "U" else 0))
    A = conditioned(rng, n, kappa, spd=True)
    B = rng.standard_normal((n, 3))
    # only the uplo triangle is read: poison the other one
    Ain = np.tril(A) + np.triu(np.full_like(A, np.nan), 1) if uplo == "L" else \
        np.triu(A) + np.tril(np.full_like(A, np.nan), -1)
    Ad, Bd = to_dev(cuda, Ain), to_dev(cuda, B)
    Xd = to_dev(cuda, np.zeros_like(B))
    fu = flame.FLA_LOWER_TRIANGULAR if uplo == "L" else flame.FLA_UPPER_TRIANGULAR
    r, it, inner = flame.chol_solve_mixed(Ad, Bd, Xd, fu, 1, 1)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    X = to_host(Xd)
    Lo, ro = oracle.chol(A)
    assert ro == -1
    Xo = oracle.chol_solve(Lo, B)
    be, be_o = backward_error(A, X, B), backward_error(A, Xo, B)
    assert be <= max(4 * be_o, 1e-15), (be, be_o, it, inner)
    assert rel_fro(X, Xo) <= kappa * 1e-14, (rel_fro(X, Xo), it)
    assert it >= 0, (it, inner)


@pytest.mark.parametrize("n,kappa,max_iter", [(1000, 1e2, 5), (1000, 1e5, 12)])
@pytest.mark.parametrize("spd", [True, False])
def test_split_fp16_factors_converge_with_classic_refinement(cuda, flame, oracle, n, kappa, max_iter, spd):
    """prec 3: FP16 hi/lo split operands, three tensor-core products per
    update (FP32-accurate factors): classic refinement alone converges at
    kappa up to 1e5, to the FP64 oracle's backward error."""
    rng = seeded(n + int(np.log10(kappa)) + (0 if spd else 99))
    A = conditioned(rng, n, kappa, spd=spd)
    B = rng.standard_normal((n, 4))
    Ad, Bd = to_dev(cuda, A), to_dev(cuda, B)
    Xd = to_dev(cuda, np.zeros_like(B))
    if spd:
        r, it, inner = flame.chol_solve_mixed(Ad, Bd, Xd, flame.FLA_LOWER_TRIANGULAR, 3, 0)
        Lo, _ = oracle.chol(A)
        Xo = oracle.chol_solve(Lo, B)
    else:
        r, it, inner = flame.lu_piv_solve_mixed(Ad, Bd, Xd, 3, 0)
        Xo = _oracle_lu_solution(oracle, A, B)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    X = to_host(Xd)
    assert 0 <= it <= max_iter, it
    assert backward_error(A, X, B) <= max(4 * backward_error(A, Xo, B), 1e-15)
    assert rel_fro(X, Xo) <= kappa * 1e-14


def test_chol_solve_mixed_falls_back(cuda, flame, oracle):
    """kappa = 1e15: the 16-bit Cholesky breaks down or refinement stalls;
    the FP64 factorization of a copy produces X (iter < 0)."""
    n = 400
    rng = seeded(77)
    A = conditioned(rng, n, 1e15, spd=True) + 1e-13 * np.eye(n)
    B = rng.standard_normal((n, 2))
    Ad, Bd = to_dev(cuda, A), to_dev(cuda, B)
    Xd = to_dev(cuda, np.zeros_like(B))
    r, it, inner = flame.chol_solve_mixed(Ad, Bd, Xd, flame.FLA_LOWER_TRIANGULAR, 0, 0)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    assert it in (-3, -31), it
    assert np.array_equal(to_host(Ad), A)
    Lo, ro = oracle.chol(A)
    Xo = oracle.chol_solve(Lo, B)
    assert backward_error(A, to_host(Xd), B) <= max(4 * backward_error(A, Xo, B), 1e-15)


def test_dsgesv_lapack_abi(cuda, flame, oracle):
    n, nrhs = 513, 5
    rng = seeded(5)
    A = conditioned(rng, n, 1e3, spd=False)
    B = rng.standard_normal((n, nrhs))
    a = np.asfortranarray(A.copy())
    b = np.asfortranarray(B.copy())
    x = np.asfortranarray(np.zeros((n, nrhs)))
    ipiv = np.zeros(n, dtype=np.int32)
    nn, nr, ld = C.c_int(n), C.c_int(nrhs), C.c_int(n)
    it, info = C.c_int(0), C.c_int(0)
    P = lambda arr: arr.ctypes.data_as(C.c_void_p)  # noqa: E731
    flame.lib().dsgesv_(C.byref(nn), C.byref(nr), P(a), C.byref(ld), P(ipiv), P(b), C.byref(ld), P(x),
                        C.byref(ld), None, None, C.byref(it), C.byref(info))
    assert info.value == 0 and it.value >= 0, (info.value, it.value)
    assert np.array_equal(a, A)  # A unchanged after converged refinement
    assert ipiv.min() >= 1 and ipiv.max() <= n
    Xo = _oracle_lu_solution(oracle, A, B)
    assert backward_error(A, x, B) <= max(4 * backward_error(A, Xo, B), 1e-15)
    # argument check: n < 0 -> info = -1 (xerbla)
    bad = C.c_int(-1)
    flame.lib().dsgesv_(C.byref(bad), C.byref(nr), P(a), C.byref(ld), P(ipiv), P(b), C.byref(ld), P(x),
                        C.byref(ld), None, None, C.byref(it), C.byref(info))
    assert info.value == -1


def test_dsposv_lapack_abi(cuda, flame, oracle):
    n, nrhs = 700, 3
    rng = seeded(6)
    A = conditioned(rng, n, 1e4, spd=True)
    B = rng.standard_normal((n, nrhs))
    a = np.asfortranarray(np.triu(A))
    b = np.asfortranarray(B.copy())
    x = np.asfortranarray(np.zeros((n, nrhs)))
    nn, nr, ld = C.c_int(n), C.c_int(nrhs), C.c_int(n)
    it, info = C.c_int(0), C.c_int(0)
    P = lambda arr: arr.ctypes.data_as(C.c_void_p)  # noqa: E731
    flame.lib().dsposv_(C.c_char_p(b"U"), C.byref(nn), C.byref(nr), P(a), C.byref(ld), P(b), C.byref(ld), P(x),
                        C.byref(ld), None, None, C.byref(it), C.byref(info))
    assert info.value == 0, info.value
    Lo, _ = oracle.chol(A)
    Xo = oracle.chol_solve(Lo, B)
    assert backward_error(A, x, B) <= max(4 * backward_error(A, Xo, B), 1e-15), it.value
