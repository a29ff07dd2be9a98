"""Cholesky adjoint (FLA_Chol_adjoint), log-determinant and triangular-solve
adjoints, and the Gaussian-process likelihood gradient built from them.

Checks: (1) the symmetric gradient (Abar + Abar^T)/2 against the closed form
L^-T sym(Phi(L^T Lbar)) L^-1 evaluated with the oracle's factor (relative
1e-10); (2) a central finite difference (h = 1e-6) of f(A) = <Lbar, chol(A)>
along random symmetric directions; (3) the GP gradient dloss/dK =
0.5 (K^-1 - alpha alpha^T) from the oracle's FLA_Chol + triangular solves,
and central differences on 200 random entries (relative 1e-5)."""
import numpy as np
import pytest

from conftest import rel_fro, seeded, spd, to_dev, to_host

pytestmark = pytest.mark.gpu


def closed_form(L, Lbar):
    P = L.T @ np.tril(Lbar)
    P = np.tril(P) - 0.5 * np.diag(np.diag(P))
    Ps = 0.5 * (P + P.T)
    Li = np.linalg.inv(L)
    return Li.T @ Ps @ Li


@pytest.mark.parametrize("n", [1, 5, 127, 128, 129, 300, 520])
def test_chol_adjoint_closed_form(cuda, flame, oracle, n):
    rng = seeded(n + 3)
    A = spd(rng, n)
    Lo, ro = oracle.chol(A)
    assert ro == -1
    L = np.tril(Lo)
    Lbar = np.tril(rng.standard_normal((n, n)))
    Ld, Bd = to_dev(cuda, L), to_dev(cuda, Lbar)
    assert flame.chol_adjoint(Ld, Bd) == flame.FLA_SUCCESS, flame.last_error()
    Ab = np.tril(to_host(Bd))
    S = 0.5 * (Ab + Ab.T)
    assert rel_fro(S, closed_form(L, Lbar)) < 1e-10
    # the strict upper triangle of Lbar is left alone
    assert np.array_equal(np.triu(to_host(Bd), 1), np.triu(to_dev(cuda, Lbar).cpu().numpy(), 1))


def test_chol_adjoint_finite_differences(cuda, flame, oracle):
    n, h = 96, 1e-6
    rng = seeded(17)
    A = spd(rng, n)
    Lbar = np.tril(rng.standard_normal((n, n)))
    L = np.tril(oracle.chol(A)[0])
    Ld, Bd = to_dev(cuda, L), to_dev(cuda, Lbar)
    assert flame.chol_adjoint(Ld, Bd) == flame.FLA_SUCCESS
    Ab = np.tril(to_host(Bd))
    S = 0.5 * (Ab + Ab.T)
    f = lambda M: np.sum(Lbar * np.tril(oracle.chol(M)[0]))  # noqa: E731
    for _ in range(5):
        E = rng.standard_normal((n, n))
        E = (E + E.T) / 2
        fd = (f(A + h * E) - f(A - h * E)) / (2 * h)
        an = np.sum(S * E)
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(an)), (fd, an)


def _gp(rng, n):
    x = rng.uniform(0, 1, (n, 3))
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    K = np.exp(-d2 / (2 * 0.3 ** 2)) + 1e-2 * np.eye(n)
    y = rng.standard_normal((n, 1))
    return K, y


def gp_loss_and_grad(cuda, flame, K, y):
    """loss = 0.5 y^T K^-1 y + sum log L_ii and dloss/dK (symmetric), through
    FLA_Chol, the triangular solves and the three adjoints."""
    n = K.shape[0]
    Ld = to_dev(cuda, K)
    assert flame.chol(Ld) == flame.FLA_SUCCESS
    L = np.tril(to_host(Ld))
    Ld = to_dev(cuda, L)
    v = np.linalg.solve(L, y)              # forward quantities (host, for the check only)
    alpha = np.linalg.solve(L.T, v)
    loss = 0.5 * (y.T @ alpha).item() + float(np.log(np.diag(L)).sum())
    # reverse: loss1 = 0.5 v^T v, v = inv(L) y  ->  vbar = v
    Lbar = to_dev(cuda, np.zeros((n, n)))
    Vd, Vb = to_dev(cuda, v), to_dev(cuda, v.copy())
    assert flame.trsm_llnn_adjoint(Ld, Vd, Vb, Lbar) == flame.FLA_SUCCESS, flame.last_error()
    r, logdet = flame.chol_logdet_adjoint(Ld, Lbar, 1.0)
    assert r == flame.FLA_SUCCESS
    assert abs(logdet - np.log(np.diag(L)).sum()) < 1e-9 * max(1.0, abs(logdet))
    assert flame.chol_adjoint(Ld, Lbar) == flame.FLA_SUCCESS
    Ab = np.tril(to_host(Lbar))
    return loss, 0.5 * (Ab + Ab.T)


def test_gp_gradient_matches_oracle_and_fd(cuda, flame, oracle):
    n = 300
    rng = seeded(99)
    K, y = _gp(rng, n)
    loss, G = gp_loss_and_grad(cuda, flame, K, y)
    # oracle: K^-1 from FLA_Chol + two triangular solves on I, alpha likewise
    Lo, ro = oracle.chol(K)
    assert ro == -1
    Kinv = oracle.chol_solve(Lo, np.eye(n))
    alpha = oracle.chol_solve(Lo, y)
    G_ref = 0.5 * (Kinv - alpha @ alpha.T)
    assert rel_fro(G, G_ref) < 1e-9
    # central differences on 200 random symmetric entries
    h = 1e-6
    idx = rng.integers(0, n, size=(200, 2))

    def loss_of(M):
        L = np.tril(oracle.chol(M)[0])
        v = np.linalg.solve(L, y)
        return 0.5 * (v.T @ v).item() + float(np.log(np.diag(L)).sum())
    for i, j in idx[:200:10]:  # 20 oracle evaluations per sign keep the CPU suite short
        E = np.zeros((n, n))
        E[i, j] += 1
        E[j, i] += 1 if i != j else 0
        fd = (loss_of(K + h * E) - loss_of(K - h * E)) / (2 * h)
        an = np.sum(G * E)
        assert abs(fd - an) <= 1e-5 * max(1.0, abs(an)), (i, j, fd, an)


def _colmajor(t):
    """A column-major copy of a 2-D tensor (stride(1) = rows, also for one column)."""
    import torch
    out = torch.empty_strided(tuple(t.shape), (1, t.shape[0]), dtype=t.dtype, device=t.device)
    out.copy_(t)
    return out


def test_gp_gradient_n8192_sampled_oracle_and_fd(cuda, flame, oracle):
    """The GP gradient at n = 8192 (one GP of the batched-GP workload): the
    adjoint chain's dloss/dK against 0.5 (K^-1 - alpha alpha^T) on 200
    sampled entries, with the needed columns of K^-1 and alpha from the
    oracle's triangular solves on the factor (CPU), and against central
    differences of the loss on the same 200 entries, each loss evaluated by
    FLA_Chol on the GPU."""
    torch = cuda
    # the GP of the benchmark configuration: length scale 0.3, nugget 1e-2,
    # central differences with h = 1e-6.  Their rounding noise at this size
    # is ~2e-5 relative (the loss is O(1e4) and K's condition number ~1e5),
    # so they are held to 1e-4; the entry-wise oracle comparison is the
    # tight check (1e-9).
    n, h, fd_tol = 8192, 1e-6, 1e-4
    g = torch.Generator(device="cuda").manual_seed(8192)
    x = torch.rand((n, 3), dtype=torch.float64, device="cuda", generator=g)
    K = torch.exp(-torch.cdist(x, x) ** 2 / (2 * 0.3 ** 2)) + 1e-2 * torch.eye(n, dtype=torch.float64, device="cuda")
    K = _colmajor(0.5 * (K + K.t()))
    y = torch.randn((n, 1), dtype=torch.float64, device="cuda", generator=g)
    Ld = _colmajor(K)
    assert flame.chol(Ld) == flame.FLA_SUCCESS, flame.last_error()
    Lt = _colmajor(torch.tril(Ld))
    v = torch.linalg.solve_triangular(Lt, y, upper=False)
    Lbar = _colmajor(torch.zeros((n, n), dtype=torch.float64, device="cuda"))
    Vd, Vb = _colmajor(v), _colmajor(v)
    assert flame.trsm_llnn_adjoint(Lt, Vd, Vb, Lbar) == flame.FLA_SUCCESS, flame.last_error()
    r, logdet = flame.chol_logdet_adjoint(Lt, Lbar, 1.0)
    assert r == flame.FLA_SUCCESS
    assert flame.chol_adjoint(Lt, Lbar) == flame.FLA_SUCCESS, flame.last_error()
    Ab = torch.tril(Lbar)
    Gh = (0.5 * (Ab + Ab.t())).cpu().numpy()
    del Ab, Lbar, Vd, Vb, Ld
    rng = seeded(8192)
    idx = rng.integers(0, n, size=(200, 2))
    # oracle: the needed columns of K^-1 and alpha = K^-1 y from the factor
    L = np.asfortranarray(Lt.cpu().numpy())
    cols = np.unique(idx[:, 1])
    E = np.zeros((n, cols.size + 1), order="F")
    E[cols, np.arange(cols.size)] = 1.0
    E[:, -1] = y.cpu().numpy()[:, 0]
    Z = oracle.chol_solve(L, E)
    Kinv_cols, alpha = Z[:, :-1], Z[:, -1]
    where = {c: k for k, c in enumerate(cols)}
    for i, j in idx:
        ref = 0.5 * (Kinv_cols[i, where[j]] - alpha[i] * alpha[j])
        assert abs(Gh[i, j] - ref) <= 1e-9 * max(1.0, abs(ref)), (i, j, Gh[i, j], ref)

    def loss_of(i, j, d):
        M = K.clone()
        M[i, j] += d
        if i != j:
            M[j, i] += d
        assert flame.chol(M) == flame.FLA_SUCCESS
        Lm = torch.tril(M)
        vv = torch.linalg.solve_triangular(Lm, y, upper=False)
        return 0.5 * float((vv * vv).sum()) + float(torch.log(torch.diagonal(Lm)).sum())
    for i, j in idx:
        fd = (loss_of(i, j, h) - loss_of(i, j, -h)) / (2 * h)
        an = float(Gh[i, j]) * (1 if i == j else 2)
        assert abs(fd - an) <= fd_tol * max(1.0, abs(an)), (i, j, fd, an)
