"""Batched Cholesky / LU (+ solve) in one persistent launch, each matrix
against the oracle's single-matrix FLA_Chol / FLA_LU_piv on the same input.

Bars: FP64 factors within 1e-12 normwise relative of the oracle's, LU
pivots identical, identical failure columns, solutions within 1e-11
relative (well-conditioned systems); FP32 factors within 1e-4 (FP32
rounding over orders up to 512)."""
import numpy as np
import pytest

from conftest import rel_fro, seeded, spd, to_dev, to_host

pytestmark = pytest.mark.gpu


def _sizes(rng, count):
    # the edges of every panel / warp block, plus random orders up to 512
    fixed = [1, 2, 31, 32, 33, 64, 65, 127, 128, 129, 255, 257, 511, 512]
    return fixed + list(rng.integers(1, 513, size=count - len(fixed)))


@pytest.mark.parametrize("nrhs", [0, 4])
def test_chol_batched_matches_oracle(cuda, flame, oracle, nrhs):
    rng = seeded(11 + nrhs)
    sizes = _sizes(rng, 24)
    mats = [spd(rng, n) for n in sizes]
    # a non-SPD member: fails at a known column
    bad = 5
    mats[bad] = mats[bad].copy()
    mats[bad][10, 10] = -1.0
    dev = [to_dev(cuda, A) for A in mats]
    rhs = [rng.standard_normal((n, nrhs)) for n in sizes] if nrhs else None
    drhs = [to_dev(cuda, b) for b in rhs] if nrhs else None
    r, info = flame.batched("chol", dev, rhs=drhs)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    for i, A in enumerate(mats):
        Lo, ro = oracle.chol(A)
        assert info[i] == ro, (i, sizes[i], info[i], ro)
        if ro != -1:
            continue
        L = np.tril(to_host(dev[i]))
        assert rel_fro(L, np.tril(Lo)) < 1e-12, (i, sizes[i])
        if nrhs:
            Xo = oracle.chol_solve(Lo, rhs[i])
            assert rel_fro(to_host(drhs[i]), Xo) < 1e-11, (i, sizes[i])


@pytest.mark.parametrize("nrhs", [0, 4])
def test_lu_batched_matches_oracle(cuda, flame, oracle, nrhs):
    rng = seeded(21 + nrhs)
    sizes = _sizes(rng, 24)
    mats = [rng.uniform(-1, 1, (n, n)) for n in sizes]
    # zero column: reported, factorization goes on
    zc = 7
    mats[zc] = mats[zc].copy()
    mats[zc][:, 3] = 0.0
    # exact ties in the pivot column
    mats[9] = mats[9].copy()
    mats[9][:, 0] = 0.5
    dev = [to_dev(cuda, A) for A in mats]
    pivs = [cuda.zeros(n, dtype=cuda.int32, device="cuda") for n in sizes]
    rhs = [rng.standard_normal((n, nrhs)) for n in sizes] if nrhs else None
    drhs = [to_dev(cuda, b) for b in rhs] if nrhs else None
    r, info = flame.batched("lu", dev, pivs=pivs, rhs=drhs)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    for i, A in enumerate(mats):
        LUo, po, ro = oracle.lu_piv(A)
        assert info[i] == ro, (i, sizes[i], info[i], ro)
        assert np.array_equal(pivs[i].cpu().numpy(), po), (i, sizes[i])
        assert rel_fro(to_host(dev[i]), LUo) < 1e-12, (i, sizes[i])
        if nrhs and ro == -1:
            Xo = oracle.lu_piv_solve(LUo, po, rhs[i])
            assert rel_fro(to_host(drhs[i]), Xo) < 1e-11, (i, sizes[i])


@pytest.mark.parametrize("kind", ["chol", "lu"])
def test_batched_fp32(cuda, flame, oracle, kind):
    rng = seeded(31 if kind == "chol" else 32)
    sizes = _sizes(rng, 18)
    mats = [spd(rng, n) if kind == "chol" else rng.uniform(-1, 1, (n, n)) + n ** 0.5 * np.eye(n) for n in sizes]
    dev = [to_dev(cuda, A, cuda.float32) for A in mats]
    pivs = [cuda.zeros(n, dtype=cuda.int32, device="cuda") for n in sizes] if kind == "lu" else None
    rhs = [rng.standard_normal((n, 4)) for n in sizes]
    drhs = [to_dev(cuda, b, cuda.float32) for b in rhs]
    r, info = flame.batched(kind, dev, pivs=pivs, rhs=drhs, f32=True)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    assert all(v == -1 for v in info)
    for i, A in enumerate(mats):
        X = np.linalg.solve(A, rhs[i])
        assert rel_fro(to_host(drhs[i]).astype(np.float64), X) < 1e-3, (i, sizes[i])


def test_batched_many_uneven(cuda, flame):
    """The benchmark's shape at a reduced count: 600 matrices, orders
    uniform in [8, 512], Cholesky + 4-RHS solve; residuals checked on the GPU."""
    torch = cuda
    rng = seeded(41)
    sizes = rng.integers(8, 513, size=600)
    g = torch.Generator(device="cuda").manual_seed(41)
    mats, rhs, orig = [], [], []
    for n in sizes:
        G = torch.randn((int(n), int(n)), dtype=torch.float64, device="cuda", generator=g)
        A = G @ G.t() / n + torch.eye(int(n), dtype=torch.float64, device="cuda")
        orig.append(A)
        mats.append(A.clone().t().contiguous().t())
        b = torch.randn((4, int(n)), dtype=torch.float64, device="cuda", generator=g).t()
        rhs.append(b)
    brhs = [b.clone() for b in rhs]
    r, info = flame.batched("chol", mats, rhs=rhs)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    assert all(v == -1 for v in info)
    worst = max(((A @ x - b).abs().max() / (A.abs().sum(1).max() * x.abs().max())).item()
                for A, x, b in zip(orig, rhs, brhs))
    assert worst < 1e-14, worst


def test_batched_tuner(cuda, flame):
    import ctypes as C
    times = (C.c_double * 20)()
    assert flame.lib().FLA_B200_batched_tune(0, 1, 8, times) == flame.FLA_SUCCESS, flame.last_error()
    nbs = [flame.lib().FLA_B200_batched_nb(0, 1, n) for n in (16, 48, 100, 200, 400)]
    assert all(v in (8, 16, 24, 32) for v in nbs)
    assert all(t > 0 for t in times)


def test_batched_sharded_single_rank(cuda, flame, oracle):
    """The sharded entry on a one-rank process group: the whole batch is this
    rank's share, factored in one launch, info gathered back in order."""
    import socket
    import torch.distributed as dist
    from libflame_b200.shard import batched_sharded
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1)
    try:
        rng = seeded(61)
        sizes = [3, 40, 129, 300]
        mats = [spd(rng, n) for n in sizes]
        mats[1] = mats[1].copy()
        mats[1][5, 5] = -1.0
        dev = [to_dev(cuda, A) for A in mats]
        r, info = batched_sharded("chol", dev)
        assert r == flame.FLA_SUCCESS, flame.last_error()
        for i, A in enumerate(mats):
            Lo, ro = oracle.chol(A)
            assert info[i] == ro
            if ro == -1:
                assert rel_fro(np.tril(to_host(dev[i])), np.tril(Lo)) < 1e-12
    finally:
        dist.destroy_process_group()


def test_chol_batched_fp64_to_order_1024_with_logdet(cuda, flame, oracle):
    """The FP64 batched Cholesky (DMMA updates) at orders up to 1024: factors,
    the solves of two right-hand sides and the log-determinants against the
    oracle; a matrix that is not SPD fails at the oracle's column, with NaN
    as its log-determinant, and does not disturb the others.  The strict
    upper triangles are left alone."""
    rng = seeded(1024)
    sizes = [1, 7, 31, 32, 33, 96, 255, 511, 512, 513, 700, 1000, 1023, 1024] + list(rng.integers(1, 1025, size=6))
    mats = [spd(rng, int(n)) for n in sizes]
    bad = 11
    mats[bad] = mats[bad].copy()
    mats[bad][600, 600] = -1.0
    dev = [to_dev(cuda, A) for A in mats]
    rhs = [rng.standard_normal((int(n), 2)) for n in sizes]
    drhs = [to_dev(cuda, b) for b in rhs]
    r, info, logdet = flame.chol_batched_logdet(dev, rhs=drhs)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    for i, A in enumerate(mats):
        Lo, ro = oracle.chol(A)
        assert info[i] == ro, (i, sizes[i], info[i], ro)
        got = to_host(dev[i])
        assert np.array_equal(np.triu(got, 1), np.triu(A, 1)), i
        if ro != -1:
            assert np.isnan(logdet[i])
            continue
        assert rel_fro(np.tril(got), np.tril(Lo)) < 1e-12, (i, sizes[i])
        ld_o = float(np.log(np.diag(Lo)).sum())
        assert abs(logdet[i] - ld_o) <= 1e-12 * max(1.0, abs(ld_o)), (i, logdet[i], ld_o)
        Xo = oracle.chol_solve(Lo, rhs[i])
        assert rel_fro(to_host(drhs[i]), Xo) < 1e-11, (i, sizes[i])


def _gp_matrix(rng, n):
    x = rng.uniform(0, 1, (n, 3))
    d2 = ((x[:, None, :] - x[None, :, :]) ** 2).sum(-1)
    return np.exp(-d2 / (2 * 0.3 ** 2)) + 1e-2 * np.eye(n), rng.standard_normal((n, 1))


def test_256_batched_gps_loss_and_gradient(cuda, flame, oracle):
    """256 Gaussian-process likelihoods with n uniform in [64, 1024]: forward
    (batched Cholesky, alpha = K^-1 y, log-determinant) and backward (the
    solve's adjoint formed from alpha and v = L^T alpha, then the batched
    log-determinant and Cholesky adjoints) give dloss/dK; checked against
    0.5 (K^-1 - alpha alpha^T) and the loss from the oracle's FLA_Chol and
    triangular solves on a sample of 12 GPs (the largest and smallest
    included), and for finiteness on all."""
    torch = cuda
    rng = seeded(256)
    sizes = [int(v) for v in rng.integers(64, 1025, size=256)]
    sizes[0], sizes[1] = 1024, 64
    data = [_gp_matrix(rng, n) for n in sizes]
    Ks = [to_dev(cuda, K) for K, _ in data]
    al = [to_dev(cuda, y) for _, y in data]
    r, info, logdet = flame.chol_batched_logdet(Ks, rhs=al)
    assert r == flame.FLA_SUCCESS, flame.last_error()
    assert all(v == -1 for v in info)
    # loss_i = 0.5 y^T alpha + sum log L_ii; backward of 0.5 v^T v, v = L^-1 y:
    # Lbar = -tril(alpha v^T) with v = L^T alpha; the log-determinant part is
    # added by the batched adjoint (logdet_scale = 1)
    Lbars = []
    for Ld, a in zip(Ks, al):
        L = torch.tril(Ld)
        v = L.t() @ a
        Lb = torch.empty_strided(tuple(Ld.shape), (1, Ld.shape[0]), dtype=torch.float64, device="cuda")
        Lb.copy_(-torch.tril(a @ v.t()))
        Lbars.append(Lb)
    assert flame.chol_adjoint_batched(Ks, Lbars, 1.0) == flame.FLA_SUCCESS, flame.last_error()
    losses = [0.5 * float((torch.from_numpy(y).cuda() * a).sum()) + ld for (K, y), a, ld in zip(data, al, logdet)]
    assert all(np.isfinite(losses))
    sample = [0, 1] + list(rng.choice(np.arange(2, 256), size=10, replace=False))
    for i in sample:
        K, y = data[i]
        Lo, ro = oracle.chol(K)
        assert ro == -1
        n = K.shape[0]
        Kinv = oracle.chol_solve(Lo, np.eye(n))
        alpha = oracle.chol_solve(Lo, y)
        loss_o = 0.5 * float(y[:, 0] @ alpha[:, 0]) + float(np.log(np.diag(Lo)).sum())
        assert abs(losses[i] - loss_o) <= 1e-10 * max(1.0, abs(loss_o)), (i, losses[i], loss_o)
        Ab = np.tril(to_host(Lbars[i]))
        G = 0.5 * (Ab + Ab.T)
        assert rel_fro(G, 0.5 * (Kinv - alpha @ alpha.T)) < 1e-9, (i, n)
