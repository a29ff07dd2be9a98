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
