"""Inputs and checks of the parity cases at the benchmarked sizes.

Three seeded inputs, each regenerated bit for bit wherever it is needed:

  * FLA_LU_piv, n = 16384, A i.i.d. U(-1, 1);
  * FLA_Chol (lower), n = 16384, A = G G^T / n + I with G i.i.d. N(0, 1)
    rounded to multiples of 1/256 and clipped to [-4, 4]: every product and
    partial sum of G G^T is then an exact FP64 number, so the input is the
    same whichever BLAS or GPU forms it and in whatever order;
  * FLA_QR_UT on m = 16384 x n = 8192 i.i.d. N(0, 1), with FLA_Apply_Q_UT
    (Q^T) on 64 N(0, 1) right-hand sides.

tests/golden/make_headline.py runs the reference libflame (flat FLA_* over
its built-in f2c BLAS, oracle/_ref/libflame_ref.so) once on each and stores
a compact record in tests/golden/headline.npz: the full pivot vector and
return code, the factor's diagonal, its first row and column, two-sided
Gaussian sketches of the factor (Omega_l^T F and F Omega_r, two vectors per
side), and the reference's own backward error.  The GPU test
(tests/test_gpu_headline.py) compares the GPU factors with that record:
pivots identical, the relative Frobenius difference (estimated by the
sketches, exact on the stored row, column and diagonal) within 1e-12, and
backward error at most the reference's.

The heavy linear algebra of the checks is written once in torch so it runs
on the CPU here and on the GPU in the test.
"""
import numpy as np

LU_N = 16384
CHOL_N = 16384
QR_M, QR_N, QR_NRHS = 16384, 8192, 64
SEED_LU, SEED_CHOL, SEED_QR = 1638401, 1638402, 1638403
SEED_SKETCH = 777
SKETCH_K = 2
EPS = np.finfo(np.float64).eps


def lu_input(n=LU_N):
    return np.random.default_rng(SEED_LU).uniform(-1.0, 1.0, (n, n))


def chol_factor_input(n=CHOL_N):
    """G (exactly representable entries): A = G G^T / n + I."""
    g = np.random.default_rng(SEED_CHOL).standard_normal((n, n))
    return np.clip(np.round(g * 256.0), -1024.0, 1024.0) / 256.0


def chol_input_torch(torch, G, device):
    """A = G G^T / n + I formed with torch on `device` (exact in FP64)."""
    n = G.shape[0]
    g = torch.from_numpy(G).to(device)
    A = g @ g.T
    A /= n
    A.diagonal().add_(1.0)
    return A


def qr_input(m=QR_M, n=QR_N, nrhs=QR_NRHS):
    rng = np.random.default_rng(SEED_QR)
    A = rng.standard_normal((m, n))
    B = rng.standard_normal((m, nrhs))
    return A, B


def sketch_vectors(m, n):
    rng = np.random.default_rng(SEED_SKETCH + 31 * m + n)
    return rng.standard_normal((m, SKETCH_K)), rng.standard_normal((n, SKETCH_K))


def sketches(torch, F, device):
    """(Omega_l^T F, F Omega_r) of the m x n factor F (a torch tensor)."""
    m, n = F.shape
    wl, wr = sketch_vectors(m, n)
    wl = torch.from_numpy(wl).to(device)
    wr = torch.from_numpy(wr).to(device)
    return (wl.T @ F).cpu().numpy(), (F @ wr).cpu().numpy()


def sketch_rel_diff(s, s_ref):
    """Relative Frobenius difference of two factors estimated from their
    sketches (E ||Omega^T D||_F^2 = k ||D||_F^2 on both sides)."""
    num = np.linalg.norm(s[0] - s_ref[0]) ** 2 + np.linalg.norm(s[1] - s_ref[1]) ** 2
    den = np.linalg.norm(s_ref[0]) ** 2 + np.linalg.norm(s_ref[1]) ** 2
    return float(np.sqrt(num / den))


def perm_from_pivots(p, m):
    """Row permutation of relative zero-based pivots: (P A) = A[perm]."""
    perm = np.arange(m)
    for i in range(len(p)):
        j = i + int(p[i])
        perm[i], perm[j] = perm[j], perm[i]
    return perm


def lu_backward_error(torch, A, LU, p, device):
    """||P A - L U||_F / (n eps ||A||_F) for a square LU (torch tensors)."""
    n = A.shape[0]
    idx = torch.from_numpy(perm_from_pivots(p, n)).to(device)
    L = torch.tril(LU, -1)
    L.diagonal().fill_(1.0)
    R = A.index_select(0, idx)
    R -= L @ torch.triu(LU)
    del L
    return float(torch.linalg.norm(R) / (n * EPS * torch.linalg.norm(A)))


def chol_backward_error(torch, A, Lf):
    n = A.shape[0]
    L = torch.tril(Lf)
    R = A - L @ L.T
    return float(torch.linalg.norm(R) / (n * EPS * torch.linalg.norm(A)))


def apply_q(torch, QR, T, X):
    """X := Q X for the UT-transform Q of FLA_QR_UT (blocks of b columns:
    Q = Q_0 Q_1 ..., Q_j = I - U_j inv(T_j) U_j^T), applied last block first."""
    m, n = QR.shape
    b = T.shape[0]
    k = min(m, n)
    for c0 in reversed(range(0, k, b)):
        w = min(b, k - c0)
        U = torch.tril(QR[c0:, c0:c0 + w], -1)
        U[:w].diagonal().fill_(1.0)
        Tb = torch.triu(T[:w, c0:c0 + w])
        W = U.T @ X[c0:]
        W = torch.linalg.solve_triangular(Tb, W, upper=True)
        X[c0:] -= U @ W
    return X


def qr_backward_error(torch, A, QR, T, device):
    """||A - Q R||_F / (m eps ||A||_F)."""
    m, n = A.shape
    X = torch.zeros((m, n), dtype=A.dtype, device=device)
    X[:n] = torch.triu(QR[:n])
    apply_q(torch, QR, T, X)
    X -= A
    return float(torch.linalg.norm(X) / (max(m, n) * EPS * torch.linalg.norm(A)))
