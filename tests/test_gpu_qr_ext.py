"""The steps after FLA_QR_UT on the GPU through the C-ABI: FLA_QR_UT_solve,
FLA_QR_UT_form_Q (separate and in place), FLA_Accum_T_UT and the LAPACK
dormqr_ (all four side/trans forms) and dorgqr_.

Checked against outputs of the reference libflame on the same inputs
(tests/golden/reference_small.npz, keys qrx_*) and against the CPU oracle's
QR_UT / Apply_Q_UT composed the way the reference composes them
(FLA_QR_UT_solve.c:26-41: Q^T B, then the triangular solve with R).
Tolerance: relative Frobenius 1e-12 (the GPU's GEMM order differs from
the reference's netlib loops, so results agree to rounding, not bitwise)."""
import numpy as np
import pytest

from conftest import rel_fro, seeded, to_dev, to_host

pytestmark = pytest.mark.gpu

TOL = 1e-12
KEYS = ["qrx_90x40", "qrx_170x130"]


def _qr_dev(cuda, flame, A):
    torch = cuda
    m, n = A.shape
    Ad = to_dev(torch, A)
    b = min(32, m, n)
    T = torch.zeros((n, b), dtype=torch.float64, device="cuda").t()
    assert flame.qr_ut(Ad, T) == flame.FLA_SUCCESS, flame.last_error()
    return Ad, T


@pytest.mark.parametrize("key", KEYS)
def test_qr_ut_solve_matches_reference(cuda, flame, golden, key):
    torch = cuda
    A, B = golden[key + "_A"], golden[key + "_B"]
    Ad, T = _qr_dev(cuda, flame, A)
    Bd = to_dev(torch, B)
    B0 = Bd.clone()
    X = torch.zeros((A.shape[1], B.shape[1]), dtype=torch.float64, device="cuda").t().contiguous().t()
    assert flame.qr_ut_solve(Ad, T, Bd, X) == flame.FLA_SUCCESS, flame.last_error()
    assert rel_fro(to_host(X), golden[key + "_X"]) < TOL
    assert torch.equal(Bd, B0)  # B is not modified


@pytest.mark.parametrize("m,n,nrhs", [(300, 300, 2), (1000, 257, 5), (4000, 640, 3)])
def test_qr_ut_solve_matches_oracle(cuda, flame, oracle, m, n, nrhs):
    torch = cuda
    rng = seeded(m + n)
    A, B = rng.standard_normal((m, n)), rng.standard_normal((m, nrhs))
    Ad, T = _qr_dev(cuda, flame, A)
    X = torch.zeros((n, nrhs), dtype=torch.float64, device="cuda").t().contiguous().t()
    assert flame.qr_ut_solve(Ad, T, to_dev(torch, B), X) == flame.FLA_SUCCESS
    QRo, To = oracle.qr_ut(A)
    Y = oracle.apply_qt(QRo, To, B)[:n]
    Xo = oracle.trsm_llt(np.ascontiguousarray(np.triu(QRo[:n]).T), Y)  # R x = y with R^T lower
    assert rel_fro(to_host(X), Xo) < TOL


@pytest.mark.parametrize("key", KEYS)
def test_form_q_matches_reference_separate_and_in_place(cuda, flame, golden, key):
    torch = cuda
    A = golden[key + "_A"]
    m, n = A.shape
    Ad, T = _qr_dev(cuda, flame, A)
    Q = torch.zeros((n, m), dtype=torch.float64, device="cuda").t()
    assert flame.qr_ut_form_q(Ad, T, Q) == flame.FLA_SUCCESS, flame.last_error()
    assert rel_fro(to_host(Q), golden[key + "_Q"]) < TOL
    # in place: Q overwrites the factor itself
    assert flame.qr_ut_form_q(Ad, T, Ad) == flame.FLA_SUCCESS, flame.last_error()
    assert rel_fro(to_host(Ad), golden[key + "_Q"]) < TOL


def test_form_q_square_orthogonal_against_oracle(cuda, flame, oracle):
    torch = cuda
    A = seeded(77).standard_normal((700, 400))
    Ad, T = _qr_dev(cuda, flame, A)
    Q = torch.zeros((700, 700), dtype=torch.float64, device="cuda").t()
    assert flame.qr_ut_form_q(Ad, T, Q) == flame.FLA_SUCCESS
    QRo, To = oracle.qr_ut(A)
    Qo = oracle.form_q(QRo, To)
    assert rel_fro(to_host(Q), Qo) < TOL


@pytest.mark.parametrize("key", KEYS)
def test_dormqr_all_forms_and_dorgqr_match_reference(cuda, flame, golden, key):
    torch = cuda
    A = golden[key + "_A"]
    m, n = A.shape
    a = to_dev(torch, A)
    tau = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert flame.dgeqrf(a, tau) == 0, flame.last_error()
    for side, trans in [("L", "T"), ("L", "N"), ("R", "N"), ("R", "T")]:
        C0 = golden[key + ("_CL" if side == "L" else "_CR")]
        c = to_dev(torch, C0)
        assert flame.dormqr(side, trans, a, tau, c) == 0, flame.last_error()
        assert rel_fro(to_host(c), golden[key + "_ormqr_%s%s" % (side, trans)]) < TOL, (side, trans)
    # host buffers take the staged path
    ah, th = to_host(a), tau.cpu().numpy()
    ch = np.asfortranarray(golden[key + "_CL"])
    assert flame.dormqr("L", "T", ah, th, ch) == 0
    assert rel_fro(ch, golden[key + "_ormqr_LT"]) < TOL
    assert flame.dorgqr(a, tau) == 0, flame.last_error()
    assert rel_fro(to_host(a), golden[key + "_orgqr"]) < TOL


@pytest.mark.parametrize("key", KEYS)
def test_accum_t_ut_matches_reference(cuda, flame, golden, key):
    torch = cuda
    A = golden[key + "_A"]
    m, n = A.shape
    a = to_dev(torch, A)
    tau = torch.zeros(n, dtype=torch.float64, device="cuda")
    assert flame.dgeqrf(a, tau) == 0
    b = min(32, n)
    T = torch.zeros((n, b), dtype=torch.float64, device="cuda").t()
    t = (1.0 / tau).contiguous()
    assert flame.accum_t_ut(a, t, T) == flame.FLA_SUCCESS, flame.last_error()
    Tg = golden[key + "_accumT"]
    assert rel_fro(np.triu(to_host(T)), np.triu(Tg)) < TOL
