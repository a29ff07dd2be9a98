"""Parity at the benchmarked sizes: FLA_LU_piv n = 16384, FLA_Chol n = 16384,
FLA_QR_UT 16384 x 8192 with FLA_Apply_Q_UT on 64 right-hand sides, on the
GPU through the C-ABI, against records the reference libflame produced on
the same seeded inputs (tests/golden/headline_*.npz, made by
tests/golden/make_headline.py; inputs and checks in tests/golden/headline.py).

Bar: return codes equal; LU pivot vector identical; factors within
max(1e-12, SPREAD_FACTOR x spread) normwise (relative Frobenius difference
estimated from two-sided Gaussian sketches of the factor, and exact on the
stored diagonal, first row and first column), where `spread` is how far the
reference itself, built over OpenBLAS instead of its f2c BLAS, lands from
the record on the same input (make_headline.py spread: 1.5e-12 for the LU,
whose U(-1,1) input has kappa ~ 1e5; a few 1e-15 for the Cholesky and QR) --
no FP64 factorization that orders its operations differently from the f2c
loops can be expected closer than that; backward error at most the
reference's own, with BE_SLACK for evaluating the two residuals in FP64
with different BLAS (the CPU record and the GPU check each sum n-term
products, whose rounding is of the order of the quantity measured; two FP64
evaluations of one residual differ by up to a few percent at these sizes).
"""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT, to_dev

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import headline as H  # noqa: E402

pytestmark = pytest.mark.gpu

FACTOR_TOL = 1e-12
SPREAD_FACTOR = 1.5
BE_SLACK = 0.05


def _record(name):
    return np.load(os.path.join(ROOT, "tests", "golden", "headline_%s.npz" % name))


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _tol(rec):
    return max(FACTOR_TOL, SPREAD_FACTOR * float(rec["spread"]))


def test_lu_n16384_pivots_identical_to_reference(cuda, flame):
    torch = cuda
    rec = _record("lu")
    A = H.lu_input()
    Ad = to_dev(torch, A)
    A0 = Ad.clone()
    del A
    p = torch.zeros(H.LU_N, dtype=torch.int32, device="cuda")
    r = flame.lu_piv(Ad, p)
    assert r == int(rec["r"]), flame.last_error()
    pv = p.cpu().numpy()
    bad = np.nonzero(pv != rec["p"])[0]
    assert bad.size == 0, "pivots differ from the reference at %d columns, first %s" % (bad.size, bad[:8])
    rel = H.sketch_rel_diff(H.sketches(torch, Ad, "cuda"), (rec["sk_l"], rec["sk_r"]))
    drel = _rel(torch.diagonal(Ad).cpu().numpy(), rec["diag"])
    be = H.lu_backward_error(torch, A0, Ad, pv, "cuda")
    print("LU n=16384: pivots identical; factor rel diff %.2e (reference over OpenBLAS: %.2e), diag %.2e, "
          "backward error %.4f (reference %.4f, over OpenBLAS %.4f)"
          % (rel, float(rec["spread"]), drel, be, float(rec["be"]), float(rec["spread_be"])))
    assert rel < _tol(rec), rel
    assert drel < _tol(rec)
    assert _rel(Ad[0].cpu().numpy(), rec["row0"]) < _tol(rec)
    assert _rel(Ad[:, 0].cpu().numpy(), rec["col0"]) < _tol(rec)
    assert be <= float(rec["be"]) * (1 + BE_SLACK), (be, float(rec["be"]))


def test_chol_n16384_matches_reference(cuda, flame):
    torch = cuda
    rec = _record("chol")
    G = H.chol_factor_input()
    A = H.chol_input_torch(torch, G, "cuda")
    del G
    assert float(A.sum()) == float(rec["a_sum"])  # the same input, bit for bit
    Ad = A.t()  # column-major view of the symmetric matrix
    A0 = A.clone()
    r = flame.chol(Ad)
    assert r == int(rec["r"]), flame.last_error()
    Lt = torch.tril(Ad)
    rel = H.sketch_rel_diff(H.sketches(torch, Lt, "cuda"), (rec["sk_l"], rec["sk_r"]))
    be = H.chol_backward_error(torch, A0, Lt)
    print("Chol n=16384: factor rel diff %.2e (reference over OpenBLAS: %.2e), backward error %.4f "
          "(reference %.4f, over OpenBLAS %.4f)" % (rel, float(rec["spread"]), be, float(rec["be"]),
                                                   float(rec["spread_be"])))
    assert rel < _tol(rec), rel
    assert _rel(torch.diagonal(Lt).cpu().numpy(), rec["diag"]) < _tol(rec)
    assert _rel(Lt[:, 0].cpu().numpy(), rec["col0"]) < _tol(rec)
    assert _rel(Lt[-1].cpu().numpy(), rec["row_last"]) < _tol(rec)
    assert be <= float(rec["be"]) * (1 + BE_SLACK), (be, float(rec["be"]))


def test_qr_16384x8192_and_apply_q_match_reference(cuda, flame):
    torch = cuda
    rec = _record("qr")
    A, B = H.qr_input()
    Ad, Bd = to_dev(torch, A), to_dev(torch, B)
    A0 = Ad.clone()
    del A, B
    b = 32
    T = torch.zeros((H.QR_N, b), dtype=torch.float64, device="cuda").t()
    r = flame.qr_ut(Ad, T)
    assert r == int(rec["r"]), flame.last_error()
    assert flame.apply_q_ut(Ad, T, Bd) == flame.FLA_SUCCESS, flame.last_error()
    rel = H.sketch_rel_diff(H.sketches(torch, Ad, "cuda"), (rec["sk_l"], rec["sk_r"]))
    relq = H.sketch_rel_diff(H.sketches(torch, Bd, "cuda"), (rec["qtb_sk_l"], rec["qtb_sk_r"]))
    be = H.qr_backward_error(torch, A0, Ad, T, "cuda")
    print("QR 16384x8192: factor rel diff %.2e (reference over OpenBLAS: %.2e), Q^T B rel diff %.2e, "
          "backward error %.4f (reference %.4f, over OpenBLAS %.4f)"
          % (rel, float(rec["spread"]), relq, be, float(rec["be"]), float(rec["spread_be"])))
    assert rel < _tol(rec), rel
    assert _rel(torch.diagonal(Ad).cpu().numpy(), rec["diag"]) < _tol(rec)
    assert _rel(Ad[0].cpu().numpy(), rec["row0"]) < _tol(rec)
    assert _rel(Ad[:, 0].cpu().numpy(), rec["col0"]) < _tol(rec)
    Th = T.cpu().numpy()
    tau = np.array([Th[j % b, j] for j in range(H.QR_N)])
    assert _rel(tau, rec["tau"]) < _tol(rec)
    assert _rel(np.triu(Th[:, :b]), np.triu(rec["t_first"])) < _tol(rec)
    assert _rel(np.triu(Th[:, -b:]), np.triu(rec["t_last"])) < _tol(rec)
    assert relq < _tol(rec), relq
    assert _rel(Bd[:128].cpu().numpy(), rec["qtb_top"]) < _tol(rec)
    assert be <= float(rec["be"]) * (1 + BE_SLACK), (be, float(rec["be"]))
