"""Generate the parity records at the benchmarked sizes by running the
reference libflame itself (oracle/_ref/libflame_ref.so: flat FLA_Chol,
FLA_LU_piv, FLA_QR_UT and FLA_Apply_Q_UT over the reference's built-in f2c
BLAS, single thread) on the seeded inputs of tests/golden/headline.py.

    python tests/golden/make_headline.py lu|chol|qr
    python tests/golden/make_headline.py spread

Each of the first three takes minutes of one CPU core (the reference's f2c
BLAS runs at a few GFLOP/s) and writes tests/golden/headline_<op>.npz.  See
headline.py for what the records hold and how the GPU test uses them.

"spread" adds to each record how far the same reference, built over
OpenBLAS instead of its f2c BLAS (oracle/_ref/libflame_ref_openblas.so,
all host threads), lands from it on the same input: the relative Frobenius
difference of the two factors (from the sketches) and the OpenBLAS build's
backward error.  Two correct FP64 builds of the reference differ by this
much only through the order of their floating-point operations.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, HERE)
import headline as H  # noqa: E402
import refbind as R  # noqa: E402


def _record(name, out):
    path = os.path.join(HERE, "headline_%s.npz" % name)
    np.savez_compressed(path, **out)
    print(path, os.path.getsize(path), "bytes")


def make_lu():
    import torch
    A = H.lu_input()
    t0 = time.time()
    LU, p, r = R.lu_piv(A)
    secs = time.time() - t0
    At, LUt = torch.from_numpy(A), torch.from_numpy(LU)
    be = H.lu_backward_error(torch, At, LUt, p, "cpu")
    sl, sr = H.sketches(torch, LUt, "cpu")
    _record("lu", dict(p=p.astype(np.int32), r=np.array(r), diag=np.diag(LU).copy(), row0=LU[0].copy(),
                       col0=LU[:, 0].copy(), sk_l=sl, sk_r=sr, be=np.array(be), secs=np.array(secs)))
    print("lu: r=%d be=%.4f %.0fs" % (r, be, secs))


def make_chol():
    import torch
    G = H.chol_factor_input()
    A = H.chol_input_torch(torch, G, "cpu").numpy()
    del G
    t0 = time.time()
    L, r = R.chol(A)
    secs = time.time() - t0
    At, Lt = torch.from_numpy(A), torch.tril(torch.from_numpy(L))
    be = H.chol_backward_error(torch, At, Lt)
    sl, sr = H.sketches(torch, Lt, "cpu")
    _record("chol", dict(r=np.array(r), diag=np.diag(L).copy(), col0=L[:, 0].copy(), row_last=L[-1].copy(),
                         sk_l=sl, sk_r=sr, be=np.array(be), secs=np.array(secs),
                         a_sum=np.array(float(At.sum()))))
    print("chol: r=%d be=%.4f %.0fs" % (r, be, secs))


def make_qr():
    import torch
    A, B = H.qr_input()
    t0 = time.time()
    QR, T, r = R.qr_ut(A)
    QtB, _ = R.apply_q_ut(QR, T, B)
    secs = time.time() - t0
    At, QRt, Tt = torch.from_numpy(A), torch.from_numpy(QR), torch.from_numpy(T)
    be = H.qr_backward_error(torch, At, QRt, Tt, "cpu")
    sl, sr = H.sketches(torch, QRt, "cpu")
    ql, qr_ = H.sketches(torch, torch.from_numpy(QtB), "cpu")
    b = T.shape[0]
    _record("qr", dict(r=np.array(r), diag=np.diag(QR).copy(), row0=QR[0].copy(), col0=QR[:, 0].copy(),
                       tau=np.array([T[j % b, j] for j in range(T.shape[1])]), t_first=T[:, :b].copy(),
                       t_last=T[:, -b:].copy(), sk_l=sl, sk_r=sr, qtb_sk_l=ql, qtb_sk_r=qr_,
                       qtb_top=QtB[:128].copy(), be=np.array(be), secs=np.array(secs)))
    print("qr: r=%d be=%.4f %.0fs" % (r, be, secs))


def _add(name, **kw):
    path = os.path.join(HERE, "headline_%s.npz" % name)
    rec = dict(np.load(path))
    rec.update({k: np.array(v) for k, v in kw.items()})
    np.savez_compressed(path, **rec)


def make_spread():
    import torch
    R.openblas_threads(os.cpu_count() or 1)
    rec = np.load(os.path.join(HERE, "headline_lu.npz"))
    A = H.lu_input()
    LU, p, r = R.lu_piv(A, kind="openblas")
    rel = H.sketch_rel_diff(H.sketches(torch, torch.from_numpy(LU), "cpu"), (rec["sk_l"], rec["sk_r"]))
    be = H.lu_backward_error(torch, torch.from_numpy(A), torch.from_numpy(LU), p, "cpu")
    _add("lu", spread=rel, spread_pivots_identical=bool(np.array_equal(p, rec["p"])), spread_be=be)
    print("lu spread %.3e (pivots identical %s), OpenBLAS build be %.4f" % (rel, np.array_equal(p, rec["p"]), be))
    del A, LU
    rec = np.load(os.path.join(HERE, "headline_chol.npz"))
    G = H.chol_factor_input()
    A = H.chol_input_torch(torch, G, "cpu").numpy()
    del G
    Lf, r = R.chol(A, kind="openblas")
    Lt = torch.tril(torch.from_numpy(Lf))
    rel = H.sketch_rel_diff(H.sketches(torch, Lt, "cpu"), (rec["sk_l"], rec["sk_r"]))
    be = H.chol_backward_error(torch, torch.from_numpy(A), Lt)
    _add("chol", spread=rel, spread_be=be)
    print("chol spread %.3e, OpenBLAS build be %.4f" % (rel, be))
    del A, Lf, Lt
    rec = np.load(os.path.join(HERE, "headline_qr.npz"))
    A, B = H.qr_input()
    QR, T, r = R.qr_ut(A, kind="openblas")
    rel = H.sketch_rel_diff(H.sketches(torch, torch.from_numpy(QR), "cpu"), (rec["sk_l"], rec["sk_r"]))
    be = H.qr_backward_error(torch, torch.from_numpy(A), torch.from_numpy(QR), torch.from_numpy(T), "cpu")
    _add("qr", spread=rel, spread_be=be)
    print("qr spread %.3e, OpenBLAS build be %.4f" % (rel, be))


if __name__ == "__main__":
    {"lu": make_lu, "chol": make_chol, "qr": make_qr, "spread": make_spread}[sys.argv[1]]()
