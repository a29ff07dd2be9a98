#!/usr/bin/env python3
"""Benchmark: FP64 FLA_LU_piv at n=16384 (and FLA_Chol) on one B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one factorization of a fresh matrix):
  FLA_LU_piv, n = 16384, A i.i.d. U(-1,1) (seeded), column-major FP64 in HBM
  (2 GiB, larger than L2; restoring A between steps also flushes L2).
Metric: TFLOP/s = (2/3 n^3) / device time of the factorization, whole job.

Rank 0 prints ONE JSON line.  `value` is the device-timed throughput with A
resident in HBM (time = CUDA events the library records on its own stream
around the factorization, max over ranks); `e2e` is the same metric through
the LAPACK entry point dgetrf_ on pinned host buffers, host<->device copies
inside the timed region.  `roofline` describes the dominant kernel (the FP64
DMMA GEMM engine) against the FP64 peak measured in this run with cuBLAS
DGEMM (MEASURED_PEAKS.json carries no FP64 figure).  `cpu_baseline` times
the reference libflame's own multithreaded CPU path (SuperMatrix
FLASH_LU_piv over its built-in BLAS, all host cores) on a bounded sample.

Multi-GPU: a single factorization does not shard ("replicas only"): each
rank factors its own matrix, `value` = all ranks' flops / max time.

--impl reference: times the reference libflame on the host cores (rank 0
only; other ranks exit 0) on a bounded sample of the same workload.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "FP64 Chol/LU TFLOP/s & %peak; mixed-IR solve speedup vs FP64 at equal error"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=16384)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-ir", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-count", type=int, default=10000)
    ap.add_argument("--ir-n", type=int, default=16384)
    ap.add_argument("--profile-op", default=None,
                    choices=["lu", "chol", "qr", "apply_q", "mixed_spd", "mixed_general", "batched_chol"],
                    help="run one operation twice at order --n (for ncu captures) and exit")
    return ap.parse_args()


def profile_op(args):
    """One operation at order n, twice (the second call is the one a capture
    would look at), for ncu: lu / chol (FLA_LU_piv / FLA_Chol on n x n),
    qr / apply_q (FLA_QR_UT on 2n x n, then FLA_Apply_Q_UT on 64 columns),
    mixed_spd / mixed_general (the default mixed solvers, 32 right-hand
    sides, kappa 1e2), batched_chol (n matrices of orders U{8..512}).
    Prints one JSON line with the device times of the calls."""
    import torch
    import libflame_b200 as F
    F.init()
    dev = "cuda"
    n = args.n
    g = torch.Generator(device=dev).manual_seed(11)
    out = {"profile_op": args.profile_op, "n": n, "ms": []}

    def colmajor(t):
        return t.t().contiguous().t()
    for rep in range(2):
        if args.profile_op == "lu":
            A = colmajor(torch.rand((n, n), dtype=torch.float64, device=dev, generator=g) * 2 - 1)
            p = torch.zeros(n, dtype=torch.int32, device=dev)
            r = F.lu_piv(A, p)
        elif args.profile_op == "chol":
            G = torch.randn((n, n), dtype=torch.float64, device=dev, generator=g)
            A = colmajor(G @ G.t() / n + torch.eye(n, dtype=torch.float64, device=dev))
            r = F.chol(A)
        elif args.profile_op in ("qr", "apply_q"):
            A = colmajor(torch.randn((2 * n, n), dtype=torch.float64, device=dev, generator=g))
            T = torch.zeros((n, 32), dtype=torch.float64, device=dev).t()
            r = F.qr_ut(A, T)
            if args.profile_op == "apply_q" and r == F.FLA_SUCCESS:
                B = colmajor(torch.randn((2 * n, 64), dtype=torch.float64, device=dev, generator=g))
                r = F.apply_q_ut(A, T, B)
        elif args.profile_op in ("mixed_spd", "mixed_general"):
            Q = torch.linalg.qr(torch.randn((n, n), dtype=torch.float64, device=dev, generator=g))[0]
            s = torch.logspace(0, -2, n, dtype=torch.float64, device=dev)
            A = (Q * s) @ Q.t()
            if args.profile_op == "mixed_general":
                V = torch.linalg.qr(torch.randn((n, n), dtype=torch.float64, device=dev, generator=g))[0]
                A = (Q * s) @ V.t()
            else:
                A = (A + A.t()) / 2
            A = colmajor(A)
            B = colmajor(torch.randn((n, 32), dtype=torch.float64, device=dev, generator=g))
            X = colmajor(torch.empty((n, 32), dtype=torch.float64, device=dev))
            if args.profile_op == "mixed_spd":
                r = F.chol_solve_mixed(A, B, X, F.FLA_LOWER_TRIANGULAR)[0]
            else:
                r = F.lu_piv_solve_mixed(A, B, X)[0]
        else:
            rng = np.random.default_rng(5)
            mats = []
            for m in rng.integers(8, 513, size=n):
                m = int(m)
                G = torch.randn((m, m), dtype=torch.float64, device=dev, generator=g)
                mats.append(colmajor(G @ G.t() / m + torch.eye(m, dtype=torch.float64, device=dev)))
            r = F.batched("chol", mats)[0]
        torch.cuda.synchronize()
        if r != F.FLA_SUCCESS:
            raise RuntimeError("%s failed: %s" % (args.profile_op, F.last_error()))
        out["ms"].append(F.last_op_ms())
    print(json.dumps(out))


# ---------------------------------------------------------------------------
# Clock sampling during the timed region.
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Reference CPU path.
# ---------------------------------------------------------------------------
def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def headline():
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import headline as H
    return H


def lu_input(n):
    """The LU workload's input: the seeded U(-1,1) matrix of the parity
    record at n = 16384, a seeded U(-1,1) matrix of its own at other n."""
    if n == headline().LU_N:
        return headline().lu_input()
    return np.random.default_rng(2026 + n).uniform(-1.0, 1.0, (n, n))


def lu_config(n, world):
    return {"workload": "FLA_LU_piv n=%d FP64, A iid U(-1,1) seeded, column-major" % n, "n": n,
            "parallelism": "replicas" if world > 1 else "single",
            "l2": "inputs (2 GiB at n=16384) larger than L2; the per-step restore of A also flushes L2"}


def reference_lu_openblas(n, nthreads):
    """The reference libflame's flat FLA_LU_piv over OpenBLAS
    (oracle/_ref/libflame_ref_openblas.so) on `nthreads` host threads, one
    factorization of lu_input(n); returns (TFLOP/s, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refbind as R
    R.openblas_threads(nthreads)
    secs, r = R.timed_call("lu", lu_input(n), "openblas")
    if r != -1:
        raise RuntimeError("reference FLA_LU_piv returned %d" % r)
    return (2.0 / 3.0) * n ** 3 / secs / 1e12, secs


def reference_lu_flash(n_cpu, nthreads):
    """FLASH_LU_piv (SuperMatrix over the reference's built-in f2c BLAS) on
    `nthreads` host threads; returns (TFLOP/s, seconds)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refbind as R
    A = np.random.default_rng(2026).uniform(-1, 1, (n_cpu, n_cpu))
    _, _, r, dt = R.lu_piv_flash(A, nthreads, 256)
    return (2.0 / 3.0) * n_cpu ** 3 / dt / 1e12, dt


def pick_reference_n(n_full, nthreads, runs, budget_s):
    """Largest order (n_full if it fits) whose `runs` reference
    factorizations fit in budget_s seconds, from one probe at n_full / 2."""
    half = n_full // 2
    _, s_half = reference_lu_openblas(half, nthreads)
    t_full = 8.0 * s_half * 0.9
    if runs * t_full <= budget_s:
        return n_full, t_full
    n = int(half * (budget_s / (runs * s_half)) ** (1.0 / 3.0)) // 512 * 512
    return max(2048, min(n, n_full)), None


def run_reference(args, rank):
    if rank != 0:
        return
    nthreads = host_threads()
    n, _ = pick_reference_n(args.n, nthreads, args.warmup + args.steps, 200.0)
    vals, tot = [], 0.0
    for _ in range(args.warmup):
        reference_lu_openblas(n, nthreads)
    for _ in range(args.steps):
        tf, secs = reference_lu_openblas(n, nthreads)
        vals.append(tf)
        tot += secs
    v = statistics.median(vals)
    desc = ("reference libflame flat FLA_LU_piv over OpenBLAS 0.3.30 (SciPy's bundled LP64 build), "
            "%d host threads, n=%d%s" % (nthreads, n, "" if n == args.n else " (bounded sample of n=%d)" % args.n))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": "TFLOP/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * tot / max(1, args.steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": lu_config(n, args.gpus),
        "cpu_baseline": {"value": v, "unit": "TFLOP/s", "cores": nthreads, "kind": "reference",
                         "sample": desc},
        "e2e": {"value": v, "unit": "TFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Our path.
# ---------------------------------------------------------------------------
def measure_fp64_peak(torch, dev):
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def mixed_ir_section(torch, dev, F, n, nrhs, cpu=False):
    """Time-to-solution of the mixed-precision solvers (16-bit/3xTF32
    tensor-core factorization + FP64 refinement) against the FP64 form
    (FLA_LU_piv + FLA_LU_piv_solve, FLA_Chol + FLA_Chol_solve) on
    A = Q diag(s) Q^T (SPD) and U diag(s) V^T (general), s log-spaced so that
    kappa = 1e2, 1e5, 1e8; nrhs N(0,1) right-hand sides.  Both times are
    device times of the library's own calls (CUDA events on its stream);
    errors are normwise backward errors max_c |b - A x|_inf /
    (|A|_inf |x|_inf + |b|_inf) and the forward difference to the FP64 form."""
    g = torch.Generator(device=dev).manual_seed(4242)
    Q = torch.linalg.qr(torch.randn((n, n), dtype=torch.float64, device=dev, generator=g))[0]
    V = torch.linalg.qr(torch.randn((n, n), dtype=torch.float64, device=dev, generator=g))[0]
    B = torch.randn((nrhs, n), dtype=torch.float64, device=dev, generator=g).t()  # column-major n x nrhs
    X64 = torch.empty((nrhs, n), dtype=torch.float64, device=dev).t()
    Xmx = torch.empty((nrhs, n), dtype=torch.float64, device=dev).t()
    work = torch.empty((n, n), dtype=torch.float64, device=dev).t()
    piv = torch.empty(n, dtype=torch.int32, device=dev)
    vW, vp, vB, v64, vmx = F.View(work), F.View(piv), F.View(B), F.View(X64), F.View(Xmx)
    L = F.lib()

    def berr(A, X):
        R = B - A @ X
        an = A.abs().sum(dim=1).max()
        return (R.abs().amax(dim=0) / (an * X.abs().amax(dim=0) + B.abs().amax(dim=0))).max().item()

    out = {}
    for kind in ("spd", "general"):
        for kappa in (1e2, 1e5, 1e8):
            s = torch.logspace(0, -float(np.log10(kappa)), n, dtype=torch.float64, device=dev)
            A = (Q * s) @ (Q.t() if kind == "spd" else V.t())
            if kind == "spd":
                A = (A + A.t()) / 2
            A = A.t().contiguous().t()  # column-major
            vA = F.View(A)
            t64 = []
            tmx = []
            rec = {}
            for rep in range(2):
                work.copy_(A)
                torch.cuda.synchronize()
                if kind == "spd":
                    r1 = L.FLA_Chol(F.FLA_LOWER_TRIANGULAR, vW.obj)
                    m1 = F.last_op_ms()
                    r2 = L.FLA_Chol_solve(F.FLA_LOWER_TRIANGULAR, vW.obj, vB.obj, v64.obj)
                else:
                    r1 = L.FLA_LU_piv(vW.obj, vp.obj)
                    m1 = F.last_op_ms()
                    r2 = L.FLA_LU_piv_solve(vW.obj, vp.obj, vB.obj, v64.obj)
                m2 = F.last_op_ms()
                if r1 != F.FLA_SUCCESS or r2 != F.FLA_SUCCESS:
                    raise RuntimeError("FP64 form failed (%s, kappa %.0e, rep %d): %d %d %s"
                                       % (kind, kappa, rep, r1, r2, F.last_error()))
                t64.append(m1 + m2)
                if kind == "spd":
                    r, it, inner = F.chol_solve_mixed(A, B, Xmx, F.FLA_LOWER_TRIANGULAR)
                else:
                    r, it, inner = F.lu_piv_solve_mixed(A, B, Xmx)
                if r != F.FLA_SUCCESS:
                    raise RuntimeError("mixed solver failed (%s, kappa %.0e, rep %d): %d %s"
                                       % (kind, kappa, rep, r, F.last_error()))
                tmx.append(F.last_op_ms())
                rec = {"iter": it, "path": "FP16 hi/lo split factors + refinement" if it >= 0 else "FP64 fallback"}
            f64, fmx = min(t64), min(tmx)
            rec.update({"fp64_ms": f64, "mixed_ms": fmx, "speedup": f64 / fmx,
                        "backward_error_fp64": berr(A, X64), "backward_error_mixed": berr(A, Xmx),
                        "forward_diff_vs_fp64": ((Xmx - X64).norm() / X64.norm()).item()})
            # GMRES-IR on the FP16 factors (the form for ill-conditioned A)
            if kind == "spd":
                r, it, inner = F.chol_solve_mixed(A, B, Xmx, F.FLA_LOWER_TRIANGULAR, 1, 1)
            else:
                r, it, inner = F.lu_piv_solve_mixed(A, B, Xmx, 1, 1)
            if r != F.FLA_SUCCESS:
                raise RuntimeError("GMRES-IR failed: %d %s" % (r, F.last_error()))
            rec["gmres_ir"] = {"ms": F.last_op_ms(), "speedup": f64 / F.last_op_ms(), "iter": it,
                               "gmres_iters": inner, "backward_error": berr(A, Xmx)}
            if cpu and kappa == 1e2:
                rec["reference_cpu"] = reference_ir_cpu(kind, A.cpu().numpy(), B.cpu().numpy())
            out["%s_kappa_%.0e" % (kind, kappa)] = rec
            del A, vA
    del Q, V, work
    torch.cuda.empty_cache()
    return {"workload": "n=%d, nrhs=%d, A = Q diag(s) Q^T / U diag(s) V^T, s log-spaced to kappa" % (n, nrhs),
            "solver": "default (adaptive): FP16 hi/lo split (FP32-accurate) tcgen05 factors + classic FP64 "
                      "refinement while each step cuts the backward error >= 4x, else the FP64 factorization; "
                      "gmres_ir: GMRES-IR on plain FP16 factors (then the split, 3xTF32 and FP64 when it stalls)",
            "cases": out}


def reference_ir_cpu(kind, A, B):
    """The reference's own mixed-precision drivers (dsposv_ / dsgesv_: FP32
    factorization, FP64 refinement) beside its FP64 solvers (dposv_ /
    dgesv_), all from the reference built over OpenBLAS, on the host cores."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refbind as R
    nthreads = host_threads()
    R.openblas_threads(nthreads)
    if kind == "spd":
        _, _, info = R.dposv(A, B, "L", kind="openblas")
        t64 = R.last_secs
        _, it, info2 = R.dsposv(A, B, "L", kind="openblas")
    else:
        _, _, _, info = R.dgesv(A, B, kind="openblas")
        t64 = R.last_secs
        _, it, info2 = R.dsgesv(A, B, kind="openblas")
    tmx = R.last_secs
    return {"driver": "dsposv_" if kind == "spd" else "dsgesv_", "fp64_s": t64, "mixed_s": tmx,
            "speedup": t64 / tmx, "iter": it, "info": [info, info2], "threads": nthreads,
            "build": "reference libflame over OpenBLAS 0.3.30"}


def batched_section(torch, dev, F, count):
    """count matrices, orders uniform in [8, 512] (seeded): SPD A = G G^T/n + I
    through FLA_Chol_batched + 4-RHS solve (FP64 and FP32), and U(-1,1)
    matrices through FLA_LU_piv_batched + 4-RHS solve (FP64), each a single
    persistent launch.  Inputs are restored from a pristine copy (one copy of
    the flat buffer) before every timed call; time = the library's device
    time of the call.  flops: n^3/3 + 4 n^2 * 2 (Cholesky), 2n^3/3 + 4 n^2 * 2
    (LU) per matrix."""
    import ctypes as C
    rng = np.random.default_rng(2027)
    sizes = rng.integers(8, 513, size=count).astype(np.int32)
    nrhs = 4
    offs = np.zeros(count + 1, dtype=np.int64)
    offs[1:] = np.cumsum(sizes.astype(np.int64) ** 2)
    boffs = np.zeros(count + 1, dtype=np.int64)
    boffs[1:] = np.cumsum(sizes.astype(np.int64) * nrhs)
    g = torch.Generator(device=dev).manual_seed(2027)
    L = F.lib()
    out = {"workload": "%d matrices, n ~ U{8..512} (seed 2027), 4 right-hand sides" % count}
    flop_chol = float(np.sum(sizes.astype(np.float64) ** 3 / 3 + 8.0 * sizes.astype(np.float64) ** 2))
    flop_lu = float(np.sum(2 * sizes.astype(np.float64) ** 3 / 3 + 8.0 * sizes.astype(np.float64) ** 2))
    lda = sizes.copy()
    info = np.zeros(count, dtype=np.int32)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    for kind, dt in (("chol", torch.float64), ("chol", torch.float32), ("lu", torch.float64)):
        src = torch.empty(int(offs[-1]), dtype=dt, device=dev)
        for nval in np.unique(sizes):
            idx = np.nonzero(sizes == nval)[0]
            nv = int(nval)
            if kind == "chol":
                G = torch.randn((len(idx), nv, nv), dtype=torch.float64, device=dev, generator=g)
                M = G @ G.transpose(1, 2) / nv + torch.eye(nv, dtype=torch.float64, device=dev)
            else:
                M = torch.rand((len(idx), nv, nv), dtype=torch.float64, device=dev, generator=g) * 2 - 1
            for q, i in enumerate(idx):
                src[int(offs[i]):int(offs[i + 1])] = M[q].t().reshape(-1).to(dt)  # column-major
        work = src.clone()
        bsrc = torch.randn(int(boffs[-1]), dtype=dt, device=dev, generator=g)
        bwork = bsrc.clone()
        es = work.element_size()
        A = (C.c_void_p * count)(*[work.data_ptr() + int(offs[i]) * es for i in range(count)])
        B = (C.c_void_p * count)(*[bwork.data_ptr() + int(boffs[i]) * es for i in range(count)])
        pivbuf = torch.empty(int(sizes.sum()), dtype=torch.int32, device=dev)
        poffs = np.concatenate([[0], np.cumsum(sizes)])
        PV = (C.c_void_p * count)(*[pivbuf.data_ptr() + int(poffs[i]) * 4 for i in range(count)])
        times = []
        for rep in range(4):
            work.copy_(src)
            bwork.copy_(bsrc)
            torch.cuda.synchronize()
            if kind == "chol" and dt == torch.float64:
                r = L.FLA_Chol_batched(F.FLA_LOWER_TRIANGULAR, count, P(sizes), A, P(lda), nrhs, B, P(lda), P(info))
            elif kind == "chol":
                r = L.FLA_B200_Chol_batched_f32(count, P(sizes), A, P(lda), nrhs, B, P(lda), P(info))
            else:
                r = L.FLA_LU_piv_batched(count, P(sizes), A, P(lda), PV, nrhs, B, P(lda), P(info))
            if r != F.FLA_SUCCESS:
                raise RuntimeError("batched %s failed: %s" % (kind, F.last_error()))
            if rep > 0:
                times.append(F.last_op_ms())
        ms = statistics.median(times)
        fl = flop_chol if kind == "chol" else flop_lu
        key = "%s_%s" % (kind, "fp64" if dt == torch.float64 else "fp32")
        out[key] = {"ms": ms, "tflops": fl / (ms * 1e-3) / 1e12, "matrices_per_s": count / (ms * 1e-3),
                    "failed": int((info != -1).sum())}
        del src, work, bsrc, bwork, pivbuf
        torch.cuda.empty_cache()
    out["note"] = ("FP64 Cholesky: DMMA (FP64 tensor-core) left-looking kernel; FP32 Cholesky and LU: SIMT FMA "
                   "kernels; one CTA per matrix, persistent grid, largest first; tflops includes the solves")
    return out


def gp_batched_section(torch, dev, F, count=256):
    """count Gaussian-process likelihoods, n ~ U{64..1024} (seed 256): K =
    exp(-|xi-xj|^2 / (2 0.3^2)) + 1e-2 I for x ~ U[0,1]^3, y ~ N(0,1).
    Forward: FLA_B200_Chol_batched_logdet (Cholesky, alpha = K^-1 y,
    log-determinant) in one launch; backward: Lbar = -tril(alpha v^T),
    v = L^T alpha (torch, untimed), then FLA_Chol_adjoint_batched with the
    log-determinant term.  Device times of the library's calls; forward flops
    n^3/3 + 2 n^2 per GP."""
    rng = np.random.default_rng(256)
    sizes = [int(v) for v in rng.integers(64, 1025, size=count)]
    g = torch.Generator(device=dev).manual_seed(256)

    def colmajor(t):
        out = torch.empty_strided(tuple(t.shape), (1, t.shape[0]), dtype=t.dtype, device=t.device)
        out.copy_(t)
        return out
    Ks0, ys = [], []
    for n in sizes:
        x = torch.rand((n, 3), dtype=torch.float64, device=dev, generator=g)
        K = torch.exp(-torch.cdist(x, x) ** 2 / (2 * 0.3 ** 2)) + 1e-2 * torch.eye(n, dtype=torch.float64, device=dev)
        Ks0.append(colmajor(K))
        ys.append(colmajor(torch.randn((n, 1), dtype=torch.float64, device=dev, generator=g)))
    fwd, bwd = [], []
    for rep in range(4):
        Ks = [K.clone() for K in Ks0]
        al = [y.clone() for y in ys]
        torch.cuda.synchronize()
        r, info, logdet = F.chol_batched_logdet(Ks, rhs=al)
        if r != F.FLA_SUCCESS or any(v != -1 for v in info):
            raise RuntimeError("batched GP forward failed: %s" % F.last_error())
        fms = F.last_op_ms()
        Lbars = []
        for Ld, a in zip(Ks, al):
            v = torch.tril(Ld).t() @ a
            Lbars.append(colmajor(-torch.tril(a @ v.t())))
        torch.cuda.synchronize()
        if F.chol_adjoint_batched(Ks, Lbars, 1.0) != F.FLA_SUCCESS:
            raise RuntimeError("batched GP adjoint failed: %s" % F.last_error())
        bms = F.last_op_ms()
        if rep > 0:
            fwd.append(fms)
            bwd.append(bms)
    flops = float(sum(n ** 3 / 3.0 + 2.0 * n * n for n in sizes))
    fm = statistics.median(fwd)
    return {"workload": "%d GPs, n ~ U{64..1024} (seed 256), FP64" % count,
            "forward_ms": fm, "forward_tflops": flops / (fm * 1e-3) / 1e12, "adjoint_ms": statistics.median(bwd),
            "largest_n": max(sizes), "total_rows": int(sum(sizes))}


def qr_section(torch, dev, F, m, n, nrhs):
    """FLA_QR_UT of an m x n N(0,1) matrix (T = 32 x n) and FLA_Apply_Q_UT of
    Q^T to nrhs N(0,1) right-hand sides; device times of the library's calls.
    flops: 2 m n^2 - 2 n^3 / 3 (QR), 4 m n nrhs - 2 n^2 nrhs (apply)."""
    g = torch.Generator(device=dev).manual_seed(77)
    src = torch.randn((n, m), dtype=torch.float64, device=dev, generator=g).t()  # column-major m x n
    A = torch.empty((n, m), dtype=torch.float64, device=dev).t()
    T = torch.zeros((n, 32), dtype=torch.float64, device=dev).t()
    bsrc = torch.randn((nrhs, m), dtype=torch.float64, device=dev, generator=g).t()
    B = torch.empty((nrhs, m), dtype=torch.float64, device=dev).t()
    tq, ta = [], []
    for rep in range(3):
        A.copy_(src)
        B.copy_(bsrc)
        torch.cuda.synchronize()
        if F.qr_ut(A, T) != F.FLA_SUCCESS:
            raise RuntimeError("FLA_QR_UT failed: %s" % F.last_error())
        q = F.last_op_ms()
        if F.apply_q_ut(A, T, B) != F.FLA_SUCCESS:
            raise RuntimeError("FLA_Apply_Q_UT failed: %s" % F.last_error())
        if rep > 0:
            tq.append(q)
            ta.append(F.last_op_ms())
    fq = 2.0 * m * n * n - 2.0 * n ** 3 / 3
    fa = 4.0 * m * n * nrhs - 2.0 * n * n * nrhs
    mq, ma = statistics.median(tq), statistics.median(ta)
    del src, A, T, bsrc, B
    torch.cuda.empty_cache()
    return {"workload": "FLA_QR_UT m=%d n=%d N(0,1), T 32 x n; FLA_Apply_Q_UT (Q^T) on %d N(0,1) columns" % (m, n, nrhs),
            "qr_ms": mq, "qr_tflops": fq / (mq * 1e-3) / 1e12, "apply_q_ms": ma,
            "apply_q_tflops": fa / (ma * 1e-3) / 1e12}


def gp_section(torch, dev, F, n):
    """Gaussian-process marginal likelihood: x ~ U[0,1]^3 (n points, seeded),
    K = exp(-|xi-xj|^2 / (2 0.3^2)) + 1e-2 I, y ~ N(0,1).  Forward: FLA_Chol,
    the triangular solve for v = L^-1 y (FLA_Chol_solve's first half is
    done with the library's solve on [y]), loss = 0.5 v^T v + sum log L_ii.
    Backward: triangular-solve adjoint, log-determinant adjoint, then the
    blocked in-place Cholesky adjoint (FLA_Chol_adjoint) giving dloss/dK.
    Times: device times of the library calls; the gradient is checked
    against 0.5 (K^-1 - alpha alpha^T) (K^-1 from FLA_Chol_solve on I)."""
    g = torch.Generator(device=dev).manual_seed(8192)
    x = torch.rand((n, 3), dtype=torch.float64, device=dev, generator=g)
    K = torch.exp(-torch.cdist(x, x) ** 2 / (2 * 0.3 ** 2)) + 1e-2 * torch.eye(n, dtype=torch.float64, device=dev)
    y = torch.randn((n, 1), dtype=torch.float64, device=dev, generator=g)
    Ld = K.clone().t().contiguous().t()
    rc = F.chol(Ld)
    if rc != F.FLA_SUCCESS:
        raise RuntimeError("FLA_Chol returned %d: %s" % (rc, F.last_error()))
    t_chol = F.last_op_ms()
    Ld = torch.tril(Ld).t().contiguous().t()
    v = torch.linalg.solve_triangular(Ld, y, upper=False)
    times = []
    for rep in range(2):
        Lbar = torch.zeros((n, n), dtype=torch.float64, device=dev).t()
        vb = v.clone()
        ms = 0.0
        if F.trsm_llnn_adjoint(Ld, v.clone(), vb, Lbar) != F.FLA_SUCCESS:
            raise RuntimeError("trsm adjoint failed: %s" % F.last_error())
        ms += F.last_op_ms()
        r, logdet = F.chol_logdet_adjoint(Ld, Lbar, 1.0)
        if r != F.FLA_SUCCESS:
            raise RuntimeError("logdet adjoint failed: %s" % F.last_error())
        ms += F.last_op_ms()
        if F.chol_adjoint(Ld, Lbar) != F.FLA_SUCCESS:
            raise RuntimeError("FLA_Chol_adjoint failed: %s" % F.last_error())
        t_adj = F.last_op_ms()
        ms += t_adj
        times.append((ms, t_adj))
    G = torch.tril(Lbar)
    G = 0.5 * (G + G.t())
    Kinv = torch.cholesky_inverse(Ld)
    alpha = Kinv @ y
    Gref = 0.5 * (Kinv - alpha @ alpha.t())
    rel = ((G - Gref).norm() / Gref.norm()).item()
    bw, ta = min(times)
    del K, Ld, Lbar, G, Kinv, Gref
    torch.cuda.empty_cache()
    return {"workload": "GP marginal likelihood, n=%d points in [0,1]^3, RBF 0.3 + 1e-2 I" % n,
            "chol_ms": t_chol, "backward_ms": bw, "chol_adjoint_ms": ta,
            "chol_adjoint_tflops": (2.0 * n ** 3 / 3) / (ta * 1e-3) / 1e12,
            "grad_rel_err_vs_closed_form": rel,
            "note": "closed form built with torch on the GPU; the committed tests check against the oracle and "
                    "central differences"}


def lu_parity(torch, dev, F, A0, LU, piv):
    """The timed run's factorization against the reference libflame's
    record on the same input (tests/golden/headline_lu.npz): pivots,
    factor sketches, diagonal and backward error."""
    H = headline()
    rec = np.load(os.path.join(ROOT, "tests", "golden", "headline_lu.npz"))
    pv = piv.cpu().numpy()
    bad = int((pv != rec["p"]).sum())
    rel = H.sketch_rel_diff(H.sketches(torch, LU, dev), (rec["sk_l"], rec["sk_r"]))
    d = torch.diagonal(LU).cpu().numpy()
    be = H.lu_backward_error(torch, A0, LU, pv, dev)
    return {"against": "reference libflame FLA_LU_piv (f2c BLAS) on the same seeded input",
            "pivots_identical": bad == 0, "pivot_mismatches": bad,
            "factor_rel_diff_sketch": rel,
            "diag_rel_diff": float(np.linalg.norm(d - rec["diag"]) / np.linalg.norm(rec["diag"])),
            "backward_error": be, "backward_error_reference": float(rec["be"])}


def chol_n1024_section(torch, dev, F, peak, reps=60):
    """FLA_Chol lower, n = 1024, A = G G^T / 1024 + I (the reference's own
    CPU configuration): median device time of `reps` factorizations, each of
    a freshly restored A after a 256 MiB write that evicts L2."""
    n = 1024
    G = np.random.default_rng(1024).standard_normal((n, n))
    src = torch.from_numpy(G @ G.T / n + np.eye(n)).to(dev)  # symmetric: either order
    work = torch.empty((n, n), dtype=torch.float64, device=dev).t()  # column-major
    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device=dev)
    vW = F.View(work)
    L = F.lib()
    times = []
    for i in range(reps + 5):
        flush.fill_(float(i))
        work.copy_(src)
        torch.cuda.synchronize()
        if L.FLA_Chol(F.FLA_LOWER_TRIANGULAR, vW.obj) != F.FLA_SUCCESS:
            raise RuntimeError("FLA_Chol n=1024 failed: %s" % F.last_error())
        if i >= 5:
            times.append(F.last_op_ms())
    ms = statistics.median(times)
    tf = n ** 3 / 3.0 / (ms * 1e-3) / 1e12
    del src, work, flush
    return {"workload": "FLA_Chol lower n=1024, A = G G^T/1024 + I, L2 evicted before each run",
            "runs": reps, "median_ms": ms, "min_ms": min(times), "tflops": tf, "frac_of_peak": tf / peak}


def chol_n16384_section(torch, dev, F, peak):
    """FLA_Chol lower, n = 16384, A = G G^T / n + I (the parity input of
    tests/golden/headline.py): median of 3 device-timed factorizations."""
    H = headline()
    n = H.CHOL_N
    spd_src = H.chol_input_torch(torch, H.chol_factor_input(), dev)  # symmetric
    work = torch.empty((n, n), dtype=torch.float64, device=dev).t()  # column-major
    vC = F.View(work)
    L = F.lib()
    ct = []
    for i in range(4):
        work.copy_(spd_src)
        torch.cuda.synchronize()
        r = L.FLA_Chol(F.FLA_LOWER_TRIANGULAR, vC.obj)
        if r != F.FLA_SUCCESS:
            raise RuntimeError("FLA_Chol returned %d" % r)
        if i > 0:
            ct.append(F.last_op_ms())
    cms = statistics.median(ct)
    rec = np.load(os.path.join(ROOT, "tests", "golden", "headline_chol.npz"))
    Lt = torch.tril(work)
    rel = H.sketch_rel_diff(H.sketches(torch, Lt, dev), (rec["sk_l"], rec["sk_r"]))
    be = H.chol_backward_error(torch, spd_src, Lt)
    del spd_src, work, Lt
    torch.cuda.empty_cache()
    tf = n ** 3 / 3.0 / (cms * 1e-3) / 1e12
    return {"ms": cms, "tflops": tf, "frac_of_peak": tf / peak,
            "parity": {"factor_rel_diff_sketch": rel, "backward_error": be,
                       "backward_error_reference": float(rec["be"])}}


def run_ours(args, rank, world):
    import ctypes as C
    import torch
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    sys.path.insert(0, ROOT)
    import libflame_b200 as F
    F.init()
    L = F.lib()
    n = args.n
    flops = 2.0 / 3.0 * n ** 3
    A_host = lu_input(n)
    src = torch.from_numpy(np.ascontiguousarray(A_host.T)).to(dev).t()  # column-major on the device
    del A_host
    work = torch.empty((n, n), dtype=torch.float64, device=dev).t()
    piv = torch.empty(n, dtype=torch.int32, device=dev)
    vA, vp = F.View(work), F.View(piv)

    def step():
        work.copy_(src)  # restore the input (also evicts L2: 2 GiB written)
        torch.cuda.synchronize()
        r = L.FLA_LU_piv(vA.obj, vp.obj)
        if r != F.FLA_SUCCESS:
            raise RuntimeError("FLA_LU_piv returned %d: %s" % (r, F.last_error()))
        return F.last_op_ms()

    for _ in range(args.warmup):
        step()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev.index if dev.index is not None else 0)
    sampler.start()
    l0 = F.kernel_launches()
    t_wall = time.perf_counter()
    times = [step() for _ in range(args.steps)]
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    launches = F.kernel_launches() - l0
    clocks = sampler.stop()
    if world > 1:
        torch.distributed.barrier()
    ms = sum(times) / len(times)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    value = world * flops / (ms * 1e-3) / 1e12

    # parity of the last timed factorization (still in work / piv)
    parity = None
    if rank == 0 and n == headline().LU_N:
        parity = lu_parity(torch, dev, F, src, work, piv)
        torch.cuda.empty_cache()

    # per-kernel-class profile of one more factorization (outside the timed region)
    F.profile(True)
    step()
    prof = {name: F.profile_read(c) for name, c in
            [("gemm", F.PROF_GEMM), ("panel", F.PROF_PANEL), ("trsm", F.PROF_TRSM),
             ("swap", F.PROF_SWAP), ("diag", F.PROF_DIAG)]}
    F.profile(False)
    total_ms = F.last_op_ms()
    gemm_ms, gemm_flops, gemm_n = prof["gemm"]

    result = None
    if rank == 0:
        peak = measure_fp64_peak(torch, dev)
        achieved = gemm_flops / (gemm_ms * 1e-3) / 1e12 if gemm_ms > 0 else None
        roofline = {
            "bound": "tensor", "kernel": "dgemm_tma_kernel (FP64 DMMA, trailing update A22 -= A21 A12)",
            "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak if achieved else None,
            "peak_source": "cuBLAS DGEMM 8192^3 (torch.matmul fp64, best of 10) measured in this run; "
                           "MEASURED_PEAKS.json has no FP64 figure",
            # DRAM bytes per launch: 0.0574 bytes per flop (dram__bytes_read
            # + write of an ncu capture of this kernel in an n = 6144 LU)
            # times this run's average launch
            "traffic": 0.0574 * gemm_flops / gemm_n if gemm_n else None,
            "traffic_unit": "bytes per launch (ncu DRAM read + write, scaled per flop from n=6144)",
            "launches_per_step": gemm_n,
            "share_of_step": gemm_ms / total_ms if total_ms > 0 else None,
            "whole_factorization_frac_of_peak": value / world / peak,
        }
        if parity is not None:
            roofline["lu_parity"] = parity
        breakdown = {k: {"ms": v[0], "launches": v[2]} for k, v in prof.items()}
        result = {
            "metric": METRIC, "value": value, "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": lu_config(n, world),
            "roofline": roofline, "breakdown_ms": breakdown,
            "implementation": {"lu_blocksize": 128, "chol_blocksize": 256, "lookahead": True},
            "gpu_launches": launches, "clocks": clocks,
            "wall_ms_per_step_incl_restore": 1000.0 * t_wall / args.steps,
        }

    # ---- e2e through the LAPACK ABI with pinned host buffers
    if rank == 0 and args.e2e_steps > 0:
        host_src = src.t().contiguous().t().cpu()  # column-major host copy
        pinned = torch.empty((n, n), dtype=torch.float64).pin_memory().t()
        ipiv = torch.empty(n, dtype=torch.int32).pin_memory()
        nn = C.c_int(n)
        info = C.c_int(0)
        e2e_t = []
        for i in range(args.e2e_steps + 1):
            pinned.copy_(host_src)
            t0 = time.perf_counter()
            L.dgetrf_(C.byref(nn), C.byref(nn), C.c_void_p(pinned.data_ptr()), C.byref(nn),
                      C.c_void_p(ipiv.data_ptr()), C.byref(info))
            dt = time.perf_counter() - t0
            if i > 0:  # first call warms the staging buffers
                e2e_t.append(dt)
        e2e = statistics.median(e2e_t)
        result["e2e"] = {"value": flops / e2e / 1e12, "unit": "TFLOP/s",
                         "h2d_bytes_per_step": n * n * 8, "d2h_bytes_per_step": n * n * 8 + n * 4,
                         "path": "dgetrf_ on pinned host buffers (wall clock, includes H2D + D2H)"}
        del pinned, host_src
    del src
    torch.cuda.empty_cache()

    # ---- FP64 FLA_Chol: n=16384 (target: >= 70 % of the FP64 tensor peak)
    # and n=1024 (the reference's own CPU configuration)
    if rank == 0 and not args.no_secondary:
        peak = result["roofline"]["peak"]
        result["roofline"]["chol_n16384"] = chol_n16384_section(torch, dev, F, peak)
        result["roofline"]["chol_n1024"] = chol_n1024_section(torch, dev, F, peak)

    # ---- mixed-precision refinement against the FP64 form at equal error
    if rank == 0 and not args.no_ir:
        result["mixed_ir"] = mixed_ir_section(torch, dev, F, args.ir_n, 32, not args.no_cpu_baseline)
        result["roofline"]["mixed_ir_speedup"] = {
            k: {"speedup": v["speedup"], "path": v["path"], "backward_error_mixed": v["backward_error_mixed"],
                "backward_error_fp64": v["backward_error_fp64"]}
            for k, v in result["mixed_ir"]["cases"].items()}

    # ---- batched factorizations + solves of many uneven matrices
    if rank == 0 and not args.no_batched:
        result["batched"] = batched_section(torch, dev, F, args.batch_count)
        result["batched"]["gp_256"] = gp_batched_section(torch, dev, F)

    # ---- QR_UT + Apply_Q_UT and the Gaussian-process gradient
    if rank == 0 and not args.no_secondary:
        result["qr"] = qr_section(torch, dev, F, 16384, 8192, 64)
        result["gp"] = gp_section(torch, dev, F, 8192)

    # ---- CPU baseline: the reference over OpenBLAS on all host threads, on
    # the same workload when one factorization fits in ~30 s, else a
    # bounded sample; the SuperMatrix / f2c-BLAS build beside it
    if rank == 0 and not args.no_cpu_baseline:
        try:
            nthreads = host_threads()
            nb, _ = pick_reference_n(n, nthreads, 1, 30.0)
            tf, secs = reference_lu_openblas(nb, nthreads)
            tf2, _ = reference_lu_flash(3072, nthreads)
            result["cpu_baseline"] = {
                "value": tf, "unit": "TFLOP/s", "cores": nthreads, "kind": "reference",
                "sample": "reference libflame flat FLA_LU_piv over OpenBLAS 0.3.30, %d threads, n=%d (%.1f s)"
                          % (nthreads, nb, secs),
                "secondary": {"value": tf2, "sample": "FLASH_LU_piv (SuperMatrix, built-in f2c BLAS, block 256) "
                                                      "n=3072, %d threads" % nthreads}}
        except Exception as e:  # the reference library is test infrastructure
            result["cpu_baseline"] = {"value": None, "unit": "TFLOP/s", "cores": 0, "kind": "reference",
                                      "sample": "unavailable: %s" % e}
    if rank == 0:
        print(json.dumps(result), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.profile_op:
        profile_op(args)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    try:
        run_ours(args, rank, world)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
