"""Sharding of the batched factorizations over the ranks of a process group.

The matrices of a batch are independent, so a batch splits across GPUs with
no collective on the data path: each rank factors (and solves) its own share
with one FLA_Chol_batched / FLA_LU_piv_batched launch on its own GPU.  The
share is chosen by longest-processing-time-first on the flop weight of each
matrix (n^3/3 for Cholesky, 2n^3/3 for LU, plus the solves), the same
largest-first order the batched kernel uses to take matrices off its queue.
Only the per-matrix info words travel (one all-gather), so the caller sees the
batch's info vector in the original order.
"""
import heapq

import numpy as np


def flop_weights(sizes, kind="chol", nrhs=0):
    """Flops of each matrix: factorization + a nrhs-column solve."""
    n = np.asarray(sizes, dtype=np.float64)
    f = n ** 3 / 3.0 if kind == "chol" else 2.0 * n ** 3 / 3.0
    return f + 2.0 * nrhs * n * n


def partition_lpt(weights, nparts):
    """Longest-processing-time-first: matrices in decreasing weight (ties by
    index) each go to the part with the least load so far (ties by part
    index).  Returns one ascending index array per part; deterministic, so
    every rank computes the same partition without communication."""
    w = np.asarray(weights, dtype=np.float64)
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    order = sorted(range(len(w)), key=lambda i: (-w[i], i))
    heap = [(0.0, p) for p in range(nparts)]
    parts = [[] for _ in range(nparts)]
    for i in order:
        load, p = heapq.heappop(heap)
        parts[p].append(i)
        heapq.heappush(heap, (load + w[i], p))
    return [np.array(sorted(p), dtype=np.int64) for p in parts]


def local_share(sizes, rank, world, kind="chol", nrhs=0):
    """Indices of the matrices rank `rank` of `world` factors."""
    return partition_lpt(flop_weights(sizes, kind, nrhs), world)[rank]


def gather_info(local_info, local_idx, count, group=None):
    """All ranks' info words back into batch order (one all_gather of a
    fixed-size int64 vector: -2 marks entries another rank owns)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    full = np.full(count, -2, dtype=np.int64)
    full[np.asarray(local_idx, dtype=np.int64)] = np.asarray(local_info, dtype=np.int64)
    t = torch.from_numpy(full)
    if dist.get_backend(group) == "nccl":
        t = t.cuda()
    outs = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(outs, t, group=group)
    merged = np.full(count, -2, dtype=np.int64)
    for o in outs:
        o = o.cpu().numpy()
        sel = o != -2
        merged[sel] = o[sel]
    return merged


def batched_sharded(kind, mats, pivs=None, rhs=None, f32=False, group=None):
    """FLA_Chol_batched / FLA_LU_piv_batched over the ranks of `group`: each
    rank passes the whole batch (its own CUDA tensors, e.g. generated from a
    shared seed), factors its LPT share with one launch, and gets the
    batch's info vector back in order.  Matrices outside the share are left
    untouched on this rank."""
    import torch.distributed as dist
    from . import batched
    sizes = [m.shape[0] for m in mats]
    nrhs = 0 if rhs is None else rhs[0].shape[1]
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    idx = local_share(sizes, rank, world, kind, nrhs)
    sub = lambda xs: None if xs is None else [xs[i] for i in idx]  # noqa: E731
    r, info = batched(kind, sub(mats), sub(pivs), sub(rhs), f32) if len(idx) else (-1, [])
    return r, gather_info(info, idx, len(mats), group).tolist()
