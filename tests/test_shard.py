"""Sharding of the batched factorizations: the LPT partition (CPU) and the
info gather over a world_size-2 gloo process group (CPU processes; the GPU
launch itself is covered by test_gpu_batched)."""
import os
import socket

import numpy as np
import pytest

from libflame_b200.shard import flop_weights, gather_info, local_share, partition_lpt


def test_partition_covers_every_matrix_once_and_balances():
    rng = np.random.default_rng(3)
    sizes = rng.integers(8, 513, size=10000)
    w = flop_weights(sizes, "lu", 4)
    for parts in (1, 2, 3, 8):
        p = partition_lpt(w, parts)
        allidx = np.sort(np.concatenate(p))
        assert np.array_equal(allidx, np.arange(len(sizes)))
        loads = np.array([w[q].sum() for q in p])
        # LPT bound: max load <= mean + largest item
        assert loads.max() <= loads.mean() + w.max() + 1e-6
        assert loads.max() / loads.mean() < 1.001


def test_partition_is_deterministic_and_handles_edges():
    w = [5.0, 5.0, 1.0]
    assert [list(x) for x in partition_lpt(w, 2)] == [[0, 2], [1]]
    assert [list(x) for x in partition_lpt([], 3)] == [[], [], []]
    assert [list(x) for x in partition_lpt([1.0], 4)] == [[0], [], [], []]
    with pytest.raises(ValueError):
        partition_lpt(w, 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, sizes, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        idx = local_share(sizes, rank, world, "chol", 4)
        # stand-in for the per-matrix info words of this rank's launch
        info = [(-1 if i % 7 else i % 5) for i in idx]
        merged = gather_info(info, idx, len(sizes))
        q.put((rank, list(idx), merged.tolist()))
    finally:
        dist.destroy_process_group()


def test_gather_info_world2_gloo():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    sizes = list(np.random.default_rng(5).integers(8, 513, size=257))
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, sizes, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    expect = [(-1 if i % 7 else i % 5) for i in range(len(sizes))]
    shares = {}
    for rank, idx, merged in res:
        assert merged == expect
        shares[rank] = set(idx)
    assert shares[0].isdisjoint(shares[1]) and len(shares[0] | shares[1]) == len(sizes)
