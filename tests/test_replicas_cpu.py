"""The multi-rank path on CPU: two gloo ranks (127.0.0.1), each owning a
shard of independent problems.  The shards cover the batch exactly once,
the per-rank results (here from the CPU oracle) assemble into the
single-process result, and the timing reduction takes the slowest rank."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from kami_b200 import replicas


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r, w, lr = replicas.rank_world()
        assert (r, w, lr) == (rank, world, rank)
        batch = 37
        rng = np.random.default_rng(0)
        A = rng.integers(-3, 4, (batch, 8, 8)).astype(np.float64)
        B = rng.integers(-3, 4, (batch, 8, 8)).astype(np.float64)
        lo, hi = replicas.shard(batch, rank, world)
        C = oracle.gemm(A[lo:hi], B[lo:hi])
        # gather the shards (a test-side check only; the product path has no collective)
        parts = [None] * world
        dist.all_gather_object(parts, (lo, hi, C))
        full = np.zeros((batch, 8, 8))
        for a, b, c in parts:
            full[a:b] = c
        ok_cover = sorted((a, b) for a, b, _ in parts)
        replicas.barrier()
        mx = replicas.max_over_ranks([1.0 + rank, 10.0 - rank])
        rate = replicas.aggregate_rate(100.0, mx[0], world)
        out[rank] = (np.array_equal(full, oracle.gemm(A, B)), ok_cover, mx, rate)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce():
    world = 2
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()  # no fork of this multi-threaded process
    out = mgr.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    for rank in range(world):
        same, cover, mx, rate = out[rank]
        assert same
        assert cover == [(0, 19), (19, 37)]
        assert mx == [2.0, 10.0]
        assert rate == pytest.approx(100.0 * world / 2e-3)


@pytest.mark.parametrize("total,world", [(0, 3), (5, 8), (592, 8), (37, 2), (1, 1)])
def test_shard_partitions_exactly(total, world):
    got = [replicas.shard(total, r, world) for r in range(world)]
    assert got[0][0] == 0 and got[-1][1] == total
    assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
    sizes = [b - a for a, b in got]
    assert max(sizes) - min(sizes) <= 1


def test_single_process_is_identity():
    assert replicas.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    with pytest.raises(ValueError):
        replicas.shard(10, 2, 2)
