"""Multi-GPU plumbing for the block-GEMM path: one process per GPU, each
owning a contiguous shard of independent problems (no data-path
collective; the reference is single-GPU and its problems never exchange
data).  torch.distributed is used only to align the timed region (a
barrier) and to take the slowest rank's time (a MAX reduction), so the
aggregate throughput is the units all ranks processed over the max-over-
ranks time.  Works with NCCL (GPU tensors) and gloo (CPU tensors)."""
from __future__ import annotations

import os

import torch
import torch.distributed as dist


def rank_world() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard(total: int, rank: int, world: int) -> tuple[int, int]:
    """Contiguous [start, stop) of `total` problems for `rank`; the first
    total % world ranks take one extra problem, every problem is owned by
    exactly one rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank / world")
    q, r = divmod(total, world)
    start = rank * q + min(rank, r)
    return start, start + q + (1 if rank < r else 0)


def barrier() -> None:
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()


def max_over_ranks(values, device=None) -> list[float]:
    """Element-wise maximum of a list of floats over all ranks (identity on
    one process).  device: where the reduction tensor lives (a CUDA device
    for NCCL, None / cpu for gloo)."""
    vals = [float(v) for v in values]
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return vals
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def aggregate_rate(units_per_rank: float, max_ms: float, world: int) -> float:
    """Whole-job rate: the units all ranks processed (weak scaling: the same
    count per rank) over the slowest rank's time, per second."""
    return units_per_rank * world / (max_ms * 1e-3)
