"""Multi-GPU plumbing for independent systems.

The single-system CPR-GMRES path is not sharded: one GPU owns one system (the
reference's in-house FSAI is single-rank too, README.md:10-12).  With several
GPUs each rank solves its own systems — replicas of one workload, or disjoint
shares of a batch — with no collective on the data path.  The only exchange is
the timing reduction: the job time is the maximum over ranks.
"""
from __future__ import annotations


def shard(n_items: int, rank: int, world: int) -> range:
    """Contiguous share of `n_items` independent systems for `rank` (sizes differ by at most one)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def deal(n_items: int, rank: int, world: int) -> list[int]:
    """Round-robin share of `n_items` independent systems for `rank`: items rank,
    rank + world, ...  Systems of a batch are generated in random size order, so
    dealing them spreads the large ones over the ranks (the batched bench's split)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    return list(range(rank, n_items, world))


def max_over_ranks(value: float, device=None) -> float:
    """All-reduce MAX of a per-rank scalar (identity without an initialised process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
