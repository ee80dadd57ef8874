"""Multi-GPU helpers for throughput runs: frame pairs are independent, so each
rank solves its own pairs with no data-path collective (weak scaling).  The
only collective is the timing reduction (max over ranks)."""
from __future__ import annotations


def rank_seeds(rank: int, world: int, pairs_per_rank: int, base: int = 0) -> list[int]:
    """Disjoint, reproducible generator seeds for one rank's pairs."""
    if not (0 <= rank < world) or pairs_per_rank < 0:
        raise ValueError("bad rank / world / pairs")
    start = base + rank * pairs_per_rank
    return list(range(start, start + pairs_per_rank))


def shard(items: list, rank: int, world: int) -> list:
    """Round-robin split of a work list (e.g. uneven pairs) across ranks."""
    return items[rank::world]


def max_over_ranks(x: float, device=None) -> float:
    """Max of a per-rank scalar over the default process group (no-op without
    one).  `device` is the tensor device the backend needs (cuda for NCCL)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
