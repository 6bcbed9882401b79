"""Instance sharding across ranks (one process per GPU).

SF-SCF instances of a sweep are independent, so every rank solves its own
disjoint set and the only communication is timing/count aggregation after
the timed region: the job time is the max over ranks and the solve count
the sum (weak scaling, no collective on the data path).
"""
from __future__ import annotations

from typing import List, Tuple

SEED_STRIDE = 1000


def instance_seeds(rank: int, count: int, base: int) -> List[int]:
    """Seeds of the instances one rank builds: disjoint across ranks for
    count <= SEED_STRIDE."""
    if count > SEED_STRIDE:
        raise ValueError(f"at most {SEED_STRIDE} instances per rank")
    return [base + SEED_STRIDE * rank + i for i in range(count)]


def aggregate(elapsed_s: float, solved: int, world: int, device=None) -> Tuple[float, float]:
    """(max elapsed over ranks, total solved) with one all_reduce each;
    identity without a process group."""
    if world <= 1:
        return float(elapsed_s), float(solved)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(elapsed_s)], dtype=torch.float64, device=device)
    n = torch.tensor([float(solved)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    dist.all_reduce(n, op=dist.ReduceOp.SUM)
    return t.item(), n.item()
