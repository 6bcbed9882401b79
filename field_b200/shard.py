"""Instance sharding across ranks (one process per GPU).

SF-SCF instances of a sweep are independent, so every rank solves its own
disjoint set and the only communication is timing/count aggregation after
the timed region: the job time is the max over ranks and the solve count
the sum (weak scaling, no collective on the data path).

Uneven instances (a sweep over chain length and lattice size) are spread by
their estimated cost, sum over molecules of N * M * K per residual
evaluation times the expected number of iterations, with greedy
longest-processing-time bin packing: instances in decreasing cost order, each
to the rank with the least load so far.
"""
from __future__ import annotations

from typing import Iterable, List, Optional, Sequence, Tuple

SEED_STRIDE = 1000


def instance_seeds(rank: int, count: int, base: int) -> List[int]:
    """Seeds of the instances one rank builds: disjoint across ranks for
    count <= SEED_STRIDE."""
    if count > SEED_STRIDE:
        raise ValueError(f"at most {SEED_STRIDE} instances per rank")
    return [base + SEED_STRIDE * rank + i for i in range(count)]


def residual_cost(spec) -> float:
    """Propagator site-steps of one residual evaluation: sum over molecules of
    N * M * K (forward and backward sweeps each visit N positions of K*M
    values; monomers cost one M-vector)."""
    M = spec.M
    K = spec.lattice.components
    return float(sum(max(mol.N, 1) * M * K for mol in spec.molecules))


def estimate_cost(spec, iterations: Optional[float] = None) -> float:
    """Estimated cost of a whole solve: residual_cost * iterations (50 when
    the iteration count is unknown)."""
    return residual_cost(spec) * (50.0 if iterations is None else float(iterations))


def partition(costs: Sequence[float], world: int) -> List[List[int]]:
    """Greedy LPT bin packing of instance indices over `world` ranks.
    Deterministic: ties in cost go by index, ties in load by rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    loads = [0.0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += float(costs[i])
    for p in parts:
        p.sort()
    return parts


def load_imbalance(costs: Sequence[float], parts: Iterable[Sequence[int]]) -> float:
    """max rank load / mean rank load (1.0 is perfect balance)."""
    loads = [sum(float(costs[i]) for i in p) for p in parts]
    mean = sum(loads) / len(loads)
    return max(loads) / mean if mean > 0 else 1.0


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


def gather_results(local: dict, world: int) -> dict:
    """Union of every rank's {instance index: result} after the solves (host
    objects, one all_gather_object; identity without a process group)."""
    if world <= 1:
        return dict(local)
    import torch.distributed as dist
    parts = [None] * world
    dist.all_gather_object(parts, local)
    out = {}
    for p in parts:
        overlap = set(out) & set(p)
        if overlap:
            raise ValueError(f"instances {sorted(overlap)[:5]} solved on two ranks")
        out.update(p)
    return out
