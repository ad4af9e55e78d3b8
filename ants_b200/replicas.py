"""Multi-GPU as independent replicas (one registration pair per rank, one process per GPU).

Within one pair every SyN iteration needs global gathers and global reductions, so the path is not
sharded; ranks run independent pairs and the only collectives are the end-of-run aggregation of the
timing (max over ranks) and of the work done (sum over ranks).
"""
from __future__ import annotations

from .phantoms import SEED_BASE


def pair_seed(rank: int, base: int = SEED_BASE) -> int:
    """Seed of the pair a rank registers (pair index = rank)."""
    return base + rank


def assign_pairs(n_pairs: int, world: int, rank: int) -> list[int]:
    """Round-robin assignment of pair indices to ranks (used for batches of pairs)."""
    return list(range(rank, n_pairs, world))


def aggregate(seconds: float, voxel_iterations: int, device=None) -> tuple[float, int]:
    """(max over ranks of the timed seconds, sum over ranks of voxel-iterations); identity when
    torch.distributed is not initialised."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return seconds, voxel_iterations
    t = torch.tensor([seconds], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    v = torch.tensor([float(voxel_iterations)], dtype=torch.float64, device=device)
    dist.all_reduce(v, op=dist.ReduceOp.SUM)
    return float(t.item()), int(v.item())
