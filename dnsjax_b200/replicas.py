"""Replica bookkeeping for multi-GPU runs.

The time-step path has no data exchange on one trajectory (no pencil
decomposition); N GPUs advance N independent trajectories.  The only
collectives are the timing reduction (max over ranks) and the barriers that
bracket the timed region.
"""

from __future__ import annotations


def replica_seed(base_seed: int, rank: int) -> int:
    """Seed of the trajectory advanced by ``rank``."""
    return base_seed + rank


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """``value`` reduced with MAX over the process group (identity if no
    group is initialised)."""
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def total_steps(steps_per_rank: int, world: int) -> int:
    """Units processed by the whole job (weak scaling: fixed per rank)."""
    return steps_per_rank * world
