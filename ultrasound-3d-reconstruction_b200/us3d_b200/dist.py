"""Frame sharding across ranks (one process per GPU) and max-over-ranks timing.

Frames are independent given the Gaussian parameters, so a multi-GPU run gives each rank a
disjoint set of frames and needs no collective on the data path; only the benchmark's
timing uses one (the maximum of the ranks' device times).
"""

from __future__ import annotations

from typing import List


def shard_frames(n_frames: int, rank: int, world: int) -> List[int]:
    """Frame indices owned by `rank`: a contiguous block, sizes differing by at most one."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError(f"bad rank/world {rank}/{world}")
    base, extra = divmod(n_frames, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks of the default process group (identity if none)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
