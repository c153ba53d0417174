"""Multi-GPU sharding of the population search (one process per GPU).

States, chains and temperature ladders are independent, so the work splits
across ranks with no data-path exchange: each rank owns a contiguous block of
seeds (scoring) or of whole ladders (tempering; a ladder never spans GPUs).
The only collectives are host-side bookkeeping after the device work: the max
over ranks of a measured time, and a min-reduce plus gather of the best
energies and states (a few hundred bytes per rank).  The reference has no
multi-GPU path; this mirrors its single-process population conventions
(seeds 91001 + i, src/no_three_75/cli.py:203-204).
"""
from __future__ import annotations

import numpy as np


def seed_block(rank: int, world: int, per_rank: int, base: int = 91001) -> range:
    """Seeds of rank `rank` when every rank scores `per_rank` states (weak scaling)."""
    if not 0 <= rank < world or per_rank < 0:
        raise ValueError("rank outside [0, world) or negative block")
    start = base + rank * per_rank
    return range(start, start + per_rank)


def ladder_block(n_ladders: int, rank: int, world: int) -> range:
    """Contiguous ladders owned by `rank` when `n_ladders` are split over
    `world` ranks (strong scaling); sizes differ by at most one."""
    if not 0 <= rank < world:
        raise ValueError("rank outside [0, world)")
    lo = n_ladders * rank // world
    hi = n_ladders * (rank + 1) // world
    return range(lo, hi)


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (the timing rule for multi-GPU runs)."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def global_best(best_energy: int, best_columns: np.ndarray, device=None):
    """(E, rank, columns) of the lowest best energy over all ranks; ties go to
    the lowest rank.  Every rank receives the winner's state."""
    import torch
    import torch.distributed as dist

    cols = np.asarray(best_columns, dtype=np.int16).reshape(-1)
    if not dist.is_initialized() or dist.get_world_size() == 1:
        return int(best_energy), 0, cols
    world, rank = dist.get_world_size(), dist.get_rank()
    key = torch.tensor([int(best_energy) * world + rank], dtype=torch.int64, device=device)
    dist.all_reduce(key, op=dist.ReduceOp.MIN)
    winner = int(key.item()) % world
    e = int(key.item()) // world
    buf = torch.from_numpy(cols.astype(np.int32)).to(device if device is not None else "cpu")
    dist.broadcast(buf, src=winner)
    return e, winner, buf.cpu().numpy().astype(np.int16)
