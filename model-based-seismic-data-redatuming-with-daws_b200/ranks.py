"""Shot partition over ranks and max-over-ranks timing (host side only).

Shots are independent, so ranks split them with no data-path exchange; the
only collectives are a barrier around the timed region and the max of the
per-rank device times.  The partition is the block split of the reference's
para_range (src/para_range.f90:11-22), which main_redatum_daw also uses.
"""
from __future__ import annotations

import datetime
import os


def para_range(n1: int, n2: int, nprocs: int, irank: int) -> tuple[int, int]:
    """Inclusive [ista, iend] of iterations n1..n2 for rank irank of nprocs
    (src/para_range.f90:15-20); iend < ista when the rank gets none."""
    if nprocs <= 0 or not 0 <= irank < nprocs:
        raise ValueError(f"rank {irank} outside 0..{nprocs - 1}")
    iwork1 = (n2 - n1 + 1) // nprocs
    iwork2 = (n2 - n1 + 1) % nprocs
    ista = irank * iwork1 + n1 + min(irank, iwork2)
    iend = ista + iwork1 - 1
    if iwork2 > irank:
        iend += 1
    return ista, iend


def rank_env() -> tuple[int, int, int]:
    """(rank, world_size, local_rank) from the launcher's environment."""
    g = os.environ.get
    return int(g("RANK", 0)), int(g("WORLD_SIZE", 1)), int(g("LOCAL_RANK", 0))


def rank_shots(nshot: int, per_rank: int, rank: int, world: int) -> list[int]:
    """0-based shot ids of this rank: the first `per_rank` shots of its
    para_range block of 1..nshot (wrapping inside the block if it is short)."""
    ista, iend = para_range(1, nshot, world, rank)
    if iend < ista:
        raise ValueError(f"rank {rank} of {world} has no shot of {nshot}")
    block = list(range(ista - 1, iend))
    return [block[k % len(block)] for k in range(per_rank)]


def init_group(world: int, timeout_s: float = 600.0):
    """gloo process group for the barrier and the timing max (None at world 1)."""
    if world <= 1:
        return None
    import torch.distributed as dist
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, value: float) -> float:
    """Largest `value` over all ranks (every rank calls it, in the same order)."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(dist, value: float) -> float:
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
