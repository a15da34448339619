"""Shot sharding across ranks (one process per GPU).

Shots are independent (elastic_wave.c:446 loops over them serially, every
shot restarting from a zero state), so a multi-GPU run gives each rank a
contiguous slice of the shot list, runs it with no communication inside the
time loop, and collects the seismograms once at the end.
"""
from __future__ import annotations

import numpy as np


def shard(n_shots: int, rank: int, world: int) -> slice:
    """Contiguous block of shot indices for `rank`: the first n % world ranks
    get one extra shot."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_shots, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def gather_seismograms(local: np.ndarray, n_shots: int, rank: int, world: int, group=None) -> np.ndarray | None:
    """Collect every rank's [shots][rows][receivers] block on rank 0 (shot
    order restored).  Uses torch.distributed (NCCL on GPUs, gloo on CPU);
    returns the full array on rank 0 and None elsewhere."""
    import torch
    import torch.distributed as dist

    if world == 1:
        return local
    parts = [None] * world if rank == 0 else None
    dist.gather_object(local, parts, dst=0, group=group)
    if rank != 0:
        return None
    full = np.concatenate(parts, axis=0)
    if full.shape[0] != n_shots:
        raise RuntimeError(f"gathered {full.shape[0]} shots, expected {n_shots}")
    return full
