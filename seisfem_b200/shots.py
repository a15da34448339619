"""Shot sharding across ranks (one process per GPU).

Shots are independent (elastic_wave.c:446 loops over them serially, every
shot restarting from a zero state), so a multi-GPU run gives each rank a
contiguous slice of the shot list, runs it with no communication inside the
time loop, and collects the seismograms once at the end with one collective
on device tensors (NCCL over NVLink between GPUs; gloo in the CPU tests).
"""
from __future__ import annotations

import copy

import numpy as np


def shard(n_shots: int, rank: int, world: int) -> slice:
    """Contiguous block of shot indices for `rank`: the first n % world ranks
    get one extra shot."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_shots, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


def shard_problem(prob, rank: int, world: int):
    """The problem restricted to this rank's shots (a shallow copy)."""
    mine = shard(len(prob.src_node), rank, world)
    q = copy.copy(prob)
    q.src_node = np.ascontiguousarray(prob.src_node[mine], np.int32)
    return q


def gather_seismograms_device(local, n_shots: int, rank: int, world: int, group=None):
    """Every rank's [shots][rows][receivers] tensor, concatenated in shot
    order, on every rank: one all_gather of equal-size blocks (each rank's
    block padded to the largest shard), then the padding dropped.  `local`
    lives where the process group's backend moves data (CUDA tensors for
    NCCL, CPU tensors for gloo)."""
    import torch
    import torch.distributed as dist

    if world == 1:
        return local
    mine = shard(n_shots, rank, world)
    if local.shape[0] != mine.stop - mine.start:
        raise ValueError(f"rank {rank} holds {local.shape[0]} shots, its shard has {mine.stop - mine.start}")
    per = -(-n_shots // world)
    block = torch.zeros((per,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    block[:local.shape[0]] = local
    out = torch.empty((world * per,) + tuple(local.shape[1:]), dtype=local.dtype, device=local.device)
    dist.all_gather_into_tensor(out, block, group=group)
    keep = [r * per + k for r in range(world) for k in range(shard(n_shots, r, world).stop - shard(n_shots, r, world).start)]
    return out[torch.tensor(keep, device=local.device)]


def run_sharded(prob, rank: int, world: int, runner, group=None):
    """Run this rank's shots of `prob` with `runner(sub_problem) -> (seis_u,
    seis_w)` (tensors [shots][step-2][receivers]) and return every shot's
    seismograms on every rank, in the problem's shot order."""
    sub = shard_problem(prob, rank, world)
    su, sw = runner(sub)
    n = len(prob.src_node)
    return (gather_seismograms_device(su, n, rank, world, group),
            gather_seismograms_device(sw, n, rank, world, group))


def gather_seismograms(local: np.ndarray, n_shots: int, rank: int, world: int, group=None) -> np.ndarray | None:
    """Host-array variant: collect every rank's [shots][rows][receivers]
    block on rank 0 (shot order restored); returns None on other ranks.
    Goes through gather_seismograms_device with CPU tensors, so it needs a
    process group whose backend moves CPU tensors (gloo)."""
    import torch

    if world == 1:
        return local
    full = gather_seismograms_device(torch.from_numpy(np.ascontiguousarray(local)), n_shots, rank, world, group)
    return full.numpy() if rank == 0 else None
