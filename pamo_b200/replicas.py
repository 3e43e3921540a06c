"""Replicas across GPUs: one process per GPU, no data exchange on the hot path.

A single mesh does not shard (a collapse round's independent set and the
whole-mesh intersection check are global), but meshes are independent.  So
several GPUs run replicas: each rank simplifies its own meshes, and the only
collectives are host-side bookkeeping -- agreeing on who takes which mesh and
taking the slowest rank's time.

    world, rank = init()                       # env:// rendezvous (torchrun)
    mine = my_share(sizes, rank, world)        # meshes of this rank
    t = max_over_ranks([local_seconds])[0]
"""
from __future__ import annotations

import datetime
import os


def init(backend: str | None = None, timeout_s: float = 120.0):
    """Joins the process group described by the torchrun environment (RANK,
    WORLD_SIZE, MASTER_ADDR, MASTER_PORT).  Returns (world, rank); a world of
    one needs no process group."""
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world > 1 and not dist.is_initialized():
        if backend is None:
            import torch

            backend = "nccl" if torch.cuda.is_available() else "gloo"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank


def max_over_ranks(values, device=None):
    """Element-wise maximum of `values` (floats) over all ranks."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def assign_by_footprint(sizes, world: int):
    """Rank of each item, balancing the summed sizes (faces, bytes): largest
    first, each to the least-loaded rank (lowest rank on ties).  Deterministic,
    so every rank computes the same assignment without communicating."""
    load = [0] * world
    owner = [0] * len(sizes)
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        owner[i] = r
        load[r] += int(sizes[i])
    return owner


def my_share(sizes, rank: int, world: int):
    """Indices of the items this rank takes, in input order."""
    owner = assign_by_footprint(sizes, world)
    return [i for i, r in enumerate(owner) if r == rank]


def finalize():
    import torch.distributed as dist

    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
