"""Host logic of multi-GPU bench runs.

One process per GPU (torchrun).  The reference shards each build round's batch
over MPI ranks that exchange their new out-lists (src/bsp_index.hpp:247-252,
include/bsp/broadcast_bsp_framework.cpp:166-218).  Here each rank builds an
independent partition of the same size (a differently seeded copy of the
workload) with no data-path exchange, so per-GPU work is fixed as ranks are
added (weak scaling).  The job is timed as the maximum of the ranks' device
times, and its rate counts the points of every rank.
"""
from __future__ import annotations

import dataclasses
import os


def rank_workload(w, rank: int):
    """The partition of `rank`: the same shape, a seed of its own."""
    return dataclasses.replace(w, seed=w.seed + 1000 * int(rank))


def gpu_index(local_rank: int, env=None) -> str:
    """nvidia-smi index of the GPU a local rank drives (CUDA_VISIBLE_DEVICES
    maps local ranks to physical GPUs when set)."""
    env = os.environ if env is None else env
    vis = [p.strip() for p in env.get("CUDA_VISIBLE_DEVICES", "").split(",") if p.strip()]
    if local_rank < len(vis):
        return vis[local_rank]
    return str(local_rank)


def max_over_ranks(x: float, device, distributed: bool) -> float:
    """Maximum of x over all ranks (x itself on a single rank)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if distributed:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, n: int, steps: int, t_max: float) -> float:
    """Points per second of the whole job: every rank inserts n points per step."""
    return world * n * steps / t_max
