"""Multi-GPU plumbing: one process per GPU, torch.distributed for the exchange.

Paths are independent, so a frame shards trivially: every rank renders the whole frame
with its own random streams (seed offset by the rank), the BVH replicated on each GPU, and
the linear accumulators are summed with one all-reduce per step.  The sum over ranks is the
estimate of a frame with world_size times the samples (weak scaling).  Timing is the
maximum over ranks.  NCCL over NVLink on GPUs; gloo on CPU tensors for tests.
"""
from __future__ import annotations

import datetime
import os
from dataclasses import dataclass


@dataclass
class Rank:
    world: int
    rank: int
    local: int
    backend: str | None

    @property
    def distributed(self) -> bool:
        return self.backend is not None


def init_from_env(prefer: str = "nccl", timeout_s: int = 120) -> Rank:
    """Joins the process group described by RANK / WORLD_SIZE / LOCAL_RANK / MASTER_*.
    A single process (WORLD_SIZE unset or 1) needs no process group."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return Rank(1, 0, local, None)
    import torch
    import torch.distributed as dist
    backend = prefer if (prefer != "nccl" or torch.cuda.is_available()) else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(local)
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return Rank(world, rank, local, backend)


def rank_seed(base_seed: int, rank: int) -> int:
    """Seed family of a rank: distinct PCG32 stream families per rank."""
    return int(base_seed) + int(rank)


def max_over_ranks(value: float, r: Rank) -> float:
    if not r.distributed:
        return float(value)
    import torch
    import torch.distributed as dist
    dev = "cuda" if r.backend == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def allreduce_sum_(tensors, r: Rank) -> None:
    """In-place sum over ranks of each tensor (framebuffer accumulators)."""
    if not r.distributed:
        return
    import torch.distributed as dist
    for t in tensors:
        dist.all_reduce(t)


def barrier(r: Rank) -> None:
    if r.distributed:
        import torch.distributed as dist
        dist.barrier()


def shutdown(r: Rank) -> None:
    if r.distributed:
        import torch.distributed as dist
        dist.destroy_process_group()


def weak_scaling_value(paths_per_rank_step: int, world: int, ms_per_step_max: float) -> float:
    """Whole-job Mpaths/s: all ranks' paths over the slowest rank's step time."""
    return world * paths_per_rank_step / (ms_per_step_max * 1e-3) / 1e6
