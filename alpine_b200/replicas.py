"""Replica timing across ranks (weak scaling), for one process per GPU.

Rays and pixels are independent, so the multi-GPU form of the traversal and
render workloads is N independent replicas: every rank runs the whole
single-GPU workload on its own device, with no data-path collective. The job
is timed as the slowest rank (a max all-reduce of the per-step time) and its
work is the sum over ranks, so the job's rate is world x units per rank /
max time. Only rank 0 reports. The functions take the process group and the
device of the reduction tensor, so the same code runs with NCCL on GPUs and
with gloo on CPU.
"""
from __future__ import annotations

import os


def world_info():
    """(world size, rank, local rank) from the launcher's environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def max_over_ranks(x: float, dist=None, device="cpu") -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, ms_per_step: float, world: int, dist=None, device="cpu"):
    """(whole-job units per second, the job's ms per step): every rank does
    units_per_rank per step; the step takes as long as the slowest rank."""
    ms = max_over_ranks(ms_per_step, dist, device)
    return world * units_per_rank / (ms / 1e3), ms


def reports(rank: int) -> bool:
    """Whether this rank prints the result line (rank 0 only)."""
    return rank == 0
