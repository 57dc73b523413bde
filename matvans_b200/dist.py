"""Multi-GPU plumbing for replicated runs (one process per GPU).

The entropy-coded matvec shards naturally (independent rows, independent
matrices) and needs no collective on its data path; N GPUs run N independent
replicas of a workload.  This module holds the host side of that: process-group
set-up from the torchrun environment, and the max-over-ranks timing with the
whole-job throughput that bench.py reports.  It works with "nccl" on GPUs and
with "gloo" on CPU (which is how the tests exercise it).
"""
import os
from datetime import timedelta

import torch
import torch.distributed as dist


def env_rank():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend="nccl", timeout_s=120, device=None):
    """Join the process group described by RANK/WORLD_SIZE/MASTER_* (no-op for one process)."""
    rank, world, _ = env_rank()
    if world > 1 and not dist.is_initialized():
        kw = {"timeout": timedelta(seconds=timeout_s)}
        if device is not None and backend == "nccl":
            kw["device_id"] = device
        dist.init_process_group(backend, **kw)
    return rank, world


def barrier():
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def max_over_ranks(value, device=None):
    """The maximum of a per-rank float over all ranks (the job is as slow as its slowest rank)."""
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_throughput(units_per_rank, seconds_per_rank, device=None):
    """Whole-job throughput of a replicated run: every rank processes units_per_rank
    units; the job time is the slowest rank's time."""
    world = dist.get_world_size() if (dist.is_available() and dist.is_initialized()) else 1
    t = max_over_ranks(seconds_per_rank, device)
    return world * units_per_rank / t, t


def shard_rows(rows, rank, world):
    """Contiguous row range [r0, r1) of a rank when one matrix is row-sharded
    (32-row stripe granularity, so every shard is a whole number of stripes)."""
    stripes = (rows + 31) // 32
    per = (stripes + world - 1) // world
    r0 = min(rows, rank * per * 32)
    r1 = min(rows, (rank + 1) * per * 32)
    return r0, r1


def shutdown():
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
