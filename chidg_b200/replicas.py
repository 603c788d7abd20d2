"""Replica (data-parallel) plumbing for independent solves on several GPUs.

The linear-solve path does not shard: every rank owns whole, independent
solves, so there is no data-path collective.  Ranks only meet for the timing
harness: a barrier on both sides of the timed region and the maximum of the
per-rank elapsed times.  The functions work with any torch.distributed
backend ("nccl" on GPUs, "gloo" in the CPU tests).
"""
from __future__ import annotations

import datetime
import os


def init_from_env(backend: str = "nccl", timeout_s: int = 600):
    """Initialise torch.distributed from RANK/WORLD_SIZE/MASTER_* when WORLD_SIZE > 1.

    Returns (rank, world_size, local_rank, dist or None)."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world <= 1:
        return rank, world, local, None
    import torch.distributed as dist
    if backend == "nccl":
        import torch
        torch.cuda.set_device(local)
    if not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return rank, world, local, dist


def barrier(dist, local: int | None = None):
    if dist is None:
        return
    if dist.get_backend() == "nccl":
        import torch
        dist.barrier(device_ids=[local])
        torch.cuda.synchronize()
    else:
        dist.barrier()


def allmax(dist, value: float, local: int | None = None) -> float:
    """Maximum of a per-rank float over all ranks (the job's elapsed time)."""
    if dist is None:
        return float(value)
    import torch
    dev = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def split_work(n_items: int, rank: int, world: int):
    """Contiguous share of n_items independent solves owned by `rank`."""
    base, extra = divmod(n_items, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def aggregate_throughput(units_per_rank: list, elapsed_max_s: float) -> float:
    """Whole-job throughput: all units processed by all ranks over the slowest rank's time."""
    return float(sum(units_per_rank)) / elapsed_max_s
