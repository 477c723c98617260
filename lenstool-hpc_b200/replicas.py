"""Independent replicas, one process per GPU (launched by torchrun).

Maps, posterior sets and chi2 models are independent, so nothing on the data path crosses
ranks: each rank evaluates its own copy of the workload on its own GPU.  The only
collectives are a barrier on both sides of a timed region and the maximum over ranks of
its duration; a rate is the units of all ranks divided by that maximum (weak scaling).
The reference has no multi-GPU map path (its MPI split is for chi2 rows,
src/chi_CPU_barycenter.cpp:91-101).
"""
from __future__ import annotations

import datetime
import os


def env():
    """(rank, local_rank, world_size) from the torchrun environment."""
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> int:
    """Join the process group when world_size > 1 (a short timeout, so that ranks waiting
    for a missing peer end with an error); returns the world size."""
    import torch.distributed as dist
    _, _, world = env()
    if world > 1 and not dist.is_initialized():
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world


def barrier(sync=None) -> None:
    """All ranks meet; `sync` (e.g. torch.cuda.synchronize) then drains this rank's device."""
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()
    if sync is not None:
        sync()


def _reduce(x: float, op: str, device: str) -> float:
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized():
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(seconds: float, device: str = "cpu") -> float:
    return _reduce(seconds, "max", device)


def sum_over_ranks(units: float, device: str = "cpu") -> float:
    return _reduce(units, "sum", device)


def throughput(units: float, seconds: float, device: str = "cpu"):
    """Whole-job rate: the units of all ranks over the slowest rank's time.  Every rank
    takes both collectives in the same order.  Returns (rate, max_seconds, total_units)."""
    tmax = max_over_ranks(seconds, device)
    total = sum_over_ranks(units, device)
    return total / tmax, tmax, total


def finalize() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
