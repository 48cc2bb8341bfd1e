"""One process per GPU, each with its own replica of the index.

The search path has no exchange step: queries are independent and each GPU
holds the whole index, so N GPUs run N independent searches (weak scaling,
per-GPU batch fixed) or split one batch by queries (``shard``).  Results are
identical to one GPU's.  torch.distributed is used only to line the ranks up
(barrier) and to take the slowest rank's time (``max_over_ranks``); nothing
on the data path crosses GPUs.
"""
from __future__ import annotations

import datetime
import os


def world_info():
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str | None = None, timeout_s: float = 600.0):
    """Join the process group when WORLD_SIZE > 1; returns (world, rank, local_rank)."""
    world, rank, local = world_info()
    if world > 1:
        import torch
        import torch.distributed as dist

        if backend is None:
            backend = "nccl" if torch.cuda.is_available() else "gloo"
        kwargs = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kwargs["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kwargs)
    return world, rank, local


def _device():
    import torch
    import torch.distributed as dist

    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """The largest value of x over all ranks (the job's time is the slowest rank's)."""
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return float(x)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(x)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def shard(n: int, rank: int, world: int):
    """Contiguous [lo, hi) slice of n items for this rank; slices tile [0, n)."""
    per, extra = divmod(n, world)
    lo = rank * per + min(rank, extra)
    return lo, lo + per + (1 if rank < extra else 0)


def finish(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
