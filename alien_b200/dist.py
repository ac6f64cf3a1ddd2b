"""Multi-process plumbing for running independent systems on several GPUs.

The path shards by independent systems (one per rank, weak scaling): no
collective touches the data path.  torch.distributed only synchronises the
ranks around a timed region and combines their timings -- NCCL on GPUs, gloo
on CPU (the tests run two gloo ranks).  Ranks are read from the environment
torchrun sets (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR/PORT).
"""
from __future__ import annotations

import datetime
import os


def ranks() -> tuple[int, int, int]:
    """(world, rank, local_rank) from the environment (1, 0, 0 without torchrun)."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: int = 600) -> tuple[int, int, int]:
    """Joins the process group when WORLD_SIZE > 1 and returns (world, rank, local_rank)."""
    world, rank, local = ranks()
    if world > 1:
        import torch
        import torch.distributed as dist

        kw = {}
        if backend == "nccl":
            torch.cuda.set_device(local)
            kw["device_id"] = torch.device("cuda", local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
    return world, rank, local


def _device():
    import torch
    import torch.distributed as dist

    return torch.device("cuda") if dist.get_backend() == "nccl" else torch.device("cpu")


def barrier(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def reduce_max(world: int, value: float) -> float:
    """The largest value over all ranks (the step time a multi-GPU run reports)."""
    return _reduce(world, value, "max")


def reduce_sum(world: int, value: float) -> float:
    return _reduce(world, value, "sum")


def _reduce(world: int, value: float, op: str) -> float:
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(value)], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def finish(world: int) -> None:
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
