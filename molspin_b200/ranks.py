"""Rank coordination for runs over several GPUs of one node.

One process per GPU (launched by torch.distributed.run; RANK, LOCAL_RANK,
WORLD_SIZE and MASTER_* from the environment).  Trajectories, orientations
and requests are independent, so every rank propagates its own trajectory
block with no collective in the data path (weak scaling); the process group
only serves the barrier around the timed region and the max over ranks of
the elapsed time.  NCCL on GPUs, gloo on the CPU (the tests).
"""
from __future__ import annotations

import os
from datetime import timedelta


def init(backend: str | None = None, timeout_s: int = 600) -> tuple[int, int, int]:
    """(world, rank, local rank); starts the process group when world > 1 and
    selects this rank's GPU when CUDA is available."""
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        be = backend or ("nccl" if torch.cuda.is_available() else "gloo")
        dist.init_process_group(be, timeout=timedelta(seconds=timeout_s))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def _device():
    import torch
    import torch.distributed as dist
    if dist.is_initialized() and dist.get_backend() == "nccl":
        return "cuda"
    return "cpu"


def barrier(world: int) -> None:
    """All ranks here, and this rank's device idle."""
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def max_over_ranks(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def block_seed(base: float, rank: int) -> float:
    """Seed of a rank's trajectory block: the blocks are disjoint samples."""
    return float(base) + rank


def aggregate(units_per_rank: float, world: int, elapsed_max_s: float) -> float:
    """Whole-job throughput of a weak-scaling run: every rank's units over the
    slowest rank's time."""
    return world * units_per_rank / elapsed_max_s


def finish(world: int) -> None:
    if world > 1:
        import torch.distributed as dist
        if dist.is_initialized():
            dist.destroy_process_group()
