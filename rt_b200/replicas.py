"""Replicas on one node: one process per GPU, each tracing its own rays.

Rays are independent, so `bench.py --gpus N` runs N replicas of the
workload (weak scaling) with no collective on the data path.  The only
communication is the timing: a barrier before each timed region, the
maximum of the ranks' device times and the sum of the ray-surfaces they
traced, so that the whole-job throughput is (sum of work) / (slowest rank).

Works with the NCCL backend on GPUs and with gloo on CPU (tests).
"""
from __future__ import annotations

import datetime
import os

SEED_STRIDE = 7919  # rank r draws its beams from seed + 7919 r


def env() -> tuple[int, int, int]:
    """(world size, rank, local rank) from the torchrun environment."""
    return (int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 120.0) -> tuple[int, int, int]:
    """Join the process group when there is more than one rank (NCCL: after
    selecting the local GPU).  A short timeout makes ranks that wait for a
    missing peer fail instead of hanging."""
    world, rank, local = env()
    if world > 1:
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return world, rank, local


def seed(base: int, rank: int) -> int:
    """The seed of rank `rank`'s beams: every replica traces different rays."""
    return base + SEED_STRIDE * rank


def _reduce(value: float, op: str, device) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(value: float, device="cuda") -> float:
    """The largest of the ranks' values (device times: the job's time)."""
    return _reduce(value, "max", device)


def sum_over_ranks(value: float, device="cuda") -> float:
    """The sum of the ranks' values (work done by the whole job)."""
    return _reduce(value, "sum", device)


def barrier() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.barrier()


def finish() -> None:
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        dist.destroy_process_group()
