"""Multi-GPU runs as independent replicas.

The STZ path has no exchange step: every field (or every request) is coded by
one GPU from start to finish, so N GPUs run N replicas, one process per GPU,
and nothing on the data path crosses GPUs. The only cross-rank traffic is
bookkeeping: a barrier around timed regions and the max over ranks of each
rank's device time (the job is as slow as its slowest replica).

The functions take the process group from `torch.distributed`, so the same
code runs over NCCL on GPUs and over gloo on CPU.
"""
from __future__ import annotations

import os
from datetime import timedelta


def rank_env() -> tuple[int, int, int]:
    """(rank, local_rank, world_size) from the torchrun environment."""
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)),
            int(os.environ.get("WORLD_SIZE", 1)))


def init(backend: str = "nccl", timeout_s: float = 120.0, device=None) -> bool:
    """Join the process group when launched with WORLD_SIZE > 1.

    The rendezvous address defaults to 127.0.0.1; a short timeout makes a rank
    that never arrives end its peers' next collective with an error instead of
    a hang. Returns True when a group was created."""
    import torch.distributed as dist

    _, _, world = rank_env()
    if world <= 1 or dist.is_initialized():
        return False
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    kw = {"timeout": timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return True


def world_size() -> int:
    import torch.distributed as dist

    return dist.get_world_size() if dist.is_initialized() else 1


def barrier() -> None:
    import torch.distributed as dist

    if dist.is_initialized():
        dist.barrier()


def max_over_ranks(value: float, device="cpu") -> float:
    """Max of a per-rank scalar (a device time in ms) over all ranks."""
    import torch
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seed(base: int, rank: int) -> int:
    """Seed of the field a replica codes: distinct per rank."""
    return base + rank


def owned(n_items: int, rank: int, world: int) -> list[int]:
    """Items (fields, streams, requests) a replica owns: round-robin, disjoint,
    covering 0..n_items-1 over all ranks."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    return list(range(rank, n_items, world))


def aggregate_gbs(bytes_per_rank: float, world: int, ms: float) -> float:
    """Whole-job throughput: all ranks' bytes over the slowest rank's time."""
    if ms <= 0:
        raise ValueError("time must be positive")
    return world * bytes_per_rank / (ms / 1e3) / 1e9


def finalize() -> None:
    import torch.distributed as dist

    if dist.is_initialized():
        dist.destroy_process_group()
