"""One process per GPU without a data-path collective ("replicas only").

A single scenario is not decomposed across GPUs: every rank runs its own replica, or its own
share of an ensemble's members. The only communication is the timing protocol of the
benchmark (a barrier before and after the timed region, the maximum of the per-rank times) and
a final host-side gather of per-rank results. Works with the "nccl" backend on GPUs and "gloo"
on CPUs (the tests run two gloo ranks).
"""
from __future__ import annotations

import datetime
import os


def world() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment (0, 1, 0 without it)."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def init(backend: str = "nccl", timeout_s: float = 300.0):
    """Process group of a multi-rank run (None for a single rank). A short timeout makes ranks
    that wait for a lost peer fail instead of hanging."""
    _, n, _ = world()
    if n <= 1:
        return None
    import torch.distributed as dist

    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def partition(n_items: int, rank: int, n_ranks: int) -> range:
    """Contiguous share of rank `rank` of n_items (sizes differ by at most one)."""
    lo = n_items * rank // n_ranks
    hi = n_items * (rank + 1) // n_ranks
    return range(lo, hi)


def max_over_ranks(dist, value: float, device=None) -> float:
    """Maximum of a per-rank scalar (the slowest rank's time)."""
    if dist is None:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def gather_to_root(dist, obj):
    """Per-rank Python objects collected on rank 0 (None elsewhere)."""
    if dist is None:
        return [obj]
    out = [None] * dist.get_world_size() if dist.get_rank() == 0 else None
    dist.gather_object(obj, out, dst=0)
    return out


def barrier(dist) -> None:
    if dist is not None:
        dist.barrier()


def finish(dist) -> None:
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
