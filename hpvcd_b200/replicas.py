"""Multi-GPU replicas: one process per GPU, independent work per rank.

HEIF grid tiles, images and decode requests are independent (the reference
decodes grid tiles independently, lib.rs:1641), so the path shards without
any data-path collective: every rank decodes its own units and the only
communication is timing (a barrier around the timed region and the maximum
of the ranks' times).  Throughput = all ranks' units / the slowest rank's
time (weak scaling: per-rank work is fixed as ranks are added).
"""
from __future__ import annotations

import os


def dist_info() -> tuple[int, int, int]:
    """(rank, world size, local rank) from the torchrun environment."""
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def shard_units(n_units: int, rank: int, world: int) -> range:
    """Contiguous block of unit indices owned by `rank` (sizes differ by at
    most one); the blocks of all ranks partition range(n_units)."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("bad rank / world size")
    base, extra = divmod(n_units, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def _reduce(value: float, op: str, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks of the default process group (the
    value itself without one)."""
    return _reduce(value, "max", device)


def sum_over_ranks(value: float, device=None) -> float:
    return _reduce(value, "sum", device)


def whole_job_rate(local_units: float, local_seconds: float, device=None) -> float:
    """Units of all ranks per second of the slowest rank."""
    units = sum_over_ranks(local_units, device)
    seconds = max_over_ranks(local_seconds, device)
    return units / seconds if seconds > 0 else 0.0
