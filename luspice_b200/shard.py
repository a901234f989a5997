"""Multi-GPU layout of the refactor-and-solve path: one process per GPU.

Every matrix (and every Newton refactorization of it) is an independent
unit with no exchange step, so N GPUs run N independent engines: requests
are partitioned by pattern hash (a pattern's analysis, levels and factors
then stay resident on exactly one GPU), and the only communication is the
optional host-side collection of results on rank 0.  No collective touches
the data path.
"""
from __future__ import annotations

from typing import Callable, Iterable, Sequence, TypeVar

T = TypeVar("T")

_MIX = 0x9E3779B97F4A7C15


def rank_of(pattern_hash: int, world: int) -> int:
    """Owner rank of a pattern: a fixed mix of its 64-bit hash, modulo the
    world size (stable across runs and processes)."""
    if world <= 1:
        return 0
    h = (int(pattern_hash) * _MIX) & 0xFFFFFFFFFFFFFFFF
    h ^= h >> 29
    return int(h % world)


def partition(items: Iterable[T], key: Callable[[T], int], world: int, rank: int) -> list[T]:
    """The items this rank owns, in their original order."""
    return [it for it in items if rank_of(key(it), world) == rank]


def collect(local: dict, world: int, dst: int = 0) -> dict | None:
    """Merge per-rank {request id: result} dicts on rank dst (host-side
    gather over the process group); None on the other ranks.  Raises if a
    request id was produced by two ranks."""
    if world <= 1:
        return dict(local)
    import torch.distributed as dist

    rank = dist.get_rank()
    parts: Sequence[dict] | None = [None] * world if rank == dst else None
    dist.gather_object(local, parts, dst=dst)
    if rank != dst:
        return None
    merged: dict = {}
    for p in parts:
        for k, v in p.items():
            if k in merged:
                raise RuntimeError(f"request {k!r} produced by two ranks")
            merged[k] = v
    return merged


def max_over_ranks(value: float, world: int) -> float:
    """Maximum of a per-rank timing over the process group."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
