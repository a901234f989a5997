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


def structure_key(n: int, Ap, Ai) -> int:
    """Stable 64-bit key of a sparsity pattern (n, column pointers, row
    indices), the same on every rank and in every process."""
    import hashlib

    import numpy as np

    h = hashlib.blake2b(digest_size=8)
    h.update(int(n).to_bytes(8, "little"))
    h.update(np.ascontiguousarray(Ap, dtype=np.int32).tobytes())
    h.update(np.ascontiguousarray(Ai, dtype=np.int32).tobytes())
    return int.from_bytes(h.digest(), "little")


class ShardedServer:
    """Serving across ranks: a request may be submitted on any rank; it is
    solved by its pattern's owner rank (rank_of of the pattern key), so a
    pattern's analysis, levels and factors live on exactly one GPU, and its
    result goes back to the rank that submitted it.

    backend: this rank's server (api.Server, or any object with the same
    submit(n, Ap, Ai, Ax, b) -> id and poll(id, wait_ms) -> (x, result)
    calls).  Requests move between ranks in rounds: serve_round() is a
    collective (every rank calls it, with its own, possibly empty, list);
    the exchange is host-side object passing over the process group, never
    a device collective on the data path."""

    def __init__(self, backend, world: int, rank: int):
        self.backend = backend
        self.world = max(1, int(world))
        self.rank = int(rank)
        self.served = 0                      # requests this rank's backend solved

    def _exchange(self, outgoing: list):
        """outgoing[r]: objects for rank r; returns the objects every rank
        sent to this one (in rank order)."""
        if self.world <= 1:
            return [outgoing[0]]
        import torch.distributed as dist

        everything = [None] * self.world
        dist.all_gather_object(everything, outgoing)
        return [everything[src][self.rank] for src in range(self.world)]

    def serve_round(self, requests: list, wait_ms: int = 600000) -> dict:
        """requests: [(request id, n, Ap, Ai, Ax, b)] submitted on this rank
        (ids unique across ranks).  Returns {request id: (x, result, owner
        rank)} for them, after every rank's requests were served by their
        owners."""
        outgoing = [[] for _ in range(self.world)]
        for req in requests:
            rid, n, Ap, Ai, Ax, b = req
            owner = rank_of(structure_key(n, Ap, Ai), self.world)
            outgoing[owner].append((self.rank, req))
        incoming = [item for part in self._exchange(outgoing) for item in part]
        # Submit everything this rank owns, then collect (the backend batches
        # whatever is ready together).
        handles = [(origin, req[0], self.backend.submit(*req[1:])) for origin, req in incoming]
        replies = [[] for _ in range(self.world)]
        for origin, rid, h in handles:
            x, res = self.backend.poll(h, wait_ms)
            replies[origin].append((rid, x, res, self.rank))
            self.served += 1
        back = [item for part in self._exchange(replies) for item in part]
        return {rid: (x, res, owner) for rid, x, res, owner in back}
