"""Multi-process layout on CPU (gloo, world size 2): requests partitioned by
pattern hash across ranks with no data-path collective, results collected
on rank 0, timings reduced by max over ranks; serving requests routed to
their pattern's owner rank through shard.ShardedServer.

The CPU ranks have no GPU, so the per-rank server behind ShardedServer is a
stand-in with the serving loop's submit/poll interface that solves with the
compiled reference (on a GPU rank it is api.Server); the routing, the
exchange between ranks and the collection are the product's."""
import os
import socket
import zlib

import numpy as np
import pytest
import torch.multiprocessing as mp

from luspice_b200 import mna, shard


def _requests():
    sizes = [60, 90, 120, 75, 150, 80, 110, 95]
    return [(i, mna.analog(n, 500 + i)) for i, n in enumerate(sizes)]


def _key(req):
    m = req[1]
    return zlib.crc32(m.Ap.tobytes() + m.Ai.tobytes())


def _solve(m):
    from oracle import oracle
    return oracle.ref_cpu_solve(m.n, m.Ap, m.Ai, m.Ax, None, m.b)


def _worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        mine = shard.partition(_requests(), _key, world, rank)
        local = {i: _solve(m) for i, m in mine}
        merged = shard.collect(local, world)
        t = shard.max_over_ranks(float(rank + 1), world)
        q.put((rank, sorted(local), None if merged is None else {k: v.tolist() for k, v in merged.items()}, t))
    finally:
        dist.destroy_process_group()


def _port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_is_a_stable_cover():
    reqs = _requests()
    for world in (1, 2, 3, 8):
        owned = [shard.partition(reqs, _key, world, r) for r in range(world)]
        ids = sorted(i for part in owned for i, _ in part)
        assert ids == list(range(len(reqs)))
        assert [shard.rank_of(_key(r), world) for r in reqs] == [shard.rank_of(_key(r), world) for r in reqs]


def test_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, local_ids, merged, t = q.get(timeout=120)
        out[rank] = (local_ids, merged, t)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # Every request solved exactly once, by its owner.
    assert sorted(out[0][0] + out[1][0]) == list(range(len(_requests())))
    assert set(out[0][0]).isdisjoint(out[1][0])
    assert out[1][1] is None and out[0][1] is not None
    # Rank 0's collection equals a single-process run; timing is the max.
    single = {i: _solve(m) for i, m in _requests()}
    assert sorted(out[0][1]) == sorted(single)
    for i, x in single.items():
        assert np.array_equal(np.asarray(out[0][1][i]), x)
    assert out[0][2] == out[1][2] == 2.0


class HostServer:
    """Stand-in per-rank server (api.Server's submit/poll interface): solves
    each request with the reference's CPU path and records what it served."""

    def __init__(self):
        self.pending = {}
        self.served = []
        self.next = 0

    def submit(self, n, Ap, Ai, Ax, b):
        h = self.next
        self.next += 1
        self.pending[h] = (n, Ap, Ai, Ax, b)
        return h

    def poll(self, h, wait_ms=-1):
        from oracle import oracle
        n, Ap, Ai, Ax, b = self.pending.pop(h)
        self.served.append(shard.structure_key(n, Ap, Ai))
        return oracle.ref_cpu_solve(n, Ap, Ai, Ax, None, b), {"rc": 0}


def _serving_requests(rank):
    """Rank r submits Newton steps of every pattern class (ids unique across
    ranks): the owners of half the classes are the other rank."""
    out = []
    for i, (_, m) in enumerate(_requests()):
        for s in range(2):
            rid = 1000 * rank + 10 * i + s
            v = m.perturbed(1, seed=rid)[0]
            out.append((rid, m.n, m.Ap, m.Ai, v, m.b))
    return out


def _serve_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        backend = HostServer()
        srv = shard.ShardedServer(backend, world, rank)
        mine = _serving_requests(rank)
        got = srv.serve_round(mine)
        owners = {rid: owner for rid, (_, _, owner) in got.items()}
        merged = shard.collect({rid: x.tolist() for rid, (x, _, _) in got.items()}, world)
        q.put((rank, sorted(r[0] for r in mine), sorted(got), owners, backend.served, merged))
    finally:
        dist.destroy_process_group()


def test_two_ranks_serving_routes_to_owner():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _port()
    procs = [ctx.Process(target=_serve_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(2):
        rank, submitted, returned, owners, served, merged = q.get(timeout=180)
        out[rank] = (submitted, returned, owners, served, merged)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    reqs = {r[0]: r for rank in (0, 1) for r in _serving_requests(rank)}
    for rank in (0, 1):
        submitted, returned, owners, served, _ = out[rank]
        # Each rank gets back exactly the results of the requests it submitted.
        assert submitted == returned
        # Each result was computed by the owner of its pattern ...
        for rid, owner in owners.items():
            r = reqs[rid]
            assert owner == shard.rank_of(shard.structure_key(r[1], r[2], r[3]), 2)
        # ... and each rank's server solved only patterns it owns.
        assert all(shard.rank_of(k, 2) == rank for k in served)
    # Every request served exactly once across the ranks, both ranks busy.
    assert len(out[0][3]) + len(out[1][3]) == len(reqs)
    assert len(out[0][3]) > 0 and len(out[1][3]) > 0
    # Rank 0's collection equals a single-process run through the same path.
    single = shard.ShardedServer(HostServer(), 1, 0).serve_round(list(reqs.values()))
    merged = out[0][4]
    assert out[1][4] is None and sorted(merged) == sorted(single)
    for rid, (x, _, owner) in single.items():
        assert owner == 0
        assert np.array_equal(np.asarray(merged[rid]), x)
