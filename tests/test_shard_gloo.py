"""Multi-process layout on CPU (gloo, world size 2): requests partitioned by
pattern hash across ranks with no data-path collective, results collected
on rank 0, timings reduced by max over ranks."""
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
