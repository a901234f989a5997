"""Measuring autotuner: the configuration it picks is one of its candidates,
runs correctly, and is no slower than the default rules (within timing
noise); the SELL tuner picks a valid (C, sigma)."""
import numpy as np
import pytest

from luspice_b200 import api, mna
from tests.helpers import TOL_REL, oracle_solution, rel_err

pytestmark = pytest.mark.gpu


def _launch_ms(P, nsys, vals, b, **opts):
    import torch
    B = api.Batch([P] * nsys, prec=api.MIXED, **opts)
    B.upload(list(vals), [b] * nsys)
    B.run(api.RUN_BOTH)
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 1e30
    for _ in range(3):
        a.record()
        B.run(api.RUN_BOTH)
        e.record()
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(e))
    xs = B.split(B.download())
    B.close()
    return best, xs


def test_tune_power_grid(gpu):
    m = mna.power_grid()
    nsys = 8
    t = api.autotune(m, nsys)
    assert 0 <= t["dense_tail"] <= 768 and t["ms"] > 0
    # 0, 0: the engine's own refactor rules (spread mode for this batch).
    assert t["opts"]["refactor_cluster"] in (0, 1, 2) and t["opts"]["block_threads"] in (256, 512)
    assert t["opts"]["refactor_threads"] in (0, 512, 768, 1024)
    assert (t["opts"]["refactor_threads"] == 0) == (t["opts"]["refactor_cluster"] == 0)
    assert t["opts"]["solve_sweep"] in (0, 1)
    vals = m.perturbed(nsys, seed=77)
    P = api.Pattern.from_matrix(m, dense_tail=t["dense_tail"])
    tuned, xs = _launch_ms(P, nsys, vals, m.b, **t["opts"])
    _, q = P.perm()
    for s in range(nsys):
        assert rel_err(xs[s], oracle_solution(m, vals[s], q=q)) <= TOL_REL
    default, _ = _launch_ms(api.Pattern.from_matrix(m), nsys, vals, m.b)
    assert tuned <= 1.25 * default, (tuned, default, t)


def test_sell_tune(gpu):
    m = mna.analog(3000, 9)
    A = m.csr()
    r = api.sell_tune(m.n, A.indptr, A.indices, A.data, "fp32")
    assert r["C"] in (8, 16, 32) and r["sigma"] in (32, 256, 1024) and r["us"] > 0
