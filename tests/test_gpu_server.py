"""Serving loop: continuous batching, pattern cache, escalation, and the
same result alone and in a mix."""
import threading

import numpy as np
import pytest

from luspice_b200 import api, mna
from tests.helpers import TOL_REL, oracle_solution, rel_err

pytestmark = pytest.mark.gpu


def test_same_result_alone_and_in_mix(gpu):
    m = mna.analog(989, 42)
    vals = m.perturbed(1, seed=9)[0]
    S = api.Server(max_batch=64, streams=3, arena_gb=1.0, staging_mb=64)
    rid = S.submit(m.n, m.Ap, m.Ai, vals, m.b)
    x_alone, r_alone = S.poll(rid, 120000)
    assert r_alone["rc"] == 0 and r_alone["batch_size"] == 1
    # Now the same system among 60 others of 4 patterns, from two threads.
    others = [mna.analog(int(n), 100 + i) for i, n in enumerate([300, 1500, 700, 2500])]
    ids, lock = [], threading.Lock()

    def worker(k):
        for t in range(30):
            mm = others[(t + k) % len(others)]
            v = mm.perturbed(1, seed=1000 * k + t)[0]
            i = S.submit(mm.n, mm.Ap, mm.Ai, v, mm.b)
            with lock:
                ids.append((i, mm, v))
            if t == 15 and k == 0:
                j = S.submit(m.n, m.Ap, m.Ai, vals, m.b)
                with lock:
                    ids.append((j, None, None))

    th = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    mixed = None
    batch_sizes = []
    for i, mm, v in ids:
        x, r = S.poll(i, 120000)
        assert r["rc"] == 0, r
        batch_sizes.append(r["batch_size"])
        if mm is None:
            mixed = (x, r)
        else:
            assert r["residual"] <= 1e-10, r
            assert rel_err(x, oracle_solution(mm, v)) <= TOL_REL
    x_mixed, r_mixed = mixed
    assert np.array_equal(x_alone, x_mixed), (np.abs(x_alone - x_mixed).max(), r_alone, r_mixed)
    assert rel_err(x_mixed, oracle_solution(m, vals)) <= TOL_REL
    st = S.stats()
    assert st["cache_hits"] >= 55 and st["cache_misses"] == 5
    assert max(batch_sizes) > 1          # requests were batched together
    S.close()


def test_escalation_to_fp64(gpu):
    m = mna.analog(989, 42)
    bad = mna.ill_conditioned(m, seed=3)
    S = api.Server(max_batch=16, streams=2, arena_gb=0.5, staging_mb=32)
    i_ok = S.submit(m.n, m.Ap, m.Ai, m.Ax, m.b)
    i_bad = S.submit(m.n, m.Ap, m.Ai, bad, m.b)
    x_ok, r_ok = S.poll(i_ok, 120000)
    x_bad, r_bad = S.poll(i_bad, 120000)
    assert r_ok["rc"] == 0 and not r_ok["escalated"]
    assert rel_err(x_ok, m.x_true) <= TOL_REL
    assert r_bad["rc"] == 0
    from luspice_b200 import api as A
    if r_bad["escalated"]:
        assert r_bad["status"] & A.ST_ESCALATED
    # Whatever path it took, the answer is the fp64 oracle's.
    from luspice_b200.api import Pattern
    P = Pattern.from_matrix(m)
    _, q = P.perm()
    ref = oracle_solution(m, bad, q=q)
    r = np.linalg.norm(m.matvec(x_bad, bad) - m.b) / np.linalg.norm(m.b)
    r_ref = np.linalg.norm(m.matvec(ref, bad) - m.b) / np.linalg.norm(m.b)
    assert r <= max(10 * r_ref, 1e-9), (r, r_ref, r_bad)
    S.close()


def test_singular_pattern_reported(gpu):
    S = api.Server(max_batch=4, streams=1, arena_gb=0.25, staging_mb=16)
    Ap = np.array([0, 2, 4, 5], np.int32)
    Ai = np.array([0, 1, 0, 1, 2], np.int32)
    Ax = np.array([1.0, 2.0, 2.0, 4.0, 1.0])
    rid = S.submit(3, Ap, Ai, Ax, np.ones(3))
    _, r = S.poll(rid, 120000)
    assert r["rc"] == 1
    S.close()


def test_repivot_when_frozen_pivot_vanishes(gpu):
    """A Newton step whose value at a frozen pivot is zero (a column with no
    updates above its diagonal, so U(k,k) is that value): the mixed and fp64
    frozen-pivot factors are singular, so the server analyses the request
    again with its own values (fresh partial pivoting) and returns the fp64
    oracle's answer."""
    m = mna.analog(989, 42)
    q = api.colamd(m.n, m.Ap, m.Ai)
    f = api.pivot_factor(m.n, m.Ap, m.Ai, m.Ax, q)
    rowat = np.empty(m.n, np.int64)
    rowat[f["pinv"]] = np.arange(m.n)
    bad = None
    for k in range(m.n):
        c = q[k]
        if m.Ap[c + 1] - m.Ap[c] < 2 or f["Up"][k + 1] - f["Up"][k] != 1:
            continue
        col = np.arange(m.Ap[c], m.Ap[c + 1])
        bad = m.Ax.copy()
        bad[col[m.Ai[col] == rowat[k]][0]] = 0.0
        if api.pivot_factor(m.n, m.Ap, m.Ai, bad, q)["singular_col"] < 0:
            break
    assert bad is not None
    ref = oracle_solution(m, bad)
    S = api.Server(max_batch=8, streams=1, arena_gb=0.5, staging_mb=32)
    S.poll(S.submit(m.n, m.Ap, m.Ai, m.Ax, m.b), 120000)
    x, r = S.poll(S.submit(m.n, m.Ap, m.Ai, bad, m.b), 120000)
    assert r["rc"] == 0 and r["escalated"], r
    assert rel_err(x, ref) <= TOL_REL, (rel_err(x, ref), r)
    st = S.stats()
    assert st["patterns_resident"] == 1     # the request's own analysis is gone
    S.close()


def test_oversized_request_refused_others_served(gpu):
    """A request whose inputs exceed a stream's staging area completes at once
    with LUSP_EALLOC and the capacity status; requests around it are served."""
    small = mna.analog(300, 3)
    big = mna.large_circuit(3000, seed=5)
    S = api.Server(max_batch=8, streams=1, arena_gb=0.5, staging_mb=0.1)
    i0 = S.submit(small.n, small.Ap, small.Ai, small.Ax, small.b)
    i1 = S.submit(big.n, big.Ap, big.Ai, big.Ax, big.b)
    i2 = S.submit(small.n, small.Ap, small.Ai, small.Ax, small.b)
    _, r1 = S.poll(i1, 120000)
    assert r1["rc"] == 2 and r1["status"] & api.ST_CAPACITY, r1
    for i in (i0, i2):
        x, r = S.poll(i, 120000)
        assert r["rc"] == 0
        assert rel_err(x, oracle_solution(small, small.Ax)) <= TOL_REL
    S.close()


def test_many_concurrent_submitters(gpu):
    """Eight threads submit and poll their own requests over three patterns:
    every request completes with the oracle's answer and the counters add up."""
    mats = [mna.analog(n, 40 + n) for n in (200, 600, 1200)]
    S = api.Server(max_batch=32, streams=3, arena_gb=0.5, staging_mb=32)
    errors, lock = [], threading.Lock()

    def worker(k):
        for t in range(12):
            m = mats[(k + t) % 3]
            v = m.perturbed(1, seed=100 * k + t)[0]
            x, r = S.poll(S.submit(m.n, m.Ap, m.Ai, v, m.b), 120000)
            if r["rc"] != 0 or rel_err(x, oracle_solution(m, v)) > TOL_REL:
                with lock:
                    errors.append((k, t, r))

    th = [threading.Thread(target=worker, args=(k,)) for k in range(8)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors[:3]
    st = S.stats()
    assert st["submitted"] == st["completed"] == 96
    assert st["cache_misses"] == 3 and st["cache_hits"] == 93
    S.close()


def test_escalation_off_keeps_the_failed_result(gpu):
    """escalate = 0: a system whose mixed solve fails is returned as it is,
    with its failure status and no escalation."""
    m = mna.analog(989, 42)
    S = api.Server(max_batch=4, streams=1, arena_gb=0.5, staging_mb=32, escalate=0, rtol=1e-300)
    _, r = S.poll(S.submit(m.n, m.Ap, m.Ai, m.Ax, m.b), 120000)
    assert r["rc"] == 0 and not r["escalated"]
    assert r["status"] & (api.ST_NOT_CONVERGED | api.ST_STAGNATED)
    assert S.stats()["escalated"] == 0
    S.close()


def test_lru_eviction_and_reanalysis(gpu):
    """A pattern budget of a few MB beside the arena: older patterns leave the
    device, and a pattern seen again after its eviction is analysed again and
    still gives the oracle's answer."""
    mats = [mna.analog(1500, 60 + i) for i in range(6)]
    arena = 0.25
    S = api.Server(max_batch=4, streams=1, arena_gb=arena, staging_mb=32, hbm_budget_gb=arena + 0.004)
    for m in mats:
        x, r = S.poll(S.submit(m.n, m.Ap, m.Ai, m.Ax, m.b), 120000)
        assert r["rc"] == 0
    st = S.stats()
    assert st["evictions"] > 0 and st["pattern_gb"] <= 0.004 + 1e-9, st
    m = mats[0]
    v = m.perturbed(1, seed=3)[0]
    x, r = S.poll(S.submit(m.n, m.Ap, m.Ai, v, m.b), 120000)
    assert r["rc"] == 0 and not r["cache_hit"]
    assert rel_err(x, oracle_solution(m, v)) <= TOL_REL
    S.close()


def test_admission_refuses_pattern_above_budget(gpu):
    """HBM admission: with a pattern budget of a few MB beside the arena, a
    pattern whose device layout alone exceeds it (the n = 4050 power grid,
    ~14 MB) is refused with LUSP_EALLOC / CAPACITY, while small patterns
    submitted before and after it are served."""
    small = [mna.analog(300, 80 + i) for i in range(4)]
    big = mna.power_grid()
    arena = 0.25
    S = api.Server(max_batch=4, streams=1, arena_gb=arena, staging_mb=64, hbm_budget_gb=arena + 0.002)
    ids = [S.submit(m.n, m.Ap, m.Ai, m.Ax, m.b) for m in small[:2]]
    ib = S.submit(big.n, big.Ap, big.Ai, big.Ax, big.b)
    ids += [S.submit(m.n, m.Ap, m.Ai, m.Ax, m.b) for m in small[2:]]
    xb, rb = S.poll(ib, 120000)
    assert rb["rc"] == 2 and rb["status"] & api.ST_CAPACITY, rb   # LUSP_EALLOC
    for m, i in zip(small, ids):
        x, r = S.poll(i, 120000)
        assert r["rc"] == 0, r
        assert rel_err(x, oracle_solution(m, m.Ax)) <= TOL_REL
    st = S.stats()
    assert st["refused"] == 1 and st["pattern_gb"] <= 0.002 + 1e-9, st
    S.close()


def test_pattern_escalation_memory(gpu):
    """A pattern whose mixed requests keep escalating (supply-net values over
    15 decades, pivots frozen on the nominal values: fp32 inner products
    stagnate) starts its later requests on the fp64 factor + GMRES-IR path
    after two escalations in a row, with a mixed trial every 16th request.
    The server's counters equal a replay of that rule over the observed
    outcomes, the path is taken at least once, and every answer is the fp64
    oracle's."""
    m = mna.serving_class("supply", 1748, 726)
    vals = m.perturbed(24, seed=5)
    S = api.Server(max_batch=4, streams=1, arena_gb=0.5, staging_mb=32)
    x0, r0 = S.poll(S.submit(m.n, m.Ap, m.Ai, m.Ax, m.b), 120000)   # pivots from the nominal values
    assert r0["rc"] == 0
    res = []
    for v in vals:
        x, r = S.poll(S.submit(m.n, m.Ap, m.Ai, v, m.b), 120000)
        assert r["rc"] == 0, r
        res.append((x, r))
    st = S.stats()
    S.close()
    # Replay: the nominal request first, then the 24 in order.
    outcomes = [bool(r0["escalated"])] + [bool(r["escalated"]) for _, r in res]
    run, promoted, since, n_prom, n_fp64 = 0, False, 0, 0, 0
    for i, esc in enumerate(outcomes):
        trial = False
        if promoted and i > 0:
            since += 1
            if since >= 16:
                since, trial = 0, True
            else:
                n_fp64 += 1      # (it may still escalate: a re-pivot when the fp64 factor fails)
                continue
        if esc:
            run += 1
            if run >= 2 and not promoted:
                promoted, since, n_prom = True, 0, n_prom + 1
        else:
            run = 0
            if trial and promoted:
                promoted = False
    assert n_prom >= 1, outcomes
    assert st["promoted"] == n_prom and st["fp64_starts"] == n_fp64, (st, outcomes)
    from luspice_b200.api import Pattern
    _, q = Pattern.from_matrix(m).perm()
    for (x, r), v in zip(res, vals):
        assert rel_err(x, oracle_solution(m, v, q=q)) <= TOL_REL, r
