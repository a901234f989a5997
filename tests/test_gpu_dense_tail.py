"""Dense trailing block: the last D columns/rows refactored and solved as one
dense block.  The factor values must not depend on D (bitwise equal to the
oracle for every D, including no tail and an all-dense matrix), and the
solves must reach the fp64 oracle solution."""
import numpy as np
import pytest

from luspice_b200 import api, mna
from tests.helpers import TOL_REL, oracle_refactor, oracle_solution, rel_err, rel_res, small_problems

pytestmark = pytest.mark.gpu


def _bitwise(got, exp):
    exp = exp.astype(got.dtype)
    ity = np.uint32 if got.dtype == np.float32 else np.uint64
    return np.flatnonzero(got.view(ity) != exp.view(ity))


@pytest.mark.parametrize("prec", [api.MIXED, api.FP64])
@pytest.mark.parametrize("tail", [0, 17, 64, 200, -1])
def test_tail_refactor_bitwise(gpu, prec, tail):
    m = small_problems()[1]
    P = api.Pattern.from_matrix(m, dense_tail=tail)
    info = P.info
    if tail >= 0:
        assert info["dense_tail"] == min(tail, m.n)
    assert info["tail_start"] == m.n - info["dense_tail"]
    vals = m.perturbed(3, seed=31)
    B = api.Batch([P] * 3, prec=prec)
    B.upload(list(vals), [m.b] * 3)
    B.run(api.RUN_BOTH)
    st = B.stats()
    xs = B.split(B.download())
    _, q = P.perm()
    for s in range(3):
        exp, bad = oracle_refactor(m, P, vals[s], fp32=(prec == api.MIXED))
        assert bad < 0
        mism = _bitwise(B.factor_values(s), exp)
        assert mism.size == 0, f"tail {tail} system {s}: {mism.size} slots differ, first {mism[:5]}"
        assert st[s]["status"] & api.ST_FAIL_MASK == 0, st[s]
        assert rel_err(xs[s], oracle_solution(m, vals[s], q=q)) <= TOL_REL


def test_tail_stats_match_no_tail(gpu):
    """Pivot statistics are the same with and without the dense block."""
    m = mna.power_grid()
    vals = m.perturbed(2, seed=3)
    res = []
    for tail in (0, -1):
        P = api.Pattern.from_matrix(m, dense_tail=tail)
        B = api.Batch([P] * 2, prec=api.MIXED)
        B.upload(list(vals), [m.b] * 2)
        B.run(api.RUN_REFACTOR)
        res.append((P.info["dense_tail"], [B.factor_values(s) for s in range(2)], B.stats()))
    assert res[0][0] == 0 and res[1][0] > 0, "the cost model picks a dense block for the mesh"
    for s in range(2):
        assert np.array_equal(res[0][1][s].view(np.uint32), res[1][1][s].view(np.uint32))
        for k in ("min_abs_pivot", "min_pivot_ratio", "max_abs_u"):
            assert res[0][2][s][k] == res[1][2][s][k], (k, res[0][2][s][k], res[1][2][s][k])


@pytest.mark.parametrize("sweep", [1, 2])
def test_tail_solves_both_sweeps(gpu, sweep):
    """Dataflow and level-synchronous sparse sweeps around the dense block."""
    m = mna.power_grid()
    P = api.Pattern.from_matrix(m)
    assert P.info["dense_tail"] > 0
    vals = m.perturbed(2, seed=8)
    for prec in (api.MIXED, api.FP64):
        B = api.Batch([P] * 2, prec=prec, solve_sweep=sweep)
        B.upload(list(vals), [m.b] * 2)
        B.run(api.RUN_BOTH)
        xs = B.split(B.download())
        _, q = P.perm()
        for s in range(2):
            assert rel_err(xs[s], oracle_solution(m, vals[s], q=q)) <= TOL_REL
            assert rel_res(m, vals[s], xs[s], m.b) <= 1e-9


def test_all_dense_and_mixed_tails_in_one_launch(gpu):
    """Patterns with no tail, a partial tail and an all-dense matrix share a
    launch; each system's factor equals the oracle's."""
    ms = [mna.analog(120, 5), mna.analog(700, 6), mna.analog(400, 7)]
    pats = [api.Pattern.from_matrix(ms[0], dense_tail=120), api.Pattern.from_matrix(ms[1], dense_tail=0),
            api.Pattern.from_matrix(ms[2], dense_tail=96)]
    assert pats[0].info["tail_start"] == 0
    B = api.Batch(pats, prec=api.MIXED)
    B.upload([m.Ax for m in ms], [m.b for m in ms])
    B.run(api.RUN_BOTH)
    xs = B.split(B.download())
    st = B.stats()
    for s, (m, P) in enumerate(zip(ms, pats)):
        exp, bad = oracle_refactor(m, P, m.Ax, fp32=True)
        assert _bitwise(B.factor_values(s), exp).size == 0
        _, q = P.perm()
        assert rel_err(xs[s], oracle_solution(m, m.Ax, q=q)) <= TOL_REL, st[s]
