"""n = 40,000 circuit with supply nets (the large configuration): host
analysis, GPU refactor (columns longer than the shared-memory work area spill
to global scratch, dependency columns longer than the stage are applied
directly) and both solve paths, against the fp64 oracle."""
import numpy as np
import pytest

from luspice_b200 import api, mna
from tests.helpers import TOL_REL, oracle_solution, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def large():
    m = mna.large_circuit()
    P = api.Pattern.from_matrix(m)
    _, q = P.perm()
    ref = oracle_solution(m, m.Ax, q=q)
    return m, P, ref


@pytest.mark.parametrize("prec,inner", [(api.MIXED, 1), (api.FP64, 0)])
def test_large_solve(gpu, large, prec, inner):
    """Values spanning 15 decades: the mixed path needs fp64 inner products
    (inner_prec = 1); the plain fp64 path solves directly."""
    m, P, ref = large
    B = api.Batch([P], prec=prec, inner_prec=inner, max_outer=10)
    B.upload([m.Ax], [m.b])
    B.run(api.RUN_BOTH)
    x = B.download()
    st = B.stats()[0]
    assert st["status"] & api.ST_FAIL_MASK == 0, st
    assert rel_err(x, ref) <= TOL_REL, (rel_err(x, ref), st)


def test_large_refinement_stops_on_forward_error(gpu, large):
    """Condition number ~1e15: a residual of 1e-10 alone still allows a 1%
    error, so the refinement also requires the correction-based forward
    error estimate; with too few outer steps it reports NOT_CONVERGED (the
    escalation signal) instead of a small-residual but inaccurate answer."""
    m, P, ref = large
    B = api.Batch([P], prec=api.MIXED, inner_prec=1, max_outer=2)
    B.upload([m.Ax], [m.b])
    B.run(api.RUN_BOTH)
    x = B.download()
    st = B.stats()[0]
    assert (st["status"] & api.ST_FAIL_MASK) or rel_err(x, ref) <= TOL_REL, (rel_err(x, ref), st)


def test_large_fp32_inner_stagnates_and_keeps_best(gpu, large):
    """With fp32 inner products the IR stops improving; the solver reports it
    (the escalation signal) and returns the best iterate, not a diverged one."""
    m, P, ref = large
    B = api.Batch([P], prec=api.MIXED, inner_prec=0)
    B.upload([m.Ax], [m.b])
    B.run(api.RUN_BOTH)
    x = B.download()
    st = B.stats()[0]
    if st["status"] & api.ST_FAIL_MASK == 0:
        assert rel_err(x, ref) <= TOL_REL
        return
    assert st["status"] & (api.ST_STAGNATED | api.ST_NOT_CONVERGED)
    r = np.linalg.norm(m.matvec(x) - m.b) / np.linalg.norm(m.b)
    assert r <= min(st["res"]) * (1 + 1e-6)


def test_large_spread_and_wide_sweeps_match_single_cluster(gpu, large):
    """The 40k system refactored by every SM (spread mode, the default for a
    lone large system) gives the same factor bits as one 2-SM cluster, and
    the level sweeps with several warps per long row give the same solution
    class as the per-row dataflow sweeps."""
    m, P, ref = large
    xs, fv = {}, {}
    for spread, sweep in ((0, 0), (-1, 1)):
        B = api.Batch([P], prec=api.FP64, refactor_spread=spread, solve_sweep=sweep)
        B.upload([m.Ax], [m.b])
        B.run(api.RUN_BOTH)
        xs[spread] = B.download()
        fv[spread] = B.factor_values(0)
        st = B.stats()[0]
        assert st["status"] & api.ST_FAIL_MASK == 0, st
        B.close()
    assert np.array_equal(fv[0].view(np.uint64), fv[-1].view(np.uint64))
    for k in xs:
        assert rel_err(xs[k], ref) <= TOL_REL
