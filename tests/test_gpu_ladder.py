"""Device-side escalation ladder (P-fast -> P-safe -> P-hard in one launch)
and the factor diagonal shift, through the lusp_* C-ABI on the GPU."""
import numpy as np
import pytest

from luspice_b200 import api, mna
from tests.helpers import TOL_REL, oracle_refactor, oracle_solution, rel_err, rel_res, small_problems

pytestmark = pytest.mark.gpu


def _shifted(m, values, shift):
    """values with every diagonal input entry a -> a + shift*|a| (the
    matrix has at most one stored entry per diagonal position)."""
    cols = np.repeat(np.arange(m.n), np.diff(m.Ap))
    diag = np.flatnonzero(m.Ai == cols)
    assert np.unique(m.Ai[diag]).size == diag.size
    out = values.copy()
    out[diag] = values[diag] + shift * np.abs(values[diag])
    return out


@pytest.mark.parametrize("idx", [0, 1, 2])
def test_factor_shift_bitwise(gpu, idx):
    """factor_shift: the stored factor is the frozen-pivot factor of
    A + shift diag|A(i,i)|, bit for bit the oracle's of the shifted values."""
    m = small_problems()[idx]
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(2, seed=31 + idx)
    shift = 1e-3
    B = api.Batch([P] * 2, prec=api.MIXED, factor_shift=shift)
    B.upload(list(vals), [m.b] * 2)
    B.run(api.RUN_REFACTOR)
    for s in range(2):
        got = B.factor_values(s)
        exp, bad = oracle_refactor(m, P, _shifted(m, vals[s], shift), fp32=True)
        assert bad < 0
        mism = np.flatnonzero(got.view(np.uint32) != exp.astype(np.float32).view(np.uint32))
        assert mism.size == 0, f"system {s}: {mism.size} slots differ"


def test_factor_shift_solution_uses_unshifted_matrix(gpu):
    """The shift perturbs only the preconditioner: GMRES-IR still converges
    to the solution of A itself."""
    m = mna.analog(989, 42)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(2, seed=5)
    B = api.Batch([P] * 2, prec=api.MIXED, factor_shift=1e-4, max_outer=6)
    B.upload(list(vals), [m.b] * 2)
    B.run(api.RUN_BOTH)
    xs = B.split(B.download())
    _, q = P.perm()
    for s in range(2):
        assert rel_err(xs[s], oracle_solution(m, vals[s], q=q)) <= TOL_REL
        assert rel_res(m, vals[s], xs[s], m.b) <= 1e-9


def _run(m, P, vals, **opts):
    B = api.Batch([P] * len(vals), prec=api.MIXED, **opts)
    B.upload(list(vals), [m.b] * len(vals))
    B.run(api.RUN_BOTH)
    xs = B.split(B.download())
    return B, xs, B.stats()


@pytest.mark.parametrize("ladder,rung", [(api.LADDER_SAFE, 1), (api.LADDER_HARD, 2), (api.LADDER_SAFE_HARD, 1)])
def test_ladder_takes_failed_systems(gpu, ladder, rung):
    """pivot_tol = 1 marks every P-fast factor weak (a failure on the first
    rung only): every system climbs to the first fp64 rung of the ladder
    inside the same launch and its answer is the fp64 oracle's."""
    m = mna.analog(989, 42)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(3, seed=9)
    B, xs, st = _run(m, P, vals, pivot_tol=1.0, ladder=ladder)
    _, q = P.perm()
    for s in range(3):
        assert st[s]["rung"] == rung, st[s]
        assert st[s]["status"] & api.ST_ESCALATED
        assert bool(st[s]["status"] & api.ST_SHIFTED) == (rung == 2)
        assert not st[s]["status"] & api.ST_LADDER_FULL
        assert rel_err(xs[s], oracle_solution(m, vals[s], q=q)) <= TOL_REL
        assert rel_res(m, vals[s], xs[s], m.b) <= 1e-9
        assert st[s]["res"][-1] <= 1e-10
    per_rung = 3 if P.info["dense_tail"] > 0 else 2
    assert B.launch_count() == per_rung * (1 + bin(ladder).count("1"))


def test_ladder_untouched_when_nothing_fails(gpu):
    """Systems that pass P-fast keep their P-fast result bit for bit."""
    m = mna.analog(989, 42)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(3, seed=12)
    _, x0, st0 = _run(m, P, vals)
    _, x1, st1 = _run(m, P, vals, ladder=api.LADDER_SAFE_HARD)
    for s in range(3):
        assert st1[s]["rung"] == 0
        assert not st1[s]["status"] & api.ST_ESCALATED
        assert np.array_equal(x0[s].view(np.uint64), x1[s].view(np.uint64))
        assert st0[s]["res"] == st1[s]["res"]


def test_ladder_safe_then_hard(gpu):
    """An unreachable rtol fails every rung: P-fast -> P-safe -> P-hard in one
    launch; the last rung's answer is still the best iterate of GMRES-IR on A
    and agrees with the fp64 oracle."""
    m = mna.analog(989, 42)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(2, seed=21)
    _, xs, st = _run(m, P, vals, rtol=1e-300, ladder=api.LADDER_SAFE_HARD)
    _, q = P.perm()
    for s in range(2):
        assert st[s]["rung"] == 2, st[s]
        assert st[s]["status"] & api.ST_ESCALATED and st[s]["status"] & api.ST_SHIFTED
        assert rel_err(xs[s], oracle_solution(m, vals[s], q=q)) <= TOL_REL


def test_ladder_slots_overflow(gpu):
    """More failures than slots (an unreachable rtol fails every system): the
    first ones climb, the rest keep their P-fast results and say so."""
    m = mna.analog(500, 4)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(4, seed=2)
    _, xs, st = _run(m, P, vals, rtol=1e-300, ladder=api.LADDER_SAFE, ladder_slots=2)
    rungs = sorted(s["rung"] for s in st)
    assert rungs == [0, 0, 1, 1], st
    for s in st:
        if s["rung"] == 0:
            assert s["status"] & api.ST_LADDER_FULL and not s["status"] & api.ST_ESCALATED
        else:
            assert s["status"] & api.ST_ESCALATED and not s["status"] & api.ST_LADDER_FULL


def test_ladder_ill_conditioned_mix(gpu):
    """Well- and ill-conditioned Newton steps in one launch with the ladder
    on: every answer's residual is as good as the fp64 oracle's, and the
    systems the ladder did not touch equal a launch without it."""
    m = mna.analog(989, 42)
    P = api.Pattern.from_matrix(m)
    good = m.perturbed(2, seed=3)
    bad = [mna.ill_conditioned(m, seed=s) for s in (3, 4)]
    vals = [good[0], bad[0], good[1], bad[1]]
    _, x0, st0 = _run(m, P, vals)
    _, xs, st = _run(m, P, vals, ladder=api.LADDER_SAFE_HARD)
    _, q = P.perm()
    for s in range(4):
        ref = oracle_solution(m, vals[s], q=q)
        r = rel_res(m, vals[s], xs[s], m.b)
        r_ref = rel_res(m, vals[s], ref, m.b)
        assert r <= max(10 * r_ref, 1e-9), (s, r, r_ref, st[s])
        if st[s]["rung"] == 0:
            assert np.array_equal(x0[s].view(np.uint64), xs[s].view(np.uint64))


def test_ladder_graph_replay(gpu):
    """The ladder's kernels replay from a CUDA graph with the same results."""
    m = mna.analog(700, 8)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(3, seed=4)
    B = api.Batch([P] * 3, prec=api.MIXED, rtol=1e-300, ladder=api.LADDER_SAFE)
    B.upload(list(vals), [m.b] * 3)
    B.run(api.RUN_BOTH)
    x_direct = B.download().copy()
    for _ in range(2):
        B.run(api.RUN_BOTH, graph=True)
        x_graph = B.download()
        assert np.array_equal(x_direct.view(np.uint64), x_graph.view(np.uint64))
    assert all(s["rung"] == 1 for s in B.stats())
