"""Parity of the batched engine (refactor, solves) with the oracle, through
the lusp_* C-ABI on the GPU."""
import numpy as np
import pytest

from luspice_b200 import api, mna
from tests.helpers import TOL_REL, oracle_refactor, oracle_solution, rel_err, rel_res, small_problems

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [api.MIXED, api.FP64])
@pytest.mark.parametrize("idx", [0, 1, 2])
def test_refactor_bitwise(gpu, prec, idx):
    """Frozen-pivot refactorization equals the host restatement bit for bit
    (fp64 work vector, separately rounded multiply/subtract; fp32 storage on
    the mixed path)."""
    m = small_problems()[idx]
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(3, seed=100 + idx)
    B = api.Batch([P] * 3, prec=prec)
    B.upload(list(vals), [m.b] * 3)
    B.run(api.RUN_REFACTOR)
    st = B.stats()
    for s in range(3):
        got = B.factor_values(s)
        exp, bad = oracle_refactor(m, P, vals[s], fp32=(prec == api.MIXED))
        assert bad < 0
        exp = exp.astype(got.dtype)
        ity = np.uint32 if got.dtype == np.float32 else np.uint64
        mism = np.flatnonzero(got.view(ity) != exp.view(ity))
        assert mism.size == 0, f"system {s}: {mism.size} slots differ, first {mism[:5]}"
        assert st[s]["status"] & api.ST_SINGULAR == 0


@pytest.mark.parametrize("prec", [api.MIXED, api.FP64])
def test_solve_matches_oracle(gpu, prec):
    """Mixed (fp32 factors + fp64 GMRES-IR) and plain fp64 solves reach the
    fp64 oracle solution within rel-L2 1e-6 for every perturbed system."""
    m = mna.analog(989, 42)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(4, seed=7)
    B = api.Batch([P] * 4, prec=prec)
    B.upload(list(vals), [m.b] * 4)
    B.run(api.RUN_BOTH)
    xs = B.split(B.download())
    st = B.stats()
    _, q = P.perm()
    for s in range(4):
        ref = oracle_solution(m, vals[s], q=q)
        e = rel_err(xs[s], ref)
        r = rel_res(m, vals[s], xs[s], m.b)
        assert e <= TOL_REL, f"sys {s}: rel err {e:.3e} stats {st[s]}"
        assert r <= 1e-9, f"sys {s}: residual {r:.3e} stats {st[s]}"
        if prec == api.MIXED:
            assert st[s]["status"] & api.ST_FAIL_MASK == 0, st[s]
            assert st[s]["res"][-1] <= 1e-10


def test_power_grid_batch(gpu):
    m = mna.power_grid()
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(8, seed=11)
    B = api.Batch([P] * 8, prec=api.MIXED)
    B.upload(list(vals), [m.b] * 8)
    B.run(api.RUN_BOTH)
    xs = B.split(B.download())
    _, q = P.perm()
    for s in range(8):
        ref = oracle_solution(m, vals[s], q=q)
        assert rel_err(xs[s], ref) <= TOL_REL


def test_uneven_batch_same_alone_and_mixed(gpu):
    """Different patterns in one launch; each result equals the result of the
    same system solved alone (bitwise: one CTA runs a system the same way)."""
    ms = [mna.analog(int(n), 42 + i) for i, n in enumerate([150, 700, 333, 1200])]
    pats = [api.Pattern.from_matrix(m) for m in ms]
    B = api.Batch(pats, prec=api.MIXED)
    B.upload([m.Ax for m in ms], [m.b for m in ms])
    B.run(api.RUN_BOTH)
    xs = B.split(B.download())
    for i, m in enumerate(ms):
        b1 = api.Batch([pats[i]], prec=api.MIXED)
        b1.upload([m.Ax], [m.b])
        b1.run(api.RUN_BOTH)
        x1 = b1.download()
        assert np.array_equal(x1, xs[i])
        assert rel_err(xs[i], m.x_true) <= TOL_REL


def test_graph_replay_matches(gpu):
    m = mna.analog(500, 5)
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(2, seed=3)
    B = api.Batch([P] * 2)
    B.upload(list(vals), [m.b] * 2)
    B.run(api.RUN_BOTH)
    x0 = B.download()
    B.run(api.RUN_BOTH, graph=True)
    B.run(api.RUN_BOTH, graph=True)
    x1 = B.download()
    assert np.array_equal(x0, x1)


def test_kernel_timing_events(gpu):
    """Per-kernel CUDA-event times of a run: all three kernels timed, they add
    up to no more than the whole run, the results equal an untimed run's,
    and a refactor-only run reports no solve time."""
    import torch
    m = mna.power_grid(15, 16, 6, seed=3)
    P = api.Pattern.from_matrix(m, dense_tail=64)
    vals = m.perturbed(3, seed=2)
    B = api.Batch([P] * 3)
    B.upload(list(vals), [m.b] * 3)
    B.run(api.RUN_BOTH)
    x0 = B.download().copy()
    with pytest.raises(api.LuspError):
        B.kernel_ms()
    B.time_kernels(True)
    s = torch.cuda.Stream()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(s)
    B.run(api.RUN_BOTH, stream=s)
    b.record(s)
    t = B.kernel_ms()
    torch.cuda.synchronize()
    assert t["refactor"] > 0 and t["dense"] > 0 and t["solve"] > 0
    assert t["refactor"] + t["dense"] + t["solve"] <= a.elapsed_time(b) + 1e-3
    assert np.array_equal(B.download(), x0)
    B.run(api.RUN_REFACTOR)
    t = B.kernel_ms()
    assert t["refactor"] > 0 and t["solve"] < 0.01
    B.time_kernels(False)


def test_direct_solve_fp32_factors(gpu):
    m = mna.analog(400, 9)
    P = api.Pattern.from_matrix(m)
    B = api.Batch([P])
    B.upload([m.Ax], [m.b])
    B.run(api.RUN_REFACTOR)
    B.run(api.RUN_SOLVE | api.RUN_DIRECT)
    x = B.download()
    # fp32 factors alone: a few digits; the IR path restores the rest.
    assert rel_err(x, m.x_true) < 1e-2
    B.run(api.RUN_SOLVE)
    assert rel_err(B.download(), m.x_true) <= TOL_REL


def test_singular_flagged(gpu):
    """A value set that zeroes a pivot is reported, not hidden."""
    m = mna.analog(200, 13)
    P = api.Pattern.from_matrix(m)
    B = api.Batch([P], prec=api.FP64)
    B.upload([np.zeros(m.nnz)], [m.b])
    B.run(api.RUN_BOTH)
    st = B.stats()[0]
    assert st["status"] & api.ST_SINGULAR
    assert st["singular_col"] >= 0


@pytest.mark.parametrize("prec", [api.MIXED, api.FP64])
def test_cluster_refactor_bitwise(gpu, prec):
    """One system's columns spread over a 2-CTA thread-block cluster give the
    same factor bit for bit, and the same pivot statistics, as one CTA."""
    m = mna.power_grid()
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(3, seed=21)
    out = []
    for rc in (1, 2):
        B = api.Batch([P] * 3, prec=prec, refactor_cluster=rc)
        B.upload(list(vals), [m.b] * 3)
        B.run(api.RUN_REFACTOR)
        out.append(([B.factor_values(s) for s in range(3)], B.stats()))
        B.close()
    for s in range(3):
        exp, bad = oracle_refactor(m, P, vals[s], fp32=(prec == api.MIXED))
        for f, _ in out:
            got = f[s]
            ity = np.uint32 if got.dtype == np.float32 else np.uint64
            assert np.array_equal(got.view(ity), exp.astype(got.dtype).view(ity))
        for k in ("min_abs_pivot", "min_pivot_ratio", "max_abs_u", "status", "singular_col"):
            assert out[0][1][s][k] == out[1][1][s][k], k


@pytest.mark.parametrize("prec", [api.MIXED, api.FP64])
@pytest.mark.parametrize("group", [2, 37])
def test_refactor_spread_bitwise(gpu, prec, group):
    """Spread mode (several CTAs anywhere on the GPU share each system's
    columns through a claim counter and ready bits in global memory): the
    factor is the host restatement's bit for bit, as in cluster mode, and
    the pivot statistics equal the cluster mode's."""
    m = small_problems()[1]
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(3, seed=31)
    out = {}
    for spread in (-1, group):
        B = api.Batch([P] * 3, prec=prec, refactor_spread=spread)
        B.upload(list(vals), [m.b] * 3)
        B.run(api.RUN_BOTH)
        out[spread] = ([B.factor_values(s) for s in range(3)], B.stats(), B.split(B.download()))
        B.close()
    _, q = P.perm()
    for s in range(3):
        got = out[group][0][s]
        exp, bad = oracle_refactor(m, P, vals[s], fp32=(prec == api.MIXED))
        exp = exp.astype(got.dtype)
        ity = np.uint32 if got.dtype == np.float32 else np.uint64
        assert np.array_equal(got.view(ity), exp.view(ity)), f"system {s}"
        a, b = out[-1][1][s], out[group][1][s]
        for key in ("min_abs_pivot", "min_pivot_ratio", "max_abs_u", "status", "singular_col"):
            assert a[key] == b[key], (key, a[key], b[key])
        assert np.array_equal(out[-1][2][s], out[group][2][s])
        assert rel_err(out[group][2][s], oracle_solution(m, vals[s], q=q)) <= TOL_REL


def test_refactor_spread_singular_column(gpu):
    """A zero pivot found in spread mode is reported as the first singular
    column, as in cluster mode."""
    m = small_problems()[0]
    P = api.Pattern.from_matrix(m)
    cp, ri, dg = P.structure()
    pinv, q = P.perm()
    v = m.Ax.copy()
    # Zero the whole input column that becomes pivot column k (its diagonal
    # then receives only the updates, which are zero when the column is
    # empty): pick a column with no dependencies.
    k = next(k for k in range(m.n) if dg[k] == cp[k])
    c = q[k]
    v[m.Ap[c]:m.Ap[c + 1]] = 0.0
    sts = {}
    for spread in (-1, 5):
        B = api.Batch([P], prec=api.FP64, refactor_spread=spread)
        B.upload([v], [m.b])
        B.run(api.RUN_REFACTOR)
        sts[spread] = B.stats()[0]
        B.close()
    assert sts[5]["status"] & api.ST_SINGULAR
    assert sts[5]["singular_col"] == sts[-1]["singular_col"] >= 0


def test_launch_shapes_same_factor(gpu):
    """The launch rules pick spread mode (up to 12 CTAs of 256 threads per
    system, global-memory sync) for medium systems and a 2-CTA cluster for
    the dense trailing block; the factor bits, statistics and solutions are
    the same under every shape (spread, 2-CTA cluster refactor, lone CTAs),
    and equal the host restatement."""
    m = mna.power_grid()
    P = api.Pattern.from_matrix(m)
    vals = m.perturbed(4, seed=77)
    shapes = [dict(), dict(refactor_cluster=2), dict(refactor_cluster=1, refactor_threads=768),
              dict(refactor_spread=5, refactor_threads=512)]
    res = []
    for opts in shapes:
        B = api.Batch([P] * 4, prec=api.MIXED, **opts)
        B.upload(list(vals), [m.b] * 4)
        B.run(api.RUN_BOTH)
        sh = B.launch_shape()
        res.append((sh, [B.factor_values(s) for s in range(4)], B.stats(), B.split(B.download())))
        B.close()
    sh0 = res[0][0]
    assert sh0["refactor_spread"] == 12 and sh0["refactor_block"] == 256, sh0
    assert sh0["dense_cluster"] == 2 and sh0["dense_grid"] == 8, sh0
    assert res[1][0]["refactor_cluster"] == 2 and res[1][0]["refactor_spread"] == 0, res[1][0]
    assert res[2][0]["refactor_cluster"] == 1 and res[2][0]["refactor_spread"] == 0, res[2][0]
    assert res[3][0]["refactor_spread"] == 5, res[3][0]
    for s in range(4):
        exp, bad = oracle_refactor(m, P, vals[s], fp32=True)
        assert bad < 0
        for k, (sh, fac, st, xs) in enumerate(res):
            assert np.array_equal(fac[s].view(np.uint32), exp.astype(np.float32).view(np.uint32)), (k, s)
            for key in ("min_abs_pivot", "min_pivot_ratio", "max_abs_u"):
                assert st[s][key] == res[0][2][s][key], (k, s, key)
            assert np.array_equal(xs[s], res[0][3][s]), (k, s)
