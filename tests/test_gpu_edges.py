"""Edge cases of the batched engine through the lusp_* C-ABI: the smallest
systems, duplicate entries, a zero right-hand side, ragged batches, a
structurally singular pattern, non-finite values and bad arguments."""
import numpy as np
import pytest
import scipy.sparse as sp

from luspice_b200 import api, mna

pytestmark = pytest.mark.gpu


def _csc(A):
    A = sp.csc_matrix(A)
    A.sort_indices()
    return A.shape[0], A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data.astype(np.float64)


def _solve(pats, vals, rhs, prec=api.MIXED):
    B = api.Batch(pats, prec=prec)
    B.upload(vals, rhs)
    B.run(api.RUN_BOTH)
    return B.split(B.download()), B.stats()


@pytest.mark.parametrize("prec", [api.MIXED, api.FP64])
def test_tiny_and_ragged_batch(gpu, prec):
    """n = 1, n = 2 and a 500-node circuit in one launch; each answer is the
    dense solve's."""
    n1, Ap1, Ai1, Ax1 = _csc(np.array([[3.0]]))
    n2, Ap2, Ai2, Ax2 = _csc(np.array([[2.0, -1.0], [-1.0, 4.0]]))
    m = mna.analog(500, 11)
    pats = [api.Pattern(n1, Ap1, Ai1, Ax1), api.Pattern(n2, Ap2, Ai2, Ax2), api.Pattern.from_matrix(m)]
    b1, b2 = np.array([6.0]), np.array([1.0, 2.0])
    xs, st = _solve(pats, [Ax1, Ax2, m.Ax], [b1, b2, m.b], prec)
    assert np.allclose(xs[0], [2.0], rtol=1e-12)
    assert np.allclose(xs[1], np.linalg.solve([[2.0, -1.0], [-1.0, 4.0]], b2), rtol=1e-12)
    ref = np.linalg.solve(m.csr().toarray(), m.b)
    assert np.linalg.norm(xs[2] - ref) / np.linalg.norm(ref) <= 1e-6
    for s in st:
        assert s["status"] & api.ST_FAIL_MASK == 0, s


def test_duplicate_entries_are_summed(gpu):
    """A CSC with repeated (row, column) entries (MNA stamps) solves as the
    matrix of their sums."""
    Ap = np.array([0, 3, 5, 7], np.int32)
    Ai = np.array([0, 0, 1, 1, 2, 1, 2], np.int32)
    Ax = np.array([1.5, 1.5, -1.0, 2.0, -0.5, -0.5, 1.0])
    A = np.zeros((3, 3))
    cols = np.repeat(np.arange(3), np.diff(Ap))
    np.add.at(A, (Ai, cols), Ax)
    b = np.array([1.0, 0.0, 2.0])
    xs, st = _solve([api.Pattern(3, Ap, Ai, Ax)], [Ax], [b])
    assert np.allclose(xs[0], np.linalg.solve(A, b), rtol=1e-10)
    assert st[0]["status"] & api.ST_FAIL_MASK == 0


def test_zero_rhs_gives_zero(gpu):
    m = mna.analog(300, 2)
    P = api.Pattern.from_matrix(m)
    xs, st = _solve([P, P], [m.Ax, m.Ax], [np.zeros(m.n), m.b])
    assert np.all(xs[0] == 0.0)
    assert st[0]["status"] & api.ST_FAIL_MASK == 0
    assert np.linalg.norm(m.matvec(xs[1]) - m.b) / np.linalg.norm(m.b) <= 1e-9


def test_structurally_singular_pattern_refused(gpu):
    """An empty column: the host analysis refuses the pattern."""
    Ap = np.array([0, 2, 2, 3], np.int32)
    Ai = np.array([0, 1, 2], np.int32)
    with pytest.raises(api.LuspError) as e:
        api.Pattern(3, Ap, Ai, np.ones(3))
    assert e.value.rc == 1          # LUSP_ESINGULAR


def test_nonfinite_values_flagged_without_hang(gpu):
    """A NaN in one system's values: that system is flagged, its neighbour
    in the same launch is unaffected."""
    m = mna.analog(400, 6)
    P = api.Pattern.from_matrix(m)
    bad = m.Ax.copy()
    bad[len(bad) // 2] = np.nan
    xs, st = _solve([P, P], [bad, m.Ax], [m.b, m.b])
    assert st[0]["status"] & (api.ST_NONFINITE | api.ST_SINGULAR | api.ST_STAGNATED | api.ST_NOT_CONVERGED)
    assert st[1]["status"] & api.ST_FAIL_MASK == 0
    assert np.linalg.norm(m.matvec(xs[1]) - m.b) / np.linalg.norm(m.b) <= 1e-9


def test_bad_batch_arguments(gpu):
    m = mna.analog(200, 1)
    P = api.Pattern.from_matrix(m)
    with pytest.raises(api.LuspError):
        api.Batch([])
    with pytest.raises(api.LuspError):
        api.Batch([P], krylov=0)
    with pytest.raises(api.LuspError):
        api.Batch([P], inner_prec=3)
    with pytest.raises(api.LuspError):
        api.Batch([P], ladder=4)
    B = api.Batch([P])
    with pytest.raises(ValueError):
        B.upload([m.Ax[:-1]], [m.b])
