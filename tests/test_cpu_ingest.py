"""Netlist ingest on the host: s0 and Matrix Market files, the .flt
floating-node pin, COO -> CSC (no GPU)."""
import numpy as np
import pytest
import scipy.io
import scipy.sparse as sp

from luspice_b200 import api, mna


def _write_s0(path, n, rows, cols, vals):
    with open(path, "w") as f:
        f.write(f"n {n}\n")
        for i, j, v in zip(rows, cols, vals):
            f.write(f"A {i + 1} {j + 1} {float(v)!r}\n")


def _pin_restated(n, rows, cols, vals, frows, pin):
    """The replay programs' pin rule (bench/test_lu.c:71-93), restated: per
    listed row in file order, the first stored (i, i) entry gains pin, else a
    new (i, i) = pin entry is appended."""
    rows, cols, vals = list(rows), list(cols), list(vals)
    for i in frows:
        for k in range(len(rows)):
            if rows[k] == i and cols[k] == i:
                vals[k] += pin
                break
        else:
            rows.append(i)
            cols.append(i)
            vals.append(pin)
    return np.array(rows), np.array(cols), np.array(vals)


def _csc(n, rows, cols, vals):
    """CSC with entries of a column in storage order (a stable sort)."""
    order = np.argsort(cols, kind="stable")
    Ap = np.zeros(n + 1, np.int64)
    np.add.at(Ap, cols + 1, 1)
    return np.cumsum(Ap), rows[order], vals[order]


def test_s0_with_flt_pin_matches_replay_rule(tmp_path):
    m = mna.analog(300, 5)
    coo = m.csr().tocoo()
    rng = np.random.default_rng(0)
    # Some listed rows have a stored diagonal, some do not (drop a few).
    keep = np.ones(coo.nnz, bool)
    diag = np.flatnonzero(coo.row == coo.col)
    keep[rng.choice(diag, 10, replace=False)] = False
    r, c, v = coo.row[keep], coo.col[keep], coo.data[keep]
    perm = rng.permutation(r.size)
    r, c, v = r[perm], c[perm], v[perm]
    _write_s0(tmp_path / "a.s0", m.n, r, c, v)
    frows = list(rng.choice(m.n, 25, replace=False)) + [int(r[0])]
    with open(tmp_path / "a.flt", "w") as f:
        f.write("* floating nodes\n")
        for i in frows:
            f.write(f"F {i + 1}\n")
    pin = 1e-9
    n, Ap, Ai, Ax = api.read_netlist(tmp_path / "a.s0", tmp_path / "a.flt", pin)
    er, ec, ev = _pin_restated(m.n, r, c, v, frows, pin)
    eAp, eAi, eAx = _csc(m.n, er, ec, ev)
    assert n == m.n
    assert np.array_equal(Ap, eAp) and np.array_equal(Ai, eAi)
    assert np.array_equal(Ax.view(np.uint64), eAx.view(np.uint64))
    # No pin: the file's entries only.
    n, Ap, Ai, Ax = api.read_netlist(tmp_path / "a.s0")
    assert Ai.size == r.size


@pytest.mark.parametrize("symmetry", ["general", "symmetric", "skew-symmetric"])
def test_matrix_market_matches_scipy(tmp_path, symmetry):
    A = sp.random(60, 60, density=0.08, random_state=3, format="csr")
    if symmetry == "symmetric":
        A = A + A.T
        W = sp.tril(A).tocoo()
    elif symmetry == "skew-symmetric":
        A = sp.tril(A, -1)
        A = A - A.T
        W = sp.tril(A).tocoo()
    else:
        W = A.tocoo()
    scipy.io.mmwrite(tmp_path / "m.mtx", W, symmetry=symmetry)
    n, Ap, Ai, Ax = api.read_netlist(tmp_path / "m.mtx")
    B = sp.csc_matrix((Ax, Ai, Ap), shape=(n, n))
    assert n == 60 and abs(B - A.tocsc()).max() == 0


def test_ingest_rejects_bad_files(tmp_path):
    (tmp_path / "bad.s0").write_text("n 3\nA 1 4 1.0\n")
    with pytest.raises(api.LuspError):
        api.read_netlist(tmp_path / "bad.s0")
    (tmp_path / "ok.s0").write_text("n 3\nA 1 1 1.0\nA 2 2 1\nA 3 3 1\n")
    (tmp_path / "bad.flt").write_text("F 4\n")
    with pytest.raises(api.LuspError):
        api.read_netlist(tmp_path / "ok.s0", tmp_path / "bad.flt", 1e-6)
    (tmp_path / "rect.mtx").write_text("%%MatrixMarket matrix coordinate real general\n2 3 1\n1 1 1.0\n")
    with pytest.raises(api.LuspError):
        api.read_netlist(tmp_path / "rect.mtx")
    (tmp_path / "short.mtx").write_text("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1.0\n")
    with pytest.raises(api.LuspError):
        api.read_netlist(tmp_path / "short.mtx")


def test_replayed_netlist_analyses_like_the_generator(tmp_path):
    """A generated matrix written as s0 and read back gives the same host
    analysis (column order and pivots) as the in-memory matrix."""
    m = mna.analog(400, 9)
    coo = sp.csc_matrix((m.Ax, m.Ai, m.Ap), shape=(m.n, m.n)).tocoo()
    _write_s0(tmp_path / "g.s0", m.n, coo.row, coo.col, coo.data)
    n, Ap, Ai, Ax = api.read_netlist(tmp_path / "g.s0")
    q0 = api.colamd(m.n, m.Ap, m.Ai)
    q1 = api.colamd(n, Ap, Ai)
    assert np.array_equal(q0, q1)
    f0 = api.pivot_factor(m.n, m.Ap, m.Ai, m.Ax, q0)
    f1 = api.pivot_factor(n, Ap, Ai, Ax, q1)
    assert np.array_equal(f0["pinv"], f1["pinv"])
