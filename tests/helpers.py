"""Shared test utilities: problem construction and independent re-derivations
of the static layout maps used to drive the oracle."""
from __future__ import annotations

import numpy as np

from luspice_b200 import api, mna
from oracle import oracle as O

TOL_REL = 1e-6          # acceptance: rel-L2 error vs the fp64 oracle


def a_slot_map(m, pattern):
    """(a_ptr, a_src, a_dst) of the pattern, re-derived from its public
    structure and permutations: input entry p of column c, row r lands in
    column k = invq[c] at the slot of row position pinv[r]."""
    cp, ri, dg = pattern.structure()
    pinv, q = pattern.perm()
    n = m.n
    invq = np.empty(n, np.int64)
    invq[q] = np.arange(n)
    cols = np.repeat(np.arange(n), np.diff(m.Ap))
    k = invq[cols]
    pos = pinv[m.Ai]
    dst = np.empty(m.nnz, np.int64)
    for e in range(m.nnz):
        c0, c1 = cp[k[e]], cp[k[e] + 1]
        j = np.searchsorted(ri[c0:c1], pos[e])
        assert ri[c0 + j] == pos[e]
        dst[e] = j
    order = np.lexsort((np.arange(m.nnz), dst, k))
    a_ptr = np.zeros(n + 1, np.int64)
    np.add.at(a_ptr, k + 1, 1)
    a_ptr = np.cumsum(a_ptr)
    return a_ptr, order, dst[order], (cp, ri, dg)


def oracle_refactor(m, pattern, values, fp32):
    a_ptr, a_src, a_dst, (cp, ri, dg) = a_slot_map(m, pattern)
    vals, bad = O.static_refactor(m.n, cp, ri, dg, a_ptr, a_src, a_dst, values, fp32)
    return vals, bad


def oracle_solution(m, values, rhs=None, q=None):
    """fp64 reference solve (splu lu_factor + lu_solve_perm) with the same
    column order."""
    b = m.b if rhs is None else rhs
    return O.ref_cpu_solve(m.n, m.Ap, m.Ai, values, q, b)


def rel_err(x, ref):
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


def rel_res(m, values, x, b):
    return float(np.linalg.norm(m.matvec(x, values) - b) / max(np.linalg.norm(b), 1e-300))


FP16_MIN_NORMAL = 2.0 ** -14


def ruiz_scaling(n, Ap, Ai, values, sweeps=30, tol=1e-6):
    """Restatement of the Ruiz equilibration both the standalone SELL
    (lusp_ruiz_csr) and the engine's fp16 inner products run: row maxima of
    |a| r_i c_j, r_i /= sqrt(max), then column maxima, c_j /= sqrt(max),
    until every maximum is within tol of 1 (at most `sweeps` sweeps).  The
    maxima do not depend on the order entries are visited in, so CSC input
    gives the same r, c as the CSR loops.  Returns (r, c, rows, cols)."""
    cols = np.repeat(np.arange(n), np.diff(Ap))
    rows = np.asarray(Ai, dtype=np.int64)
    a = np.abs(values)
    r = np.ones(n)
    c = np.ones(n)
    for _ in range(sweeps):
        dev = 0.0
        rm = np.zeros(n)
        np.maximum.at(rm, rows, a * r[rows] * c[cols])
        nz = rm > 0
        r[nz] = r[nz] / np.sqrt(rm[nz])
        dev = max(dev, float(np.max(np.abs(1.0 - rm[nz]), initial=0.0)))
        cm = np.zeros(n)
        np.maximum.at(cm, cols, a * r[rows] * c[cols])
        nz = cm > 0
        c[nz] = c[nz] / np.sqrt(cm[nz])
        dev = max(dev, float(np.max(np.abs(1.0 - cm[nz]), initial=0.0)))
        if dev < tol:
            break
    return r, c, rows, cols


def ruiz_fits_fp16(m, values):
    """Whether every Ruiz-scaled nonzero lies in the fp16 normal range."""
    r, c, rows, cols = ruiz_scaling(m.n, m.Ap, m.Ai, values)
    s = np.abs(values * r[rows] * c[cols])
    s = s[s != 0]
    return bool(s.min() >= FP16_MIN_NORMAL and s.max() <= 65504.0)


def small_problems():
    return [mna.analog(120, 7), mna.analog(989, 42), mna.power_grid(15, 16, 6, seed=3)]
