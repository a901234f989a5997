"""lu_static.h drop-in flow (bench/test_lu.c shape) through the C-ABI:
dsh_symbolic once, dsh_numeric several times (symbolic count stays 1),
dsh_trisolve and dsh_gmres_ir, residual and parity against the oracle."""
import ctypes as C

import numpy as np
import pytest

from luspice_b200 import _lib, api, mna
from tests.helpers import TOL_REL, oracle_solution, rel_err

pytestmark = pytest.mark.gpu


def _coo1(m):
    cols = np.repeat(np.arange(m.n), np.diff(m.Ap))
    return (np.ascontiguousarray(m.Ai + 1, dtype=np.int32), np.ascontiguousarray(cols + 1, dtype=np.int32))


def test_lu_static_flow(gpu, lib):
    m = mna.analog(989, 42)
    row1, col1 = _coo1(m)
    q = api.colamd(m.n, m.Ap, m.Ai)
    F = _lib.DshLuStatic()
    assert lib.dsh_lu_static_init(C.byref(F)) == 0
    c0 = lib.dsh_symbolic_count()
    rc = lib.dsh_symbolic(m.n, m.nnz, _lib.ptr(row1, C.c_int), _lib.ptr(col1, C.c_int), _lib.ptr(q, C.c_int),
                          C.byref(F))
    assert rc == 0 and F.n == m.n and F.cnnz == m.nnz
    assert list(np.ctypeslib.as_array(F.Q, shape=(m.n,))) == list(q)
    vals = m.perturbed(3, seed=5)
    for t in range(3):
        v = np.ascontiguousarray(vals[t])
        rc = lib.dsh_numeric(C.byref(F), _lib.ptr(row1, C.c_int), _lib.ptr(col1, C.c_int), _lib.ptr(v, C.c_double),
                             m.nnz)
        assert rc == 0, lib.dsh_lu_status_str(rc)
        assert lib.dsh_symbolic_count() == c0 + 1          # symbolic reuse (bench/test_lu.c:140-147)
        assert F.lnnz > 0 and F.unnz > 0 and F.cap == F.lnnz + F.unnz - m.n
        assert F.min_diag_U > 0 and F.dev_allocated == 1
        b = np.ascontiguousarray(m.b)
        x = np.zeros(m.n)
        assert lib.dsh_trisolve(C.byref(F), _lib.ptr(b, C.c_double), _lib.ptr(x, C.c_double)) == 0
        ref = oracle_solution(m, v, q=q)
        assert rel_err(x, ref) < 1e-2                      # fp32 factors, no refinement
        res = np.zeros(8)
        it = C.c_int()
        rc = lib.dsh_gmres_ir(C.byref(F), _lib.ptr(b, C.c_double), _lib.ptr(x, C.c_double), 3, 30, 1e-10,
                              _lib.ptr(res, C.c_double), C.byref(it))
        assert rc == 0 and it.value >= 1
        assert rel_err(x, ref) <= TOL_REL
        assert res[0] == pytest.approx(1.0) and np.min(res[res > 0]) <= 1e-10
    # merged structure published on the host
    Ap = np.ctypeslib.as_array(F.Ap, shape=(m.n + 1,))
    assert Ap[-1] == F.cap
    pinv = np.ctypeslib.as_array(F.P, shape=(m.n,))
    assert np.array_equal(np.sort(pinv), np.arange(m.n))
    lib.dsh_lu_static_free(C.byref(F))
    assert F.factor_cache is None and not F.Ap


def test_lu_static_arguments(gpu, lib):
    F = _lib.DshLuStatic()
    lib.dsh_lu_static_init(C.byref(F))
    z = np.zeros(4, np.int32)
    assert lib.dsh_symbolic(0, 0, _lib.ptr(z, C.c_int), _lib.ptr(z, C.c_int), None, C.byref(F)) == 3
    bad = np.array([1, 9], np.int32)
    assert lib.dsh_symbolic(2, 2, _lib.ptr(bad, C.c_int), _lib.ptr(bad, C.c_int), None, C.byref(F)) == 3
    x = np.zeros(2)
    assert lib.dsh_trisolve(C.byref(F), _lib.ptr(x, C.c_double), _lib.ptr(x, C.c_double)) == 3
    assert lib.dsh_lu_status_str(0) == b"OK" and lib.dsh_lu_status_str(1) == b"SINGULAR"
    assert lib.dsh_lu_status_str(4) == b"IR_STAGNATED"


def test_lu_static_singular(gpu, lib):
    """A structurally singular matrix is reported as SINGULAR (rc 1)."""
    n = 3
    row1 = np.array([1, 2, 1, 2, 3], np.int32)
    col1 = np.array([1, 1, 2, 2, 3], np.int32)
    v = np.array([1.0, 2.0, 2.0, 4.0, 1.0])
    F = _lib.DshLuStatic()
    lib.dsh_lu_static_init(C.byref(F))
    assert lib.dsh_symbolic(n, 5, _lib.ptr(row1, C.c_int), _lib.ptr(col1, C.c_int), None, C.byref(F)) == 0
    assert lib.dsh_numeric(C.byref(F), _lib.ptr(row1, C.c_int), _lib.ptr(col1, C.c_int), _lib.ptr(v, C.c_double), 5) == 1
    lib.dsh_lu_static_free(C.byref(F))
