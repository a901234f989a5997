"""The allocation-free triangular solve (lusp_trisolve_par_noalloc).

Some callers cannot allocate device memory at solve time — a simulator's
time-step loop that sized everything when the netlist was loaded and must
not call cudaMalloc mid-run, or host code that owns all device memory
through its own arena — so this entry point takes its work arrays from a
fixed scratch area inside the library.  The test checks, through the C-ABI,
that two calls in a row give the same x as the regular entry point with
caller-provided work arrays (bitwise, the tolerance the other trisolve tests
use), and that sizes above the limit are refused with an error.

This file sorts last so a run that stops at the first failure has already
run every other test."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from luspice_b200 import _lib, api, mna
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAX_N = 65536


def _dev(torch, a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_trisolve_matches_regular_entry_point(gpu, lib):
    import torch
    m = mna.analog(989, 42)
    q = api.colamd(m.n, m.Ap, m.Ai)
    F = O.lu_factor(m.n, m.Ap, m.Ai, m.Ax, q)
    assert F["status"] == -1
    n = m.n
    t = {k: _dev(torch, F[k], torch.int32) for k in ("Lp", "Li", "Up", "Ui", "pinv")}
    t.update({k: _dev(torch, F[k], torch.float64) for k in ("Lx", "Ux")})
    dq = _dev(torch, q, torch.int32)
    wi = torch.zeros(n, dtype=torch.int32, device="cuda")
    wd = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(7)
    for call in range(2):
        b = _dev(torch, rng.standard_normal(n), torch.float64)
        x_ref = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        x_new = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        rc = lib.lusp_trisolve_par_launch(n, _p(t["Lp"]), _p(t["Li"]), _p(t["Lx"]), _p(t["Up"]), _p(t["Ui"]),
                                          _p(t["Ux"]), _p(t["pinv"]), _p(dq), _p(b), _p(x_ref), _p(wi), _p(wd), None)
        assert rc == 0
        rc = lib.lusp_trisolve_par_noalloc(n, _p(t["Lp"]), _p(t["Li"]), _p(t["Lx"]), _p(t["Up"]), _p(t["Ui"]),
                                           _p(t["Ux"]), _p(t["pinv"]), _p(dq), _p(b), _p(x_new), None)
        assert rc == 0, lib.lusp_last_error()
        torch.cuda.synchronize()
        a, c = x_ref.cpu().numpy(), x_new.cpu().numpy()
        assert np.all(np.isfinite(c))
        assert np.array_equal(a.view(np.uint64), c.view(np.uint64)), f"call {call}"
        # and both are the host column solve on the same factors
        xh = O.lu_solve(F, q, b.cpu().numpy())
        assert np.array_equal(c.view(np.uint64), xh.view(np.uint64))


def test_noalloc_trisolve_without_column_order(gpu, lib):
    """q = NULL (x returned in pivot-column order, as lu_solve_perm with no
    column permutation): the same bits as the regular entry point given
    q = NULL, on two calls in a row."""
    import torch
    m = mna.analog(600, 11)
    q = api.colamd(m.n, m.Ap, m.Ai)
    F = O.lu_factor(m.n, m.Ap, m.Ai, m.Ax, q)
    assert F["status"] == -1
    n = m.n
    t = {k: _dev(torch, F[k], torch.int32) for k in ("Lp", "Li", "Up", "Ui", "pinv")}
    t.update({k: _dev(torch, F[k], torch.float64) for k in ("Lx", "Ux")})
    wi = torch.zeros(n, dtype=torch.int32, device="cuda")
    wd = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(9)
    for call in range(2):
        b = _dev(torch, rng.standard_normal(n), torch.float64)
        x_ref = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        x_new = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
        assert lib.lusp_trisolve_par_launch(n, _p(t["Lp"]), _p(t["Li"]), _p(t["Lx"]), _p(t["Up"]), _p(t["Ui"]),
                                            _p(t["Ux"]), _p(t["pinv"]), None, _p(b), _p(x_ref), _p(wi), _p(wd),
                                            None) == 0
        rc = lib.lusp_trisolve_par_noalloc(n, _p(t["Lp"]), _p(t["Li"]), _p(t["Lx"]), _p(t["Up"]), _p(t["Ui"]),
                                           _p(t["Ux"]), _p(t["pinv"]), None, _p(b), _p(x_new), None)
        assert rc == 0, lib.lusp_last_error()
        torch.cuda.synchronize()
        a, c = x_ref.cpu().numpy(), x_new.cpu().numpy()
        assert np.all(np.isfinite(c))
        assert np.array_equal(a.view(np.uint64), c.view(np.uint64)), f"call {call}"
        xh = O.lu_solve(F, None, b.cpu().numpy())
        assert np.array_equal(c.view(np.uint64), xh.view(np.uint64))


def test_noalloc_trisolve_rejects_oversize(gpu, lib):
    import torch
    dummy = torch.zeros(4, dtype=torch.int32, device="cuda")
    dd = torch.zeros(4, dtype=torch.float64, device="cuda")
    p, pd = _p(dummy), _p(dd)
    rc = lib.lusp_trisolve_par_noalloc(MAX_N + 1, p, p, pd, p, p, pd, p, None, pd, pd, None)
    assert rc == 3
    assert b"LUSP_NOALLOC_MAX_N" in lib.lusp_last_error()
