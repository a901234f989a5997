"""Reference-API kernels (lu_gpu_par.h, spmv.h) and the standalone SELL
SpMV against the oracle, on the GPU."""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

from luspice_b200 import api, mna
from oracle import oracle as O
from tests.helpers import FP16_MIN_NORMAL, ruiz_scaling

pytestmark = pytest.mark.gpu


def _dev(torch, a, dtype):
    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _p(t):
    return C.c_void_p(t.data_ptr())


def _qcsc(m, q):
    """q-ordered CSC with original row indices (build_csc_q, unsorted rows)."""
    A = sp.csc_matrix((m.Ax, m.Ai, m.Ap), shape=(m.n, m.n))[:, q]
    A.sort_indices()
    return A


@pytest.mark.parametrize("n,seed", [(60, 1), (300, 2), (989, 42)])
def test_lu_factor_par_kernel_bitwise(gpu, lib, n, seed):
    import torch
    m = mna.analog(n, seed)
    q = api.colamd(m.n, m.Ap, m.Ai)
    A = _qcsc(m, q)
    exp = O.dense_factor(m.n, A.indptr, A.indices, A.data, q)
    assert exp["status"] == -1
    cap = int(max(exp["Lp"][-1], exp["Up"][-1])) + 64
    Ap, Ai, Ax = _dev(torch, A.indptr, torch.int32), _dev(torch, A.indices, torch.int32), _dev(torch, A.data, torch.float64)
    dr = _dev(torch, q, torch.int32)
    Lp = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    Up = torch.zeros(n + 1, dtype=torch.int32, device="cuda")
    Li = torch.zeros(cap, dtype=torch.int32, device="cuda")
    Ui = torch.zeros(cap, dtype=torch.int32, device="cuda")
    Lx = torch.zeros(cap, dtype=torch.float64, device="cuda")
    Ux = torch.zeros(cap, dtype=torch.float64, device="cuda")
    pinv = torch.zeros(n, dtype=torch.int32, device="cuda")
    xi = torch.zeros(n + 2 * 1024, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(3, dtype=torch.int32, device="cuda")
    rc = lib.lusp_lu_factor_par_launch(n, _p(Ap), _p(Ai), _p(Ax), _p(dr), _p(Lp), _p(Li), _p(Lx), cap,
                                       _p(Up), _p(Ui), _p(Ux), cap, _p(pinv), _p(xi), None,
                                       C.c_void_p(cnt.data_ptr()), C.c_void_p(cnt.data_ptr() + 4),
                                       C.c_void_p(cnt.data_ptr() + 8), None)
    assert rc == 0
    torch.cuda.synchronize()
    ln, un, sing = cnt.cpu().tolist()
    assert sing == -1
    assert ln == exp["Lp"][-1] and un == exp["Up"][-1]
    for k in ("Lp", "Up", "pinv"):
        assert np.array_equal(locals()[k].cpu().numpy(), exp[k]), k
    assert np.array_equal(Li[:ln].cpu().numpy(), exp["Li"])
    assert np.array_equal(Ui[:un].cpu().numpy(), exp["Ui"])
    assert np.array_equal(Lx[:ln].cpu().numpy().view(np.uint64), exp["Lx"].view(np.uint64))
    assert np.array_equal(Ux[:un].cpu().numpy().view(np.uint64), exp["Ux"].view(np.uint64))
    # trisolve_par_kernel on these factors equals the host column solve bitwise.
    b = np.random.default_rng(seed).standard_normal(n)
    xh = O.lu_solve(exp, q, b)
    db, dx = _dev(torch, b, torch.float64), torch.zeros(n, dtype=torch.float64, device="cuda")
    wi = torch.zeros(n, dtype=torch.int32, device="cuda")
    wd = torch.zeros(2 * n, dtype=torch.float64, device="cuda")
    dq = _dev(torch, q, torch.int32)
    rc = lib.lusp_trisolve_par_launch(n, _p(Lp), _p(Li), _p(Lx), _p(Up), _p(Ui), _p(Ux), _p(pinv), _p(dq),
                                      _p(db), _p(dx), _p(wi), _p(wd), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert np.array_equal(dx.cpu().numpy().view(np.uint64), xh.view(np.uint64))


def test_spmv_launch_csr(gpu, lib):
    import torch
    m = mna.analog(3000, 5)
    A = m.csr()
    x = np.random.default_rng(0).standard_normal(m.n)
    rp, ci, v = _dev(torch, A.indptr, torch.int32), _dev(torch, A.indices, torch.int32), _dev(torch, A.data, torch.float64)
    dx, dy = _dev(torch, x, torch.float64), torch.zeros(m.n, dtype=torch.float64, device="cuda")
    lib.spmv_launch(m.n, _p(rp), _p(ci), _p(v), _p(dx), _p(dy), None)
    torch.cuda.synchronize()
    y = A @ x
    assert np.allclose(dy.cpu().numpy(), y, rtol=1e-13, atol=1e-13 * np.abs(y).max())


@pytest.mark.parametrize("Cc", [8, 16, 32])
@pytest.mark.parametrize("sigma", [32, 256, 1024])
@pytest.mark.parametrize("kind", ["fp64", "fp32"])
def test_sell_spmv(gpu, Cc, sigma, kind):
    import torch
    m = mna.analog(2000, 8)
    A = m.csr()
    x = np.random.default_rng(1).standard_normal(m.n)
    S = api.Sell(m.n, A.indptr, A.indices, A.data, Cc, sigma, kind)
    dx, dy = _dev(torch, x, torch.float64), torch.full((m.n,), np.nan, dtype=torch.float64, device="cuda")
    S.spmv(dx.data_ptr(), dy.data_ptr())
    torch.cuda.synchronize()
    if kind == "fp64":
        ref = A @ x
        tol = 1e-13
    else:
        ref = sp.csr_matrix((A.data.astype(np.float32).astype(np.float64), A.indices, A.indptr), shape=A.shape) @ x
        tol = 1e-12
    y = dy.cpu().numpy()
    assert np.all(np.abs(y - ref) <= tol * (np.abs(A) @ np.abs(x)) + 1e-300)


def test_sell_fp16_ruiz(gpu):
    """fp16 SELL values on the n = 4050 power grid, whose Ruiz-scaled range
    fits the fp16 normal range: sell_kernel<C, __half> against a host SpMV
    on the same fp16-rounded scaled values (only the summation order
    differs), and against the exact product within the fp16 storage bound
    (each stored value within 2^-11 of the scaled entry)."""
    import torch
    m = mna.power_grid()
    A = m.csr()
    n = m.n
    rows = np.repeat(np.arange(n), np.diff(A.indptr))
    assert A.nnz == m.nnz                      # no duplicate entries: same entries as the CSC
    r, c, _, _ = ruiz_scaling(n, m.Ap, m.Ai, m.Ax)
    scaled = A.data * r[rows] * c[A.indices]
    assert np.abs(scaled).min() >= FP16_MIN_NORMAL and np.abs(scaled).max() <= 65504.0
    h = scaled.astype(np.float16).astype(np.float64)
    for Cc in (32, 16, 8):
        S = api.Sell(n, A.indptr, A.indices, A.data, Cc, 256, "fp16")
        for seed in (2, 3):
            x = np.random.default_rng(seed).standard_normal(n)
            dx = _dev(torch, x, torch.float64)
            dy = torch.full((n,), np.nan, dtype=torch.float64, device="cuda")
            S.spmv(dx.data_ptr(), dy.data_ptr())
            torch.cuda.synchronize()
            y = dy.cpu().numpy()
            xs = x / c
            ref16 = (sp.csr_matrix((h, A.indices, A.indptr), shape=A.shape) @ xs) / r
            mag16 = (sp.csr_matrix((np.abs(h), A.indices, A.indptr), shape=A.shape) @ np.abs(xs)) / r
            assert np.all(np.abs(y - ref16) <= 1e-13 * mag16 + 1e-300), (Cc, seed)
            exact = A @ x
            assert np.all(np.abs(y - exact) <= 2.0 ** -10 * (np.abs(A) @ np.abs(x)) + 1e-300), (Cc, seed)
            assert np.linalg.norm(y - exact) / np.linalg.norm(exact) <= 1e-3
        S.close()


def test_sell_fp16_refused_outside_fp16_range(gpu):
    """An analog circuit (gmin 1e-12 beside 1e-1 conductances): the scaled
    values cannot all be fp16 normals, so the fp16 SELL is refused."""
    m = mna.analog(1500, 4)
    A = m.csr()
    r, c, rows, cols = ruiz_scaling(m.n, m.Ap, m.Ai, m.Ax)
    s = np.abs(m.Ax * r[rows] * c[cols])
    assert s[s != 0].min() < FP16_MIN_NORMAL
    with pytest.raises(api.LuspError, match="fp16 normal range"):
        api.Sell(m.n, A.indptr, A.indices, A.data, 32, 256, "fp16")


def test_csr_spmv32(gpu, lib):
    import torch
    m = mna.analog(3000, 6)
    A = m.csr()
    x = np.random.default_rng(3).standard_normal(m.n)
    rp, ci = _dev(torch, A.indptr, torch.int32), _dev(torch, A.indices, torch.int32)
    v32 = _dev(torch, A.data.astype(np.float32), torch.float32)
    dx, dy = _dev(torch, x, torch.float64), torch.zeros(m.n, dtype=torch.float64, device="cuda")
    assert lib.lusp_csr_spmv32(m.n, _p(rp), _p(ci), _p(v32), _p(dx), _p(dy), None) == 0
    torch.cuda.synchronize()
    ref = sp.csr_matrix((A.data.astype(np.float32).astype(np.float64), A.indices, A.indptr), shape=A.shape) @ x
    assert np.all(np.abs(dy.cpu().numpy() - ref) <= 1e-12 * (np.abs(A) @ np.abs(x)) + 1e-300)


def test_large_circuit_spmv_variants(gpu, lib):
    """n = 40,000 with supply rows: fp64/fp32 CSR and SELL agree with the host
    product; fp16 is refused because the scaled range does not fit."""
    import torch
    m = mna.large_circuit()
    A = m.csr()
    x = np.random.default_rng(4).standard_normal(m.n)
    ref = A @ x
    scale = np.abs(A) @ np.abs(x)
    dx = _dev(torch, x, torch.float64)
    for kind, tol in (("fp64", 1e-13), ("fp32", 1e-6)):
        S = api.Sell(m.n, A.indptr, A.indices, A.data, 32, 256, kind)
        dy = torch.zeros(m.n, dtype=torch.float64, device="cuda")
        S.spmv(dx.data_ptr(), dy.data_ptr())
        torch.cuda.synchronize()
        assert np.all(np.abs(dy.cpu().numpy() - ref) <= tol * scale + 1e-300), kind
    with pytest.raises(api.LuspError):
        api.Sell(m.n, A.indptr, A.indices, A.data, 32, 256, "fp16")
