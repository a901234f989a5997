"""CPU tests: the oracle restatement and the product's host analysis against
the reference's own outputs (golden fixtures from oracle/_ref), the
selector, COLAMD, the s0 readers, and the C-ABI symbol table."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from luspice_b200 import _lib, api, mna
from oracle import oracle as O

ROOT = Path(__file__).resolve().parent.parent
GOLD = ROOT / "tests" / "golden"


def _cases():
    d = np.load(GOLD / "ref_cases.npz")
    return d, [str(x) for x in d["names"]]


def _bits(a):
    a = np.asarray(a)
    return a.view(np.uint64) if a.dtype == np.float64 else a


@pytest.mark.parametrize("name", _cases()[1])
def test_oracle_lu_factor_matches_reference_golden(name):
    d, _ = _cases()
    n = int(d[f"{name}/n"][0])
    F = O.lu_factor(n, d[f"{name}/Ap"], d[f"{name}/Ai"], d[f"{name}/Ax"], d[f"{name}/q"], use_ref=False)
    assert F["status"] == int(d[f"{name}/status"][0])
    if F["status"] >= 0:
        return
    for k in ("pinv", "Lp", "Li", "Lx", "Up", "Ui", "Ux"):
        assert np.array_equal(_bits(F[k]), _bits(d[f"{name}/lu_{k}"])), k
    x = O.lu_solve(F, d[f"{name}/q"], d[f"{name}/b"])
    assert np.array_equal(_bits(x), _bits(d[f"{name}/x"]))
    lv, depth = O.levels(n, F["Up"], F["Ui"])
    assert np.array_equal(lv, d[f"{name}/levels"]) and depth == int(d[f"{name}/nlevels"][0])


@pytest.mark.parametrize("name", _cases()[1])
def test_oracle_dense_factor_matches_reference_golden(name):
    import scipy.sparse as sp
    d, _ = _cases()
    n = int(d[f"{name}/n"][0])
    q = d[f"{name}/q"]
    A = sp.csc_matrix((d[f"{name}/Ax"], d[f"{name}/Ai"], d[f"{name}/Ap"]), shape=(n, n))[:, q]
    A.sort_indices()
    D = O.dense_factor(n, A.indptr, A.indices, A.data, q)
    assert D["status"] == int(d[f"{name}/dense_status"][0])
    if D["status"] >= 0:
        return
    # symbolic_dense.c leaves L rows unpermuted; the kernel semantics remap them.
    pinv = d[f"{name}/dense_pinv"]
    assert np.array_equal(D["pinv"], pinv)
    assert np.array_equal(D["Li"], pinv[d[f"{name}/dense_Li"]])
    for k in ("Lp", "Up", "Ui"):
        assert np.array_equal(D[k], d[f"{name}/dense_{k}"]), k
    for k in ("Lx", "Ux"):
        assert np.array_equal(_bits(D[k]), _bits(d[f"{name}/dense_{k}"])), k


@pytest.mark.parametrize("name", _cases()[1])
def test_product_pivot_factor_matches_reference_golden(name):
    """The host analysis decides exactly the reference's P and L/U pattern."""
    d, _ = _cases()
    n = int(d[f"{name}/n"][0])
    F = api.pivot_factor(n, d[f"{name}/Ap"], d[f"{name}/Ai"], d[f"{name}/Ax"], d[f"{name}/q"])
    st = int(d[f"{name}/status"][0])
    if st >= 0:
        assert F["singular_col"] == st
        return
    for k in ("pinv", "Lp", "Li", "Lx", "Up", "Ui", "Ux"):
        assert np.array_equal(_bits(F[k]), _bits(d[f"{name}/lu_{k}"])), k


@pytest.mark.parametrize("name", _cases()[1])
def test_product_levels_match_reference_golden(name, lib):
    d, _ = _cases()
    if int(d[f"{name}/status"][0]) >= 0:
        return
    n = int(d[f"{name}/n"][0])
    Up, Ui = np.ascontiguousarray(d[f"{name}/lu_Up"]), np.ascontiguousarray(d[f"{name}/lu_Ui"])
    lv = np.zeros(n, np.int32)
    nl = C.c_int()
    assert lib.dsh_level_compute(n, _lib.ptr(Up, C.c_int), _lib.ptr(Ui, C.c_int), _lib.ptr(lv, C.c_int), C.byref(nl)) == 0
    assert np.array_equal(lv, d[f"{name}/levels"]) and nl.value == int(d[f"{name}/nlevels"][0])
    hist = np.zeros(nl.value, np.int32)
    lib.dsh_level_hist(n, _lib.ptr(lv, C.c_int), nl.value, _lib.ptr(hist, C.c_int))
    assert np.array_equal(hist, np.bincount(lv, minlength=nl.value))


@pytest.mark.parametrize("n,seed", [(300, 5), (989, 42), (2500, 7)])
def test_product_pivot_factor_matches_live_reference(n, seed):
    """Against the reference compiled here (skipped where it is absent)."""
    if not O.ref_available():
        pytest.skip("oracle/_ref not built on this machine")
    m = mna.analog(n, seed)
    vals = m.perturbed(1, seed)[0]
    q = api.colamd(m.n, m.Ap, m.Ai)
    R = O.lu_factor(m.n, m.Ap, m.Ai, vals, q, use_ref=True)
    F = api.pivot_factor(m.n, m.Ap, m.Ai, vals, q)
    Fo = O.lu_factor(m.n, m.Ap, m.Ai, vals, q, use_ref=False)
    for k in ("pinv", "Lp", "Li", "Lx", "Up", "Ui", "Ux"):
        assert np.array_equal(_bits(F[k]), _bits(R[k])), k
        assert np.array_equal(_bits(Fo[k]), _bits(R[k])), k


def test_power_grid_pivot_factor_matches_live_reference():
    if not O.ref_available():
        pytest.skip("oracle/_ref not built on this machine")
    m = mna.power_grid()
    q = api.colamd(m.n, m.Ap, m.Ai)
    R = O.lu_factor(m.n, m.Ap, m.Ai, m.Ax, q, use_ref=True)
    F = api.pivot_factor(m.n, m.Ap, m.Ai, m.Ax, q)
    for k in ("pinv", "Lp", "Li", "Ui"):
        assert np.array_equal(F[k], R[k]), k


def test_selector_matches_reference_golden(lib):
    g = np.load(GOLD / "selector.npz")
    for f, exp in zip(g["features"], g["outputs"]):
        mi = _lib.DshMatrixInfo(int(f[0]), int(f[1]), *[float(v) for v in f[2:9]], int(f[9]))
        cfg = _lib.DshConfig()
        lib.dsh_format_select(C.byref(mi), C.byref(cfg))
        got = [cfg.spmv_format, cfg.sigma, cfg.use_ruiz, cfg.use_shift, cfg.shift, cfg.factor_prec,
               cfg.ir_outer, cfg.ir_inner, cfg.ir_rtol, cfg.mp_path, cfg.pre_ruiz_hint, cfg.fp16_candidate]
        assert np.allclose(got, exp, rtol=0, atol=0), (f, got, exp)
    assert [lib.dsh_mp_escalate(i) for i in range(-1, 5)] == list(g["escalate"])
    assert lib.dsh_mp_name(0) == b"P-fast" and lib.dsh_fmt_name(1) == b"SELL-C-sigma32"


def test_selector_analyze_matches_numpy(lib):
    m = mna.analog(989, 42)
    A = m.csr()
    rp = A.indptr.astype(np.int32)
    mi = _lib.DshMatrixInfo()
    lib.dsh_matrix_analyze(m.n, A.nnz, _lib.ptr(rp, C.c_int), C.byref(mi))
    lens = np.diff(rp)
    assert mi.n == m.n and mi.nnz == A.nnz
    assert mi.max_rowlen == lens.max() and mi.p50_rowlen == np.sort(lens)[m.n // 2]
    assert abs(mi.avg_rowlen - lens.mean()) < 1e-12
    assert abs(mi.row_skew - lens.max() / lens.mean()) < 1e-12


def test_colamd_is_a_good_permutation():
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla
    for m in (mna.analog(989, 42), mna.power_grid(), mna.analog(3000, 3)):
        q = api.colamd(m.n, m.Ap, m.Ai)
        assert np.array_equal(np.sort(q), np.arange(m.n))
        F = api.pivot_factor(m.n, m.Ap, m.Ai, m.Ax, q)
        A = sp.csc_matrix((m.Ax, m.Ai, m.Ap), shape=(m.n, m.n))
        lu = sla.splu(A, permc_spec="COLAMD", diag_pivot_thresh=1.0)
        natural = api.pivot_factor(m.n, m.Ap, m.Ai, m.Ax, None)
        ours = F["lnnz"] + F["unnz"]
        # Fill comparable to SuperLU's COLAMD (run only as a yardstick) and
        # far below the natural order.
        assert ours <= 1.5 * (lu.L.nnz + lu.U.nnz), (m.name, ours, lu.L.nnz + lu.U.nnz)
        assert ours < natural["lnnz"] + natural["unnz"]


def test_colamd_dense_and_empty_columns_last():
    n = 40
    rng = np.random.default_rng(0)
    cols = []
    for c in range(n):
        if c == 7:
            rows = np.arange(n)                 # dense column (> 16 entries)
        elif c == 11:
            rows = np.array([], dtype=int)      # empty column
        else:
            rows = np.unique(np.r_[c, rng.integers(0, n, 3)])
        cols.append(rows)
    Ap = np.r_[0, np.cumsum([len(r) for r in cols])].astype(np.int32)
    Ai = np.concatenate(cols).astype(np.int32)
    q = api.colamd(n, Ap, Ai)
    assert q[-2] == 7 and q[-1] == 11


def test_s0_reader_roundtrip(tmp_path, lib):
    m = mna.analog(120, 3)
    A = m.csr()
    f = tmp_path / "a.s0"
    coo = A.tocoo()
    with open(f, "w") as fh:
        fh.write(f"n {m.n}\n")
        for r, c, v in zip(coo.row, coo.col, coo.data):
            fh.write(f"A {r + 1} {c + 1} {float(v)!r}\n")
    M = _lib.CSRMatrix()
    assert lib.read_s0_to_csr(str(f).encode(), C.byref(M)) == 0
    assert M.n == m.n and M.nnz == A.nnz
    rp = np.ctypeslib.as_array(M.rowptr, shape=(m.n + 1,)).copy()
    ci = np.ctypeslib.as_array(M.colidx, shape=(A.nnz,)).copy()
    vv = np.ctypeslib.as_array(M.values, shape=(A.nnz,)).copy()
    assert np.array_equal(rp, A.indptr) and np.array_equal(ci, A.indices) and np.array_equal(vv, A.data)
    lib.csr_free(C.byref(M))
    r = tmp_path / "b.rhs"
    r.write_text(f"n {m.n}\nRHS 1 2.5\nRHS {m.n} -1\n")
    x = np.zeros(m.n)
    assert lib.read_rhs(str(r).encode(), m.n, _lib.ptr(x, C.c_double)) == 0
    assert x[0] == 2.5 and x[-1] == -1 and np.count_nonzero(x) == 2
    assert lib.read_s0_to_csr(str(tmp_path / "missing").encode(), C.byref(M)) != 0


def test_every_declared_symbol_is_exported(lib):
    """Each function the public headers declare resolves in the library."""
    names = set()
    for h in (ROOT / "include").glob("*.h"):
        txt = h.read_text()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        txt = re.sub(r"#ifdef __CUDACC__.*?#endif", "", txt, flags=re.S)
        for mt in re.finditer(r"^[A-Za-z_][\w \*]*?\b([a-z_][a-z0-9_]*)\s*\(", txt, flags=re.M):
            name = mt.group(1)
            if name not in ("if", "sizeof", "LU_PAR_SHARED_BYTES"):
                names.add(name)
    assert len(names) > 40
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    # The CUDA kernel entry points of lu_gpu_par.h (C++ linkage) are exported too.
    import subprocess
    syms = subprocess.run(["nm", "-D", "--defined-only", str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    assert "lu_factor_par_kernel" in syms and "trisolve_par_kernel" in syms


def test_batch_opts_defaults_cover_every_field(lib):
    """lusp_batch_opts_default sets every field the Python mirror declares
    (the struct is mirrored field for field), the ladder off."""
    from luspice_b200 import api
    o = api.default_opts()
    assert o.ladder == 0 and o.ladder_slots == 0
    assert o.factor_shift == 0.0 and o.hard_shift == 1e-7
    assert o.krylov == 30 and o.rtol == 1e-10 and o.xtol == 1e-8
    s = _lib.ServerOpts()
    lib.lusp_server_opts_default(C.byref(s))
    assert s.escalate == 1 and s.solver.ladder == 0 and s.analysis_threads == 4


def test_generators_deterministic_and_sized():
    a, b = mna.analog(989, 42), mna.analog(989, 42)
    assert np.array_equal(a.Ai, b.Ai) and np.array_equal(a.Ax, b.Ax)
    assert a.n == 989 and a.meta["branches"] == 89 and a.meta["nodes"] == 900 and a.meta["mosfets"] == 150
    g = mna.power_grid()
    assert g.n == 4050
    v = g.perturbed(3, 1)
    assert v.shape == (3, g.nnz) and not np.array_equal(v[0], v[1])
    # Incidence entries of the pad rows do not move under perturbation.
    assert np.all(v[:, g.const != 0] == g.const[g.const != 0])
    sizes = mna.batch_sizes()
    assert sizes.size == 512 and sizes.min() >= 100 and sizes.max() <= 5000


def test_large_circuit_fp16_fraction():
    m = mna.large_circuit()
    assert m.n == 40000 and 180_000 <= m.nnz <= 260_000
    assert 0.04 <= m.meta["frac_below_fp16_normal"] <= 0.45
    lens = np.diff(m.csr().indptr)
    assert lens.max() >= 700          # supply rows


def test_library_fails_loudly_without_build(tmp_path, monkeypatch):
    import importlib
    from luspice_b200 import _lib as L
    monkeypatch.setattr(L, "_lib", None)
    with pytest.raises(RuntimeError):
        L.load(tmp_path / "nope.so")
    monkeypatch.setattr(L, "_lib", None)
    importlib.reload(L)


def test_reference_arm_column_order_fixture():
    """bench.py's reference arm reads the power grid's column order from a
    committed file (that process never loads the product library); the file
    is the library's COLAMD order of the same matrix."""
    q = np.load(ROOT / "oracle" / "power_grid_colamd_q.npy")
    m = mna.power_grid()
    assert np.array_equal(q, api.colamd(m.n, m.Ap, m.Ai))


def test_cpu_reference_solve_factors_once(monkeypatch):
    """ref_cpu_solve runs one factorization per solve (the timed CPU unit is
    one factor + one solve) and matches the restatement's answer."""
    if not O.ref_available():
        pytest.skip("compiled reference (oracle/_ref) not built")
    m = mna.analog(300, 3)
    q = api.colamd(m.n, m.Ap, m.Ai)
    lib = O.ref()
    calls = []
    real = lib.ref_lu_factor

    class Counting:
        def __call__(self, *a):
            calls.append(1)
            return real(*a)

    monkeypatch.setattr(lib, "ref_lu_factor", Counting())
    x = O.ref_cpu_solve(m.n, m.Ap, m.Ai, m.Ax, q, m.b)
    assert len(calls) == 1
    monkeypatch.undo()
    F = O.lu_factor(m.n, m.Ap, m.Ai, m.Ax, q, use_ref=False)
    assert np.array_equal(x.view(np.uint64), O.lu_solve(F, q, m.b).view(np.uint64))
