"""ctypes access to the checker libraries (TEST INFRASTRUCTURE ONLY).

liboracle.so   our C restatement of the reference path (oracle.c)
_ref/libluref.so  the reference's own sources compiled read-only (Makefile)

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_SO = HERE / "_ref" / "libluref.so"

ip = C.POINTER(C.c_int)
dp = C.POINTER(C.c_double)
lp = C.POINTER(C.c_long)

_orc = None
_ref = None


REF_ENV = "LUSPICE_REF_ROOT"


def build(ref_root: str | None = None) -> None:
    """Build liboracle.so, and _ref/ from the reference's sources.

    ref_root: the LUSpice source tree (default: the LUSPICE_REF_ROOT
    environment variable).  Without either, only the restatement is built and
    a message says why _ref/ was not (an existing _ref/ is kept)."""
    subprocess.run(["make", "-s", "oracle"], cwd=HERE, check=True)
    root = ref_root or os.environ.get(REF_ENV)
    if not root:
        print(f"oracle: {REF_ENV} is not set and no reference tree was given: "
              f"_ref/ (the reference compiled from its sources) not rebuilt", file=sys.stderr)
        return
    if not (Path(root) / "src" / "third_party" / "splu.h").is_file():
        raise FileNotFoundError(f"oracle: {root} is not a LUSpice source tree (no src/third_party/splu.h)")
    subprocess.run(["make", "-s", "ref", f"REF={root}"], cwd=HERE, check=True)


def _p(a, t):
    return None if a is None else a.ctypes.data_as(C.POINTER(t))


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORACLE_SO.exists():
            build(None)
        lib = C.CDLL(str(ORACLE_SO))
        lib.orc_lu_factor.restype = C.c_int
        lib.orc_lu_factor.argtypes = [C.c_int, ip, ip, dp, ip, C.c_double, ip, ip, ip, dp, C.c_long,
                                      ip, ip, dp, C.c_long, lp, lp]
        lib.orc_lu_solve.restype = None
        lib.orc_lu_solve.argtypes = [C.c_int, ip, ip, ip, dp, ip, ip, dp, ip, dp, dp]
        lib.orc_dense_factor.restype = C.c_int
        lib.orc_dense_factor.argtypes = [C.c_int, ip, ip, dp, ip, ip, ip, ip, dp, C.c_long,
                                         ip, ip, dp, C.c_long, lp, lp]
        lib.orc_levels.restype = C.c_int
        lib.orc_levels.argtypes = [C.c_int, ip, ip, ip]
        lib.orc_static_refactor.restype = C.c_int
        lib.orc_static_refactor.argtypes = [C.c_int, ip, ip, ip, ip, ip, ip, dp, C.c_int, dp]
        lib.orc_spmv_csr.restype = None
        lib.orc_spmv_csr.argtypes = [C.c_int, ip, ip, dp, dp, dp]
        lib.orc_gmres_ir.restype = C.c_int
        lib.orc_gmres_ir.argtypes = [C.c_int, ip, ip, dp, ip, ip, ip, dp, ip, ip, dp, ip, dp, dp,
                                     C.c_int, C.c_int, C.c_double, dp, ip]
        _orc = lib
    return _orc


def ref_available() -> bool:
    return REF_SO.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_SO))
        lib.ref_lu_factor.restype = C.c_void_p
        lib.ref_lu_factor.argtypes = [C.c_int, ip, ip, dp, ip, C.c_double]
        lib.ref_lu_status.restype = C.c_int
        lib.ref_lu_status.argtypes = [C.c_void_p]
        lib.ref_lu_lnnz.restype = C.c_long
        lib.ref_lu_lnnz.argtypes = [C.c_void_p]
        lib.ref_lu_unnz.restype = C.c_long
        lib.ref_lu_unnz.argtypes = [C.c_void_p]
        lib.ref_lu_get.restype = None
        lib.ref_lu_get.argtypes = [C.c_void_p, ip, ip, ip, dp, ip, ip, dp]
        lib.ref_lu_solve.restype = None
        lib.ref_lu_solve.argtypes = [C.c_void_p, ip, dp, dp]
        lib.ref_lu_free.restype = None
        lib.ref_lu_free.argtypes = [C.c_void_p]
        lib.cpu_lu_ref.restype = C.c_int
        lib.cpu_lu_ref.argtypes = [C.c_int, ip, ip, dp, ip, dp, C.c_double, dp, lp, lp]
        lib.dsh_level_compute.restype = C.c_int
        lib.dsh_level_compute.argtypes = [C.c_int, ip, ip, ip, ip]
        lib.symbolic_dense.restype = C.c_int
        lib.symbolic_dense.argtypes = [C.c_int, ip, ip, dp, ip] + [C.c_void_p] * 10
        lib.free.restype = None
        lib.free.argtypes = [C.c_void_p]
        _ref = lib
    return _ref


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def lu_factor(n, Ap, Ai, Ax, q=None, tol=1.0, use_ref=True):
    """splu lu_factor (compiled reference when available, else restatement).
    Returns dict(pinv, Lp, Li, Lx, Up, Ui, Ux, status)."""
    Ap, Ai, Ax = _i32(Ap), _i32(Ai), _f64(Ax)
    qq = None if q is None else _i32(q)
    if use_ref and ref_available():
        lib = ref()
        h = lib.ref_lu_factor(n, _p(Ap, C.c_int), _p(Ai, C.c_int), _p(Ax, C.c_double), _p(qq, C.c_int), tol)
        st = lib.ref_lu_status(h)
        if st >= 0:
            lib.ref_lu_free(h)
            return {"status": st}
        ln, un = lib.ref_lu_lnnz(h), lib.ref_lu_unnz(h)
        out = {"pinv": np.empty(n, np.int32), "Lp": np.empty(n + 1, np.int32), "Li": np.empty(ln, np.int32),
               "Lx": np.empty(ln), "Up": np.empty(n + 1, np.int32), "Ui": np.empty(un, np.int32),
               "Ux": np.empty(un), "status": -1}
        lib.ref_lu_get(h, *[_p(out[k], C.c_int if out[k].dtype == np.int32 else C.c_double)
                            for k in ("pinv", "Lp", "Li", "Lx", "Up", "Ui", "Ux")])
        lib.ref_lu_free(h)
        return out
    lib = orc()
    cap = 4 * int(Ap[-1]) + 16 * n + 64
    while True:
        out = {"pinv": np.empty(n, np.int32), "Lp": np.empty(n + 1, np.int32), "Li": np.empty(cap, np.int32),
               "Lx": np.empty(cap), "Up": np.empty(n + 1, np.int32), "Ui": np.empty(cap, np.int32),
               "Ux": np.empty(cap)}
        ln, un = C.c_long(), C.c_long()
        st = lib.orc_lu_factor(n, _p(Ap, C.c_int), _p(Ai, C.c_int), _p(Ax, C.c_double), _p(qq, C.c_int), tol,
                               _p(out["pinv"], C.c_int), _p(out["Lp"], C.c_int), _p(out["Li"], C.c_int),
                               _p(out["Lx"], C.c_double), cap, _p(out["Up"], C.c_int), _p(out["Ui"], C.c_int),
                               _p(out["Ux"], C.c_double), cap, C.byref(ln), C.byref(un))
        if st == -2:
            cap *= 2
            continue
        if st >= 0:
            return {"status": st}
        for k, v in (("Li", ln.value), ("Lx", ln.value), ("Ui", un.value), ("Ux", un.value)):
            out[k] = out[k][:v]
        out["status"] = -1
        return out


def lu_solve(F, q, b, use_ref_handle=None):
    n = F["pinv"].size
    x = np.empty(n)
    b = _f64(b)
    qq = None if q is None else _i32(q)
    orc().orc_lu_solve(n, _p(F["pinv"], C.c_int), _p(F["Lp"], C.c_int), _p(F["Li"], C.c_int),
                       _p(F["Lx"], C.c_double), _p(F["Up"], C.c_int), _p(F["Ui"], C.c_int),
                       _p(F["Ux"], C.c_double), _p(qq, C.c_int), _p(b, C.c_double), _p(x, C.c_double))
    return x


def ref_cpu_solve(n, Ap, Ai, Ax, q, b, tol=1.0):
    """The reference's CPU path (src/cpu_ref_lu.c:15-58): one lu_factor, then
    lu_solve_perm with the same factors, with a modest initial capacity
    instead of cpu_ref_lu.c's n*n slots.  The compiled reference when it is
    built, else the restatement.  Returns x, or None if singular."""
    Ap, Ai, Ax, bb = _i32(Ap), _i32(Ai), _f64(Ax), _f64(b)
    qq = None if q is None else _i32(q)
    if ref_available():
        lib = ref()
        h = lib.ref_lu_factor(n, _p(Ap, C.c_int), _p(Ai, C.c_int), _p(Ax, C.c_double), _p(qq, C.c_int), tol)
        try:
            if lib.ref_lu_status(h) >= 0:
                return None
            x = np.empty(n)
            lib.ref_lu_solve(h, _p(qq, C.c_int), _p(bb, C.c_double), _p(x, C.c_double))
            return x
        finally:
            lib.ref_lu_free(h)
    F = lu_factor(n, Ap, Ai, Ax, q, tol, use_ref=False)
    if F["status"] >= 0:
        return None
    return lu_solve(F, q, bb)


def dense_factor(n, Ap, Ai, Ax, diagrow):
    """Dense-scan single-thread semantics (lu_gpu.cu / symbolic_dense.c)."""
    Ap, Ai, Ax, dr = _i32(Ap), _i32(Ai), _f64(Ax), _i32(diagrow)
    cap = max(4 * int(Ap[-1]) + 16 * n + 64, 1024)
    lib = orc()
    while True:
        out = {"pinv": np.empty(n, np.int32), "Lp": np.empty(n + 1, np.int32), "Li": np.empty(cap, np.int32),
               "Lx": np.empty(cap), "Up": np.empty(n + 1, np.int32), "Ui": np.empty(cap, np.int32),
               "Ux": np.empty(cap)}
        ln, un = C.c_long(), C.c_long()
        st = lib.orc_dense_factor(n, _p(Ap, C.c_int), _p(Ai, C.c_int), _p(Ax, C.c_double), _p(dr, C.c_int),
                                  _p(out["pinv"], C.c_int), _p(out["Lp"], C.c_int), _p(out["Li"], C.c_int),
                                  _p(out["Lx"], C.c_double), cap, _p(out["Up"], C.c_int), _p(out["Ui"], C.c_int),
                                  _p(out["Ux"], C.c_double), cap, C.byref(ln), C.byref(un))
        if st == -2:
            cap *= 2
            continue
        out["status"] = st
        if st < 0:
            for k, v in (("Li", ln.value), ("Lx", ln.value), ("Ui", un.value), ("Ux", un.value)):
                out[k] = out[k][:v]
        return out


def levels(n, Up, Ui):
    lv = np.zeros(n, np.int32)
    depth = orc().orc_levels(n, _p(_i32(Up), C.c_int), _p(_i32(Ui), C.c_int), _p(lv, C.c_int))
    return lv, depth


def static_refactor(n, cp, ri, dg, a_ptr, a_src, a_dst, a_val, fp32):
    cap = int(cp[-1])
    vals = np.empty(cap)
    bad = orc().orc_static_refactor(n, _p(_i32(cp), C.c_int), _p(_i32(ri), C.c_int), _p(_i32(dg), C.c_int),
                                    _p(_i32(a_ptr), C.c_int), _p(_i32(a_src), C.c_int), _p(_i32(a_dst), C.c_int),
                                    _p(_f64(a_val), C.c_double), 1 if fp32 else 0, _p(vals, C.c_double))
    return vals, bad


def gmres_ir(n, rp, ci, av, F, q, b, m=30, max_outer=3, rtol=1e-10):
    x = np.empty(n)
    res = np.zeros(max_outer + 1)
    nres = C.c_int()
    b = _f64(b)
    qq = None if q is None else _i32(q)
    it = orc().orc_gmres_ir(n, _p(_i32(rp), C.c_int), _p(_i32(ci), C.c_int), _p(_f64(av), C.c_double),
                            _p(F["pinv"], C.c_int), _p(F["Lp"], C.c_int), _p(F["Li"], C.c_int),
                            _p(F["Lx"], C.c_double), _p(F["Up"], C.c_int), _p(F["Ui"], C.c_int),
                            _p(F["Ux"], C.c_double), _p(qq, C.c_int), _p(b, C.c_double), _p(x, C.c_double),
                            m, max_outer, rtol, _p(res, C.c_double), C.byref(nres))
    return x, it, res[: nres.value]
