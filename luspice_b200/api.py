"""Python host wrapper over the lusp_* C-ABI (luspice_b200.h).

Patterns, batches and the standalone SELL SpMV as Python objects; every call
goes through libluspice_b200.so.  Streams are raw cudaStream_t handles
(e.g. torch.cuda.Stream().cuda_stream) or None for the default stream.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib as L

MIXED, FP64 = 0, 1
RUN_REFACTOR, RUN_SOLVE, RUN_BOTH, RUN_DIRECT = 1, 2, 3, 4

ST_SINGULAR, ST_PIVOT_WEAK, ST_STAGNATED, ST_NOT_CONVERGED = 1, 2, 4, 8
ST_NONFINITE, ST_WAIT_TIMEOUT, ST_CAPACITY, ST_ESCALATED = 16, 32, 64, 128
ST_SHIFTED, ST_LADDER_FULL, ST_FP16_OFF = 256, 512, 1024
INNER_FP32, INNER_FP64, INNER_FP16 = 0, 1, 2
# Device-side escalation ladder (Batch(..., ladder=...)): rungs after a failed
# mixed solve, inside the same launch.
LADDER_OFF, LADDER_SAFE, LADDER_HARD, LADDER_SAFE_HARD = 0, 1, 2, 3
ST_FAIL_MASK = ST_SINGULAR | ST_STAGNATED | ST_NOT_CONVERGED | ST_NONFINITE | ST_WAIT_TIMEOUT | ST_CAPACITY


class LuspError(RuntimeError):
    def __init__(self, rc: int, what: str):
        lib = L.load()
        msg = lib.lusp_last_error().decode(errors="replace")
        super().__init__(f"{what}: rc={rc} {msg}")
        self.rc = rc


def _check(rc: int, what: str) -> None:
    if rc != 0:
        raise LuspError(rc, what)


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.int32)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def _stream(s) -> C.c_void_p:
    if s is None:
        return None
    if hasattr(s, "cuda_stream"):
        return C.c_void_p(s.cuda_stream)
    return C.c_void_p(int(s))


class Pattern:
    """Host analysis + device-resident static layout of one sparsity pattern."""

    def __init__(self, n: int, Ap, Ai, Ax, q=None, dense_tail: int = -1):
        """dense_tail: trailing columns factored and solved as one dense
        block (-1 chosen by the library's cost model, 0 none)."""
        lib = L.load()
        self.n = int(n)
        self._Ap, self._Ai, self._Ax = _i32(Ap), _i32(Ai), _f64(Ax)
        qq = None if q is None else _i32(q)
        h = C.c_void_p()
        rc = lib.lusp_pattern_create_ex(self.n, L.ptr(self._Ap, C.c_int), L.ptr(self._Ai, C.c_int),
                                        L.ptr(self._Ax, C.c_double), L.ptr(qq, C.c_int), int(dense_tail),
                                        C.byref(h))
        _check(rc, "lusp_pattern_create")
        self.handle = h
        info = L.PatternInfo()
        _check(lib.lusp_pattern_get_info(h, C.byref(info)), "lusp_pattern_get_info")
        self.info = {k: getattr(info, k) for k, _ in L.PatternInfo._fields_}

    @classmethod
    def from_matrix(cls, m, q=None, values=None, dense_tail: int = -1):
        return cls(m.n, m.Ap, m.Ai, m.Ax if values is None else values, q, dense_tail)

    def perm(self) -> tuple[np.ndarray, np.ndarray]:
        pinv = np.empty(self.n, np.int32)
        q = np.empty(self.n, np.int32)
        _check(L.load().lusp_pattern_get_perm(self.handle, L.ptr(pinv, C.c_int), L.ptr(q, C.c_int)), "perm")
        return pinv, q

    def structure(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        cp = np.empty(self.n + 1, np.int32)
        ri = np.empty(self.info["cap"], np.int32)
        dg = np.empty(self.n, np.int32)
        _check(L.load().lusp_pattern_get_structure(self.handle, L.ptr(cp, C.c_int), L.ptr(ri, C.c_int),
                                                   L.ptr(dg, C.c_int)), "structure")
        return cp, ri, dg

    def levels(self) -> np.ndarray:
        lv = np.empty(self.n, np.int32)
        _check(L.load().lusp_pattern_get_levels(self.handle, L.ptr(lv, C.c_int)), "levels")
        return lv

    def close(self) -> None:
        if getattr(self, "handle", None):
            L.load().lusp_pattern_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def default_opts() -> L.BatchOpts:
    o = L.BatchOpts()
    L.load().lusp_batch_opts_default(C.byref(o))
    return o


class Batch:
    """N systems refactored and solved by one persistent launch."""

    def __init__(self, patterns: Sequence[Pattern], prec: int = MIXED, **opts):
        lib = L.load()
        o = default_opts()
        o.prec = prec
        for k, v in opts.items():
            if not hasattr(o, k):
                raise TypeError(f"unknown batch option {k}")
            setattr(o, k, v)
        self.opts = o
        self.patterns = list(patterns)
        arr = (C.c_void_p * len(self.patterns))(*[p.handle for p in self.patterns])
        h = C.c_void_p()
        _check(lib.lusp_batch_create(len(self.patterns), arr, C.byref(o), C.byref(h)), "lusp_batch_create")
        self.handle = h
        self.nsys = len(self.patterns)
        self.sizes = np.array([p.n for p in self.patterns], dtype=np.int64)
        self.nnzs = np.array([p.info["nnz_a"] for p in self.patterns], dtype=np.int64)

    def set_params(self, **opts) -> None:
        for k, v in opts.items():
            setattr(self.opts, k, v)
        _check(L.load().lusp_batch_set_params(self.handle, C.byref(self.opts)), "set_params")

    def upload(self, values=None, rhs=None, stream=None) -> None:
        v = None if values is None else _f64(np.concatenate([np.ravel(a) for a in values])
                                             if isinstance(values, (list, tuple)) else np.ravel(values))
        b = None if rhs is None else _f64(np.concatenate([np.ravel(a) for a in rhs])
                                          if isinstance(rhs, (list, tuple)) else np.ravel(rhs))
        if v is not None and v.size != self.nnzs.sum():
            raise ValueError("values size mismatch")
        if b is not None and b.size != self.sizes.sum():
            raise ValueError("rhs size mismatch")
        self._keep = (v, b)  # host buffers must outlive asynchronous copies
        _check(L.load().lusp_batch_upload(self.handle, L.ptr(v, C.c_double), L.ptr(b, C.c_double),
                                          _stream(stream)), "upload")

    def run(self, what: int = RUN_BOTH, stream=None, graph: bool = False) -> None:
        lib = L.load()
        fn = lib.lusp_batch_run_graph if graph else lib.lusp_batch_run
        _check(fn(self.handle, what, _stream(stream)), "run")

    def download(self, out: np.ndarray | None = None, stream=None) -> np.ndarray:
        x = np.empty(int(self.sizes.sum())) if out is None else out
        _check(L.load().lusp_batch_download(self.handle, L.ptr(x, C.c_double), _stream(stream)), "download")
        return x

    def split(self, flat: np.ndarray) -> list[np.ndarray]:
        return np.split(flat, np.cumsum(self.sizes)[:-1])

    def stats(self, stream=None) -> list[dict]:
        arr = (L.SysStats * self.nsys)()
        _check(L.load().lusp_batch_stats(self.handle, arr, _stream(stream)), "stats")
        out = []
        for s in arr:
            d = {k: getattr(s, k) for k, _ in L.SysStats._fields_ if k not in ("res", "pad_")}
            d["res"] = [s.res[i] for i in range(min(max(s.nres, 0), 16))]
            out.append(d)
        return out

    def factor_values(self, sys: int, stream=None) -> np.ndarray:
        cap = self.patterns[sys].info["cap"]
        out = np.empty(cap, np.float32 if self.opts.prec == MIXED else np.float64)
        _check(L.load().lusp_batch_factor_values(self.handle, sys, out.ctypes.data_as(C.c_void_p),
                                                 _stream(stream)), "factor_values")
        return out

    def device_ptrs(self, sys: int) -> tuple[int, int, int]:
        a, b, x = C.c_void_p(), C.c_void_p(), C.c_void_p()
        _check(L.load().lusp_batch_device_ptrs(self.handle, sys, C.byref(a), C.byref(b), C.byref(x)), "ptrs")
        return a.value, b.value, x.value

    def launch_count(self) -> int:
        return L.load().lusp_batch_launch_count(self.handle)

    def time_kernels(self, on: bool = True) -> None:
        """Record CUDA events around each kernel of later run() calls
        (graph=False)."""
        _check(L.load().lusp_batch_time_kernels(self.handle, int(on)), "time_kernels")

    def kernel_ms(self) -> dict:
        """Device times (ms) of the last timed run's refactor, dense-block and
        solve kernels."""
        ms = (C.c_float * 3)()
        _check(L.load().lusp_batch_kernel_ms(self.handle, ms), "kernel_ms")
        return {"refactor": ms[0], "dense": ms[1], "solve": ms[2]}

    def launch_shape(self) -> dict:
        """The launch shape the library chose for this batch."""
        v = (C.c_int * 10)()
        _check(L.load().lusp_batch_launch_shape(self.handle, v), "launch_shape")
        keys = ("refactor_grid", "refactor_block", "refactor_cluster", "refactor_spread", "dense_grid",
                "dense_block", "solve_grid", "solve_block", "sweeps", "dense_cluster")
        return dict(zip(keys, list(v)))

    def close(self) -> None:
        if getattr(self, "handle", None):
            L.load().lusp_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Sell:
    """Standalone SELL-C-sigma SpMV over a 0-based CSR matrix."""

    KINDS = {"fp64": 0, "fp32": 1, "fp16": 2}

    def __init__(self, n, rowptr, colidx, vals, C_: int = 32, sigma: int = 256, kind: str = "fp32"):
        lib = L.load()
        self.n = int(n)
        rp, ci, v = _i32(rowptr), _i32(colidx), _f64(vals)
        h = C.c_void_p()
        _check(lib.lusp_sell_create(self.n, L.ptr(rp, C.c_int), L.ptr(ci, C.c_int), L.ptr(v, C.c_double),
                                    C_, sigma, self.KINDS[kind], C.byref(h)), "lusp_sell_create")
        self.handle = h
        st, nz, mn, mx = C.c_long(), C.c_long(), C.c_double(), C.c_double()
        lib.lusp_sell_info(h, C.byref(st), C.byref(nz), C.byref(mn), C.byref(mx))
        self.stored, self.nnz, self.scaled_min, self.scaled_max = st.value, nz.value, mn.value, mx.value

    def spmv(self, d_x: int, d_y: int, stream=None) -> None:
        _check(L.load().lusp_sell_spmv(self.handle, C.c_void_p(d_x), C.c_void_p(d_y), _stream(stream)), "spmv")

    def close(self) -> None:
        if getattr(self, "handle", None):
            L.load().lusp_sell_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (lusp_server_*)."""

    def __init__(self, prec: int = MIXED, **opts):
        lib = L.load()
        o = L.ServerOpts()
        lib.lusp_server_opts_default(C.byref(o))
        o.solver.prec = prec
        for k, v in opts.items():
            if hasattr(o, k):
                setattr(o, k, v)
            elif hasattr(o.solver, k):
                setattr(o.solver, k, v)
            else:
                raise TypeError(f"unknown server option {k}")
        h = C.c_void_p()
        _check(lib.lusp_server_create(C.byref(o), C.byref(h)), "lusp_server_create")
        self.handle = h
        self.sizes = {}

    def submit(self, n, Ap, Ai, Ax, b) -> int:
        Ap, Ai, Ax, b = _i32(Ap), _i32(Ai), _f64(Ax), _f64(b)
        rid = L.load().lusp_serve_submit(self.handle, int(n), L.ptr(Ap, C.c_int), L.ptr(Ai, C.c_int),
                                         L.ptr(Ax, C.c_double), L.ptr(b, C.c_double))
        if rid < 0:
            raise LuspError(-rid, "lusp_serve_submit")
        self.sizes[rid] = int(n)
        return rid

    def poll(self, rid: int, wait_ms: int = -1):
        """(x, result dict) when done, None while running."""
        n = self.sizes[rid]
        x = np.empty(n)
        r = L.ServeResult()
        rc = L.load().lusp_serve_poll(self.handle, rid, L.ptr(x, C.c_double), C.byref(r), wait_ms)
        if rc == 6:
            return None
        _check(rc, "lusp_serve_poll")
        del self.sizes[rid]
        return x, {k: getattr(r, k) for k, _ in L.ServeResult._fields_ if k != "pad_"}

    def stats(self) -> dict:
        st = L.ServerStats()
        _check(L.load().lusp_server_get_stats(self.handle, C.byref(st)), "stats")
        return {k: getattr(st, k) for k, _ in L.ServerStats._fields_}

    def close(self) -> None:
        if getattr(self, "handle", None):
            L.load().lusp_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def colamd(n: int, Ap, Ai, knob_row: float = 0.0, knob_col: float = 0.0) -> np.ndarray:
    Ap, Ai = _i32(Ap), _i32(Ai)
    q = np.empty(n, np.int32)
    _check(L.load().lusp_colamd(n, n, L.ptr(Ap, C.c_int), L.ptr(Ai, C.c_int), knob_row, knob_col,
                                L.ptr(q, C.c_int)), "lusp_colamd")
    return q


def pivot_factor(n: int, Ap, Ai, Ax, q=None, tol: float = 1.0) -> dict:
    """Host pivoting LU in splu layout (the analysis step of pattern creation)."""
    lib = L.load()
    Ap, Ai, Ax = _i32(Ap), _i32(Ai), _f64(Ax)
    qq = None if q is None else _i32(q)
    ln, un, sc = C.c_long(), C.c_long(), C.c_int()
    pinv = np.empty(n, np.int32)
    Lp = np.empty(n + 1, np.int32)
    Up = np.empty(n + 1, np.int32)
    args = lambda Li, Lx, Ui, Ux, cap: (n, L.ptr(Ap, C.c_int), L.ptr(Ai, C.c_int), L.ptr(Ax, C.c_double),
                                        L.ptr(qq, C.c_int), tol, L.ptr(pinv, C.c_int), L.ptr(Lp, C.c_int),
                                        L.ptr(Li, C.c_int), L.ptr(Lx, C.c_double), cap, L.ptr(Up, C.c_int),
                                        L.ptr(Ui, C.c_int), L.ptr(Ux, C.c_double), cap, C.byref(ln),
                                        C.byref(un), C.byref(sc))
    rc = lib.lusp_pivot_factor(*args(None, None, None, None, 0))
    if rc == 1:
        return {"singular_col": sc.value}
    if rc not in (0, 2):
        _check(rc, "lusp_pivot_factor")
    cap = max(ln.value, un.value)
    Li, Ui = np.empty(cap, np.int32), np.empty(cap, np.int32)
    Lx, Ux = np.empty(cap), np.empty(cap)
    _check(lib.lusp_pivot_factor(*args(Li, Lx, Ui, Ux, cap)), "lusp_pivot_factor")
    return {"singular_col": -1, "pinv": pinv, "Lp": Lp, "Li": Li[:ln.value], "Lx": Lx[:ln.value],
            "Up": Up, "Ui": Ui[:un.value], "Ux": Ux[:un.value], "lnnz": ln.value, "unnz": un.value}


def autotune(m, nsys: int, prec: int = MIXED, **opts) -> dict:
    """Measure candidate configurations for nsys copies of matrix m (an
    MNAMatrix-like object with n, Ap, Ai, Ax, b) on this GPU; returns the
    fastest as {"dense_tail": D, "opts": {...}, "ms": t}: build the pattern
    with Pattern(..., dense_tail=D) and the batch with **opts."""
    lib = L.load()
    o = default_opts()
    o.prec = prec
    for k, v in opts.items():
        setattr(o, k, v)
    Ap, Ai, Ax, b = _i32(m.Ap), _i32(m.Ai), _f64(m.Ax), _f64(m.b)
    d, ms = C.c_int(), C.c_double()
    _check(lib.lusp_tune(int(m.n), L.ptr(Ap, C.c_int), L.ptr(Ai, C.c_int), L.ptr(Ax, C.c_double),
                         L.ptr(b, C.c_double), int(nsys), C.byref(o), C.byref(d), C.byref(ms)), "lusp_tune")
    keys = ("refactor_threads", "refactor_cluster", "block_threads", "ctas_per_sm", "solve_sweep")
    return {"dense_tail": d.value, "opts": {k: getattr(o, k) for k in keys}, "ms": ms.value}


def sell_tune(n, rowptr, colidx, vals, kind: str = "fp32") -> dict:
    """Fastest SELL (C, sigma) for this CSR matrix: {"C", "sigma", "us"}."""
    rp, ci, v = _i32(rowptr), _i32(colidx), _f64(vals)
    c, sg, us = C.c_int(), C.c_int(), C.c_double()
    _check(L.load().lusp_sell_tune(int(n), L.ptr(rp, C.c_int), L.ptr(ci, C.c_int), L.ptr(v, C.c_double),
                                   Sell.KINDS[kind], C.byref(c), C.byref(sg), C.byref(us)), "lusp_sell_tune")
    return {"C": c.value, "sigma": sg.value, "us": us.value}


def read_netlist(path, flt=None, pin: float = 0.0):
    """Matrix of a netlist file (s0: "n <n>" + "A i j v" lines; Matrix
    Market: a "%%MatrixMarket" banner) as 0-based CSC (n, Ap, Ai, Ax), with
    the floating-node list of an .flt file pinned onto the diagonal when
    pin > 0 (lusp_read_flt / lusp_coo_pin_rows)."""
    lib = L.load()
    path = str(path)
    with open(path, "rb") as fh:
        mtx = fh.read(14) == b"%%MatrixMarket"
    A = L.Coo()
    _check((lib.lusp_read_mtx_coo if mtx else lib.lusp_read_s0_coo)(path.encode(), C.byref(A)), "read " + path)
    try:
        if flt is not None and pin > 0:
            cnt = C.c_int(0)
            rc = lib.lusp_read_flt(str(flt).encode(), A.n, None, 0, C.byref(cnt))
            if rc not in (0, 2):          # LUSP_EALLOC: only counted
                _check(rc, "read " + str(flt))
            rows = np.empty(max(cnt.value, 1), np.int32)
            _check(lib.lusp_read_flt(str(flt).encode(), A.n, L.ptr(rows, C.c_int), rows.size, C.byref(cnt)),
                   "read " + str(flt))
            _check(lib.lusp_coo_pin_rows(C.byref(A), L.ptr(rows, C.c_int), cnt.value, pin), "pin")
        n = A.n
        Ap = np.empty(n + 1, np.int32)
        Ai = np.empty(max(A.nnz, 1), np.int32)
        Ax = np.empty(max(A.nnz, 1))
        _check(lib.lusp_coo_to_csc(C.byref(A), L.ptr(Ap, C.c_int), L.ptr(Ai, C.c_int), L.ptr(Ax, C.c_double)),
               "coo_to_csc")
        return n, Ap, Ai[:A.nnz], Ax[:A.nnz]
    finally:
        lib.lusp_coo_free(C.byref(A))
