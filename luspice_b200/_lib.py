"""ctypes bindings of libluspice_b200.so (every symbol the include/*.h headers
declare as extern "C").  Loading fails loudly when the library is missing:
there is no Python or CPU fallback for any operation."""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libluspice_b200.so"

c_int_p = C.POINTER(C.c_int)
c_long_p = C.POINTER(C.c_long)
c_double_p = C.POINTER(C.c_double)
c_void_pp = C.POINTER(C.c_void_p)


class PatternInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz_a", C.c_int), ("lnnz", C.c_long), ("unnz", C.c_long),
                ("cap", C.c_long), ("ncol_levels", C.c_int), ("nfwd_levels", C.c_int),
                ("nbwd_levels", C.c_int), ("max_col", C.c_int), ("nslices", C.c_int),
                ("sell_total", C.c_int), ("flops", C.c_long), ("gathered", C.c_long),
                ("hash", C.c_ulonglong), ("device_bytes", C.c_size_t), ("singular_col", C.c_int),
                ("dense_tail", C.c_int), ("tail_start", C.c_int)]


class SysStats(C.Structure):
    _fields_ = [("min_abs_pivot", C.c_double), ("min_pivot_ratio", C.c_double),
                ("max_abs_u", C.c_double), ("res", C.c_double * 16), ("nres", C.c_int),
                ("inner_iters", C.c_int), ("outer_iters", C.c_int), ("status", C.c_int),
                ("singular_col", C.c_int), ("rung", C.c_int), ("cyc_wait", C.c_longlong),
                ("cyc_gather", C.c_longlong), ("cyc_update", C.c_longlong), ("cyc_refactor", C.c_longlong),
                ("cyc_lsolve", C.c_longlong), ("cyc_tail", C.c_longlong), ("cyc_usolve", C.c_longlong),
                ("cyc_spmv", C.c_longlong), ("cyc_solve", C.c_longlong), ("cyc_tpanel", C.c_longlong),
                ("cyc_ttrsm", C.c_longlong), ("cyc_tupdate", C.c_longlong), ("cyc_tdiag", C.c_longlong),
                ("cyc_tgemv", C.c_longlong)]


class BatchOpts(C.Structure):
    _fields_ = [("prec", C.c_int), ("krylov", C.c_int), ("max_outer", C.c_int),
                ("rtol", C.c_double), ("inner_rel", C.c_double), ("stag_ratio", C.c_double),
                ("pivot_tol", C.c_double), ("block_threads", C.c_int), ("ctas_per_sm", C.c_int),
                ("solve_sweep", C.c_int), ("refactor_mode", C.c_int), ("inner_prec", C.c_int),
                ("xtol", C.c_double), ("refactor_threads", C.c_int),
                ("refactor_cluster", C.c_int), ("ladder", C.c_int), ("ladder_slots", C.c_int),
                ("factor_shift", C.c_double), ("hard_shift", C.c_double), ("refactor_spread", C.c_int)]


class ServerOpts(C.Structure):
    _fields_ = [("solver", BatchOpts), ("max_batch", C.c_int), ("streams", C.c_int),
                ("hbm_budget_gb", C.c_double), ("arena_gb", C.c_double), ("staging_mb", C.c_double),
                ("escalate", C.c_int), ("analysis_threads", C.c_int)]


class ServeResult(C.Structure):
    _fields_ = [("rc", C.c_int), ("status", C.c_int), ("latency_ms", C.c_double), ("queue_ms", C.c_double),
                ("device_ms", C.c_double), ("residual", C.c_double), ("inner_iters", C.c_int),
                ("outer_iters", C.c_int), ("batch_size", C.c_int), ("cache_hit", C.c_int),
                ("escalated", C.c_int), ("pad_", C.c_int), ("pattern_hash", C.c_ulonglong)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("escalated", C.c_longlong),
                ("cache_hits", C.c_longlong), ("cache_misses", C.c_longlong), ("evictions", C.c_longlong),
                ("launches", C.c_longlong), ("patterns_resident", C.c_longlong),
                ("max_batch_seen", C.c_longlong), ("pattern_gb", C.c_double), ("refused", C.c_longlong),
                ("promoted", C.c_longlong), ("fp64_starts", C.c_longlong)]


class Coo(C.Structure):
    """lusp_coo (luspice_b200.h): 1-based COO triplets."""
    _fields_ = [("n", C.c_int), ("nnz", C.c_longlong), ("cap", C.c_longlong),
                ("row", C.POINTER(C.c_int)), ("col", C.POINTER(C.c_int)), ("val", C.POINTER(C.c_double))]


class DshLuStatic(C.Structure):
    """dsh_lu_static (lu_static.h), field for field."""
    _fields_ = [("n", C.c_int), ("cnnz", C.c_long), ("lnnz", C.c_long), ("unnz", C.c_long),
                ("cap", C.c_long), ("Ap", c_int_p), ("Ai", c_int_p), ("Ax", C.c_void_p),
                ("P", c_int_p), ("Q", c_int_p), ("min_diag_U", C.c_double),
                ("pivot_growth", C.c_double), ("dev_allocated", C.c_int),
                ("factor_cache", C.c_void_p), ("pin", C.c_double)]


class CSRMatrix(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_longlong), ("rowptr", c_int_p),
                ("colidx", c_int_p), ("values", c_double_p)]


class DshMatrixInfo(C.Structure):
    _fields_ = [("n", C.c_int), ("nnz", C.c_long), ("avg_rowlen", C.c_double),
                ("max_rowlen", C.c_double), ("p50_rowlen", C.c_double), ("row_skew", C.c_double),
                ("kappa_ruiz", C.c_double), ("kappa_est", C.c_double),
                ("dyn_range_log10", C.c_double), ("singular_flag", C.c_int)]


class DshConfig(C.Structure):
    _fields_ = [("spmv_format", C.c_int), ("sigma", C.c_int), ("use_ruiz", C.c_int),
                ("use_shift", C.c_int), ("shift", C.c_double), ("factor_prec", C.c_int),
                ("ir_outer", C.c_int), ("ir_inner", C.c_int), ("ir_rtol", C.c_double),
                ("mp_path", C.c_int), ("pre_ruiz_hint", C.c_int), ("fp16_candidate", C.c_int)]


# name -> (restype, argtypes)
SIGNATURES = {
    # luspice_b200.h
    "lusp_last_error": (C.c_char_p, []),
    "lusp_version": (C.c_char_p, []),
    "lusp_device_count": (C.c_int, []),
    "lusp_pattern_create": (C.c_int, [C.c_int, c_int_p, c_int_p, c_double_p, c_int_p, c_void_pp]),
    "lusp_pattern_create_ex": (C.c_int, [C.c_int, c_int_p, c_int_p, c_double_p, c_int_p, C.c_int, c_void_pp]),
    "lusp_tune": (C.c_int, [C.c_int, c_int_p, c_int_p, c_double_p, c_double_p, C.c_int, C.c_void_p,
                            C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "lusp_sell_tune": (C.c_int, [C.c_int, c_int_p, c_int_p, c_double_p, C.c_int, C.POINTER(C.c_int),
                                 C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "lusp_pattern_destroy": (None, [C.c_void_p]),
    "lusp_pattern_get_info": (C.c_int, [C.c_void_p, C.POINTER(PatternInfo)]),
    "lusp_pattern_get_perm": (C.c_int, [C.c_void_p, c_int_p, c_int_p]),
    "lusp_pattern_get_structure": (C.c_int, [C.c_void_p, c_int_p, c_int_p, c_int_p]),
    "lusp_pattern_get_levels": (C.c_int, [C.c_void_p, c_int_p]),
    "lusp_colamd": (C.c_int, [C.c_int, C.c_int, c_int_p, c_int_p, C.c_double, C.c_double, c_int_p]),
    "lusp_pivot_factor": (C.c_int, [C.c_int, c_int_p, c_int_p, c_double_p, c_int_p, C.c_double,
                                    c_int_p, c_int_p, c_int_p, c_double_p, C.c_long,
                                    c_int_p, c_int_p, c_double_p, C.c_long,
                                    c_long_p, c_long_p, c_int_p]),
    "lusp_batch_opts_default": (None, [C.POINTER(BatchOpts)]),
    "lusp_batch_create": (C.c_int, [C.c_int, c_void_pp, C.POINTER(BatchOpts), c_void_pp]),
    "lusp_batch_destroy": (None, [C.c_void_p]),
    "lusp_batch_device_ptrs": (C.c_int, [C.c_void_p, C.c_int, c_void_pp, c_void_pp, c_void_pp]),
    "lusp_batch_upload": (C.c_int, [C.c_void_p, c_double_p, c_double_p, C.c_void_p]),
    "lusp_batch_download": (C.c_int, [C.c_void_p, c_double_p, C.c_void_p]),
    "lusp_batch_run": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "lusp_batch_run_graph": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "lusp_batch_stats": (C.c_int, [C.c_void_p, C.POINTER(SysStats), C.c_void_p]),
    "lusp_batch_factor_values": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]),
    "lusp_batch_copy_values": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "lusp_batch_factor_device_ptr": (C.c_int, [C.c_void_p, C.c_int, c_void_pp]),
    "lusp_batch_set_params": (C.c_int, [C.c_void_p, C.POINTER(BatchOpts)]),
    "lusp_batch_launch_count": (C.c_int, [C.c_void_p]),
    "lusp_batch_time_kernels": (C.c_int, [C.c_void_p, C.c_int]),
    "lusp_batch_kernel_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "lusp_batch_launch_shape": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "lusp_sell_create": (C.c_int, [C.c_int, c_int_p, c_int_p, c_double_p, C.c_int, C.c_int,
                                   C.c_int, c_void_pp]),
    "lusp_sell_destroy": (None, [C.c_void_p]),
    "lusp_csr_spmv32": (C.c_int, [C.c_int] + [C.c_void_p] * 6),
    "lusp_server_opts_default": (None, [C.POINTER(ServerOpts)]),
    "lusp_server_create": (C.c_int, [C.POINTER(ServerOpts), c_void_pp]),
    "lusp_server_destroy": (None, [C.c_void_p]),
    "lusp_serve_submit": (C.c_longlong, [C.c_void_p, C.c_int, c_int_p, c_int_p, c_double_p, c_double_p]),
    "lusp_serve_poll": (C.c_int, [C.c_void_p, C.c_longlong, c_double_p, C.POINTER(ServeResult), C.c_int]),
    "lusp_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "lusp_sell_spmv": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "lusp_sell_info": (C.c_int, [C.c_void_p, c_long_p, c_long_p, c_double_p, c_double_p]),
    # lu_gpu_par.h (C-ABI launchers)
    "lusp_lu_factor_par_launch": (C.c_int, [C.c_int] + [C.c_void_p] * 7 + [C.c_long]
                                  + [C.c_void_p] * 3 + [C.c_long] + [C.c_void_p] * 7),
    "lusp_trisolve_par_launch": (C.c_int, [C.c_int] + [C.c_void_p] * 13),
    "lusp_trisolve_par_noalloc": (C.c_int, [C.c_int] + [C.c_void_p] * 11),
    # lu_static.h
    "dsh_symbolic": (C.c_int, [C.c_int, C.c_long, c_int_p, c_int_p, c_int_p, C.POINTER(DshLuStatic)]),
    "dsh_numeric": (C.c_int, [C.POINTER(DshLuStatic), c_int_p, c_int_p, c_double_p, C.c_int]),
    "dsh_trisolve": (C.c_int, [C.POINTER(DshLuStatic), c_double_p, c_double_p]),
    "dsh_gmres_ir": (C.c_int, [C.POINTER(DshLuStatic), c_double_p, c_double_p, C.c_int, C.c_int,
                               C.c_double, c_double_p, c_int_p]),
    "dsh_lu_static_init": (C.c_int, [C.POINTER(DshLuStatic)]),
    "dsh_lu_static_alloc": (C.c_int, [C.POINTER(DshLuStatic)]),
    "dsh_lu_static_free": (None, [C.POINTER(DshLuStatic)]),
    "dsh_lu_status_str": (C.c_char_p, [C.c_int]),
    "dsh_symbolic_count": (C.c_long, []),
    # level.h
    "dsh_level_compute": (C.c_int, [C.c_int, c_int_p, c_int_p, c_int_p, c_int_p]),
    "dsh_level_hist": (C.c_int, [C.c_int, c_int_p, C.c_int, c_int_p]),
    # netlist ingest (luspice_b200.h)
    "lusp_read_s0_coo": (C.c_int, [C.c_char_p, C.POINTER(Coo)]),
    "lusp_read_mtx_coo": (C.c_int, [C.c_char_p, C.POINTER(Coo)]),
    "lusp_read_flt": (C.c_int, [C.c_char_p, C.c_int, c_int_p, C.c_int, c_int_p]),
    "lusp_coo_pin_rows": (C.c_int, [C.POINTER(Coo), c_int_p, C.c_int, C.c_double]),
    "lusp_coo_to_csc": (C.c_int, [C.POINTER(Coo), c_int_p, c_int_p, c_double_p]),
    "lusp_coo_free": (None, [C.POINTER(Coo)]),
    # spmv.h
    "read_s0_to_csr": (C.c_int, [C.c_char_p, C.POINTER(CSRMatrix)]),
    "csr_free": (None, [C.POINTER(CSRMatrix)]),
    "read_rhs": (C.c_int, [C.c_char_p, C.c_int, c_double_p]),
    "spmv_host": (C.c_int, [C.POINTER(CSRMatrix), c_double_p, c_double_p, c_double_p]),
    "csr_alloc_device": (C.c_int, [C.POINTER(CSRMatrix), C.POINTER(c_int_p), C.POINTER(c_int_p),
                                   C.POINTER(c_double_p)]),
    "spmv_launch": (None, [C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                           C.c_void_p]),
    # selector.h
    "dsh_matrix_analyze": (None, [C.c_int, C.c_long, c_int_p, C.POINTER(DshMatrixInfo)]),
    "dsh_format_select": (None, [C.POINTER(DshMatrixInfo), C.POINTER(DshConfig)]),
    "dsh_fmt_name": (C.c_char_p, [C.c_int]),
    "dsh_mp_initial": (None, [C.POINTER(DshMatrixInfo), C.POINTER(DshConfig)]),
    "dsh_mp_escalate": (C.c_int, [C.c_int]),
    "dsh_mp_name": (C.c_char_p, [C.c_int]),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load the library once and attach signatures.  Raises when it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m luspice_b200.build` "
                           "(the package has no fallback implementation)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a, ctype):
    """ctypes pointer to a contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(ctype))
