"""Generate golden vectors from the reference's own code (oracle/_ref, compiled
from the reference sources by oracle/Makefile).

  python tests/golden/make_golden.py        (needs oracle/_ref/libluref.so)

Writes tests/golden/ref_cases.npz: for each case the input CSC, column order
and right-hand side, and the reference outputs of
  splu.h lu_factor (tol = 1)      pinv, Lp/Li/Lx, Up/Ui/Ux, status
  splu.h lu_solve_perm            x
  symbolic_dense.c                dense-scan pivots and L/U (GPU kernel semantics)
  level.c dsh_level_compute       column levels of U
and tests/golden/selector.npz: dsh_format_select outputs of the reference
selector for the five feature vectors of bench/test_selector.c plus seeded
random feature vectors.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from luspice_b200 import api, mna  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cases():
    out = []
    out.append(("analog40", mna.analog(40, 1)))
    out.append(("analog150", mna.analog(150, 2)))
    out.append(("analog500", mna.analog(500, 3)))
    out.append(("grid10x12", mna.power_grid(10, 12, 6, seed=4)))
    # Tiny hand-made cases: 1x1, diagonal, a branch row needing pivoting with
    # +-1 ties, and a structurally singular matrix.
    def csc(n, entries):
        e = sorted(entries, key=lambda t: (t[1], t[0]))
        Ap = np.zeros(n + 1, np.int32)
        for (_, c, _) in e:
            Ap[c + 1] += 1
        Ap = np.cumsum(Ap).astype(np.int32)
        Ai = np.array([r for r, _, _ in e], np.int32)
        Ax = np.array([v for _, _, v in e], np.float64)
        return Ap, Ai, Ax
    tiny = {
        "one": (1, [(0, 0, 2.5)]),
        "diag4": (4, [(i, i, float(i + 1)) for i in range(4)]),
        "ties": (3, [(0, 0, 1.0), (1, 0, -1.0), (2, 0, 1.0), (0, 1, 1.0), (1, 2, 1.0), (2, 1, 1.0), (2, 2, -1.0)]),
        "branch": (3, [(0, 0, 1e-3), (0, 2, 1.0), (2, 0, 1.0), (1, 1, 2e-3), (1, 2, -1.0), (2, 1, -1.0)]),
        "singular": (3, [(0, 0, 1.0), (1, 0, 2.0), (0, 1, 2.0), (1, 1, 4.0), (2, 2, 1.0)]),
    }
    for name, (n, ent) in tiny.items():
        Ap, Ai, Ax = csc(n, ent)
        m = mna.MNAMatrix(name=name, n=n, Ap=Ap, Ai=Ai, Ax=Ax, stamp=None, const=np.zeros(Ai.size),
                          elem_val=np.zeros(1), b=np.arange(1, n + 1, dtype=np.float64))
        out.append((name, m))
    return out


def ref_symbolic_dense(n, Ap, Ai, Ax, diagrow):
    lib = O.ref()
    ptrs = [C.c_void_p() for _ in range(10)]
    lnnz, unnz = C.c_long(), C.c_long()
    Ap, Ai, Ax, dr = (np.ascontiguousarray(a) for a in (Ap, Ai, Ax, diagrow))
    args = [n, Ap.ctypes.data_as(O.ip), Ai.ctypes.data_as(O.ip), Ax.ctypes.data_as(O.dp), dr.ctypes.data_as(O.ip),
            C.byref(ptrs[0]), C.byref(ptrs[1]), C.byref(ptrs[2]), C.byref(lnnz),
            C.byref(ptrs[3]), C.byref(ptrs[4]), C.byref(ptrs[5]), C.byref(unnz),
            C.byref(ptrs[6]), C.byref(ptrs[7])]
    lib.symbolic_dense.argtypes = [C.c_int, O.ip, O.ip, O.dp, O.ip] + [C.c_void_p] * 10
    st = lib.symbolic_dense(*args)
    if st >= 0:
        return {"status": st}
    ln, un = lnnz.value, unnz.value

    def arr(p, cnt, ct, dt):
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(ct)), shape=(cnt,)).astype(dt).copy()
    out = {"status": -1,
           "Lp": arr(ptrs[0], n + 1, C.c_int, np.int32), "Li": arr(ptrs[1], ln, C.c_int, np.int32),
           "Lx": arr(ptrs[2], ln, C.c_double, np.float64), "Up": arr(ptrs[3], n + 1, C.c_int, np.int32),
           "Ui": arr(ptrs[4], un, C.c_int, np.int32), "Ux": arr(ptrs[5], un, C.c_double, np.float64),
           "pinv": arr(ptrs[6], n, C.c_int, np.int32)}
    for p in ptrs[:8]:
        lib.free(p)
    return out


def main():
    assert O.ref_available(), "build oracle/_ref first (make -C oracle ref)"
    data = {}
    names = []
    for name, m in cases():
        names.append(name)
        q = api.colamd(m.n, m.Ap, m.Ai)
        F = O.lu_factor(m.n, m.Ap, m.Ai, m.Ax, q, use_ref=True)
        data[f"{name}/n"] = np.array([m.n])
        for k, v in (("Ap", m.Ap), ("Ai", m.Ai), ("Ax", m.Ax), ("q", q), ("b", m.b)):
            data[f"{name}/{k}"] = np.asarray(v)
        data[f"{name}/status"] = np.array([F["status"]])
        if F["status"] < 0:
            for k in ("pinv", "Lp", "Li", "Lx", "Up", "Ui", "Ux"):
                data[f"{name}/lu_{k}"] = F[k]
            data[f"{name}/x"] = O.ref_cpu_solve(m.n, m.Ap, m.Ai, m.Ax, q, m.b)
            lv = np.zeros(m.n, np.int32)
            nl = C.c_int()
            O.ref().dsh_level_compute(m.n, F["Up"].ctypes.data_as(O.ip), F["Ui"].ctypes.data_as(O.ip),
                                      lv.ctypes.data_as(O.ip), C.byref(nl))
            data[f"{name}/levels"] = lv
            data[f"{name}/nlevels"] = np.array([nl.value])
        # dense-scan semantics on the q-permuted CSC with original rows
        import scipy.sparse as sp
        A = sp.csc_matrix((m.Ax, m.Ai, m.Ap), shape=(m.n, m.n))[:, q]
        A.sort_indices()
        D = ref_symbolic_dense(m.n, A.indptr.astype(np.int32), A.indices.astype(np.int32), A.data, q.astype(np.int32))
        data[f"{name}/dense_status"] = np.array([D["status"]])
        if D["status"] < 0:
            for k in ("pinv", "Lp", "Li", "Lx", "Up", "Ui", "Ux"):
                data[f"{name}/dense_{k}"] = D[k]
    data["names"] = np.array(names)
    np.savez_compressed(HERE / "ref_cases.npz", **data)

    # Selector golden vectors.
    lib = C.CDLL(str(O.REF_SO))
    from luspice_b200._lib import DshConfig, DshMatrixInfo
    lib.dsh_format_select.argtypes = [C.POINTER(DshMatrixInfo), C.POINTER(DshConfig)]
    lib.dsh_mp_escalate.restype = C.c_int
    lib.dsh_mp_escalate.argtypes = [C.c_int]
    five = [(113, 616, 5.5, 16, 5, 2.9, 7.6e7, 7.6e7, 28.2, 0),
            (39899, 195429, 4.9, 60, 4, 12.2, 2.8e15, 2.8e15, 81.7, 0),
            (989, 5798, 5.9, 32, 5, 5.4, 1.5e13, 1.5e13, 46.5, 0),
            (42, 210, 5.0, 20, 4, 5.0, 1.5e13, 1.5e13, 27.0, 0),
            (94294, 432866, 4.6, 50, 4, 10.9, 0, 0, 82.5, 1)]
    rng = np.random.default_rng(42)
    rand = []
    for _ in range(200):
        rand.append((int(rng.integers(1, 100000)), int(rng.integers(1, 10 ** 6)), float(rng.uniform(1, 10)),
                     float(rng.integers(1, 100)), float(rng.integers(1, 10)), float(rng.choice([1.0, 4.9, 5.0, 5.1, 12.0])),
                     float(10 ** rng.uniform(-1, 16) * rng.choice([1, 1, 0, -1])), float(10 ** rng.uniform(-1, 16)),
                     float(rng.choice([0.0, 0.5, 1.0, 1.5, 20.0, 21.0, 80.0])), int(rng.random() < 0.1)))
    feats = np.array(five + rand, dtype=np.float64)
    outs = []
    for f in feats:
        mi = DshMatrixInfo(int(f[0]), int(f[1]), *f[2:9], int(f[9]))
        cfg = DshConfig()
        lib.dsh_format_select(C.byref(mi), C.byref(cfg))
        outs.append([cfg.spmv_format, cfg.sigma, cfg.use_ruiz, cfg.use_shift, cfg.shift, cfg.factor_prec,
                     cfg.ir_outer, cfg.ir_inner, cfg.ir_rtol, cfg.mp_path, cfg.pre_ruiz_hint, cfg.fp16_candidate])
    esc = np.array([lib.dsh_mp_escalate(i) for i in range(-1, 5)])
    np.savez_compressed(HERE / "selector.npz", features=feats, outputs=np.array(outs), escalate=esc)
    print("wrote", HERE / "ref_cases.npz", HERE / "selector.npz")


if __name__ == "__main__":
    main()
