"""Build libluspice_b200.so (host analysis + sm_100a kernels + C-ABI) in-tree.

Usage: python -m luspice_b200.build [--force] [--jobs N]

Host C/C++ is compiled with -ffp-contract=off (pivot decisions must follow
the reference's exact operation sequence); CUDA sources are compiled for
sm_100a only.  Objects go to luspice_b200/_build/, the library to
luspice_b200/lib/.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
INCLUDE = ROOT / "include"
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIBDIR = PKG / "lib"
LIB = LIBDIR / "libluspice_b200.so"

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

C_SOURCES = ["host/selector.c", "host/level.c", "host/s0io.c", "host/ingest.c"]
CXX_SOURCES = ["host/symbolic.cpp", "host/colamd.cpp", "host/lu_static.cpp"]
CU_SOURCES = ["cuda/engine.cu", "cuda/capi.cu", "cuda/lu_gpu_par.cu", "cuda/spmv.cu", "cuda/noalloc.cu", "cuda/server.cu", "cuda/tune.cu"]
HEADERS = sorted(str(p) for p in list(CSRC.rglob("*.h")) + list(CSRC.rglob("*.cuh")) + list(INCLUDE.glob("*.h")))


def _cmd(src: str) -> tuple[list[str], Path]:
    path = CSRC / src
    obj = BUILD / (src.replace("/", "_") + ".o")
    inc = ["-I", str(INCLUDE), "-I", str(CSRC)]
    if src.endswith(".c"):
        cmd = ["gcc", "-O2", "-std=c11", "-fPIC", "-ffp-contract=off", "-Wall", *inc, "-c", str(path), "-o", str(obj)]
    elif src.endswith(".cpp"):
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", *inc, "-c", str(path), "-o", str(obj)]
    else:
        # LUSP_REFACTOR_PHASE_CYCLES=1 in the environment: the refactor's
        # per-phase cycle counters (diagnostics, ~3 % of its time; rebuild
        # with --force after changing it).
        opt = ["-DLUSP_REFACTOR_PHASE_CYCLES=1"] if os.environ.get("LUSP_REFACTOR_PHASE_CYCLES") == "1" else []
        cmd = [NVCC, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-ffp-contract=off", *opt, *inc, "-c", str(path), "-o", str(obj)]
    return cmd, obj


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    if src.stat().st_mtime > t:
        return True
    return any(Path(h).stat().st_mtime > t for h in HEADERS)


def build(force: bool = False, jobs: int = 8, verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    LIBDIR.mkdir(exist_ok=True)
    todo = []
    objs = []
    for src in C_SOURCES + CXX_SOURCES + CU_SOURCES:
        cmd, obj = _cmd(src)
        objs.append(obj)
        if force or _stale(obj, CSRC / src):
            todo.append((src, cmd))

    def run(item):
        src, cmd = item
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, cmd, r

    failed = []
    with cf.ThreadPoolExecutor(max_workers=max(1, jobs)) as ex:
        for src, cmd, r in ex.map(run, todo):
            if verbose or r.returncode != 0:
                sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            if r.returncode != 0:
                failed.append(src)
    if failed:
        raise RuntimeError(f"compilation failed: {failed}")
    if force or todo or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [NVCC, "-shared", *ARCH, "-o", str(tmp), *map(str, objs), "-Xlinker", "-soname=libluspice_b200.so"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
            raise RuntimeError("link failed")
        shutil.move(str(tmp), str(LIB))
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, jobs=a.jobs, verbose=a.verbose))


if __name__ == "__main__":
    main()
