"""Register budget of the level sweeps (CPU: compiles only).

The level-synchronous sweeps (`staged_sweep`) are calls inside the solve
kernel, and their registers come out of the same 128 per thread as the GMRES
code around them.  Code inlined into that kernel which raises its register
peak makes ptxas spill inside every sweep instance, and on the B200 the solve
then runs 35-40 % slower although none of that code runs in the sweeps.  This
test compiles engine.cu with the library's own flags and `-Xptxas -v` and
requires every `staged_sweep` instance used with the solve vector in shared
memory to spill nothing.
"""
import re
import shutil
import subprocess

import pytest

from luspice_b200 import build as b


def _ptxas_report(tmp_path):
    cmd, _ = b._cmd("cuda/engine.cu")
    if shutil.which(cmd[0]) is None and not shutil.os.path.exists(cmd[0]):
        pytest.skip("nvcc not found")
    out = tmp_path / "engine.o"
    cmd = cmd[:-1] + [str(out)] + ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return r.stderr


def test_level_sweeps_do_not_spill(tmp_path):
    text = _ptxas_report(tmp_path)
    # "Function properties for <mangled name>" followed by the spill line.
    lines = text.splitlines()
    found = 0
    for i, line in enumerate(lines):
        if "Function properties for" not in line or "staged_sweep" not in line:
            continue
        name = subprocess.run(["c++filt"], input=line.split("for", 1)[1].strip(), capture_output=True,
                              text=True).stdout.strip()
        # Instances with the solve vector in shared memory: third template
        # argument (GY) false.
        m = re.search(r"staged_sweep<(float|double), (true|false), (true|false)>", name)
        if not m or m.group(3) != "false":
            continue
        spill = re.search(r"(\d+) bytes spill stores, (\d+) bytes spill loads", lines[i + 1])
        assert spill, lines[i + 1]
        assert spill.group(1) == "0" and spill.group(2) == "0", f"{name}: {lines[i + 1].strip()}"
        found += 1
    # Four solve-kernel instantiations x two sweeps, each reported once per
    # kernel that calls it.
    assert found >= 4, f"only {found} staged_sweep reports in the ptxas output"
