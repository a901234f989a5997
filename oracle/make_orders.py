"""Write the COLAMD column order of bench.py's power-grid workload (n = 4050)
to oracle/power_grid_colamd_q.npy (TEST/BENCH INFRASTRUCTURE).

`bench.py --impl reference` times the reference's CPU path on the same column
order as the GPU arm; the reference ships no COLAMD, and that process must
not load this project's library, so it reads the order from this file.
tests/test_cpu_parity.py checks the file against the library's COLAMD.

  python oracle/make_orders.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
OUT = HERE / "power_grid_colamd_q.npy"


def main() -> None:
    sys.path.insert(0, str(ROOT))
    from luspice_b200 import api, mna
    m = mna.power_grid()
    q = api.colamd(m.n, m.Ap, m.Ai).astype(np.int32)
    np.save(OUT, q)
    print(f"wrote {OUT} (n={m.n})")


if __name__ == "__main__":
    main()
