"""Runs the reference's own CPU dual simplex (oracle/_ref/ref_dual_simplex, built by
`make -C oracle ref` from the reference's unmodified sources) on an LP — TEST INFRASTRUCTURE ONLY.

Used by tests/ and bench.py's CPU baseline legs; never by the product library.  The binary exists
only where it was built (it is not committed) and travels with the working tree.
"""
from __future__ import annotations

import json
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

BINARY = Path(__file__).resolve().parent / "_ref" / "ref_dual_simplex"


def available() -> bool:
    return BINARY.exists()


def solve(lp, time_limit: float = 0.0, threads: int = 0, maximize: bool = False,
          timeout: float | None = None):
    """Solves `lp` (row_off, col_idx, val, c, con_lo, con_up, var_lo, var_up) with the reference's
    solve_linear_program.  Returns (result dict, x or None): status name, objective, solve_seconds
    (the solve call alone), primal_residual, threads."""
    m, n = len(lp.row_off) - 1, len(lp.c)
    nnz = int(lp.row_off[-1])
    with tempfile.TemporaryDirectory() as d:
        src, xout = os.path.join(d, "lp.bin"), os.path.join(d, "x.bin")
        with open(src, "wb") as f:
            f.write(np.array([m, n, nnz, int(maximize), threads], np.int32).tobytes())
            f.write(np.array([time_limit], np.float64).tobytes())
            f.write(np.ascontiguousarray(lp.row_off, np.int32).tobytes())
            f.write(np.ascontiguousarray(lp.col_idx[:nnz], np.int32).tobytes())
            for a in (lp.val[:nnz], lp.c, lp.con_lo, lp.con_up, lp.var_lo, lp.var_up):
                f.write(np.ascontiguousarray(a, np.float64).tobytes())
        r = subprocess.run([str(BINARY), src, xout], capture_output=True, text=True,
                           timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"ref_dual_simplex failed ({r.returncode}): {r.stderr.strip()}")
        res = json.loads(r.stdout.strip().splitlines()[-1])
        x = np.fromfile(xout, dtype=np.float64) if os.path.exists(xout) else None
    return res, x
