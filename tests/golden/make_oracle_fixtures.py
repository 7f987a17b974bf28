"""Regenerates tests/golden/oracle_results.json: the CPU oracle's results on the benchmark
workloads, so that GPU tests and the bench can compare every result with the FP64 oracle without
re-running it (the largest case takes minutes of CPU time).

For each case and tolerance (1e-6 and 1e-8, all six tolerances equal) the file holds the oracle's
termination status, iteration count, primal and dual objectives and relative KKT errors, next to the
optimum known by construction.  Cases: the 512 instances of the uneven batch
(generators.batch_instance), the 750k x 1.5M and 1M x 2M constructed LPs.

    python tests/golden/make_oracle_fixtures.py [--skip-c1]

The oracle (oracle/liboracle_pdlp.so, `make -C oracle`) is test infrastructure; this script is the
only writer of the fixture.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from cuopt_b200 import generators as gen  # noqa: E402
from oracle import oracle as O  # noqa: E402

TOLS = (1e-6, 1e-8)
OUT = HERE / "oracle_results.json"


def record(lp, tol):
    res, _, _, _ = O.solve(lp, tol=tol)
    return {"status": res["status"], "iterations": res["iterations"],
            "primal_objective": res["primal_obj"], "dual_objective": res["dual_obj"],
            "relative_kkt": max(res["rel_primal"], res["rel_dual"], res["rel_gap"])}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--skip-c1", action="store_true", help="leave the 1M x 2M LP out")
    a = ap.parse_args()
    out = {"tolerances": list(TOLS), "batch": [], "single": {}}
    t0 = time.time()
    for i in range(512):
        lp = gen.batch_instance(i)
        out["batch"].append({"m": lp.m, "n": lp.n, "optimal_objective": lp.optimal_objective,
                             **{f"{t:g}": record(lp, t) for t in TOLS}})
    print(f"batch done in {time.time() - t0:.0f} s", flush=True)
    singles = [("c1_small", 750_000, 1_500_000, 1000)]
    if not a.skip_c1:
        singles.append(("c1", 1_000_000, 2_000_000, 1000))
    for name, m, n, seed in singles:
        lp = gen.constructed_lp(m, n, 8, seed=seed)
        out["single"][name] = {"m": m, "n": n, "seed": seed,
                               "optimal_objective": lp.optimal_objective,
                               **{f"{t:g}": record(lp, t) for t in TOLS}}
        print(f"{name} done in {time.time() - t0:.0f} s", flush=True)
    OUT.write_text(json.dumps(out, indent=1) + "\n")
    print("wrote", OUT)


if __name__ == "__main__":
    main()
