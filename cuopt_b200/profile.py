"""Profiling driver for the PDLP kernels (used under ncu; also a quick standalone timing tool).

    python -m cuopt_b200.profile --config c1 --mode solve  --precision mixed
    python -m cuopt_b200.profile --config c1_small --mode sweeps --precision mixed --iterations 3

`solve`  runs one full solve to 1e-6 relative KKT from device-resident inputs (cuOptSolveDevice);
`sweeps` prepares the LP and launches the two fused PDHG sweeps separately between CUDA events
         (cuOptProfilePDHGSweeps).
`batch`  (config c3) solves the 512-instance batch in one cuOptBatchSolve call and a sample of the
         same instances one by one with cuOptSolve (1e-6; FP64, or mixed precision with
         --batch-precision mixed, for both).
`adjoint` (config c4) solves 64 non-degenerate 5000 x 10000 LPs in one batched call (crossover
         on), back-propagates L = sum w * x* through the matrix-free KKT adjoint, and checks the
         gradients of every instance against its vertex's exact derivatives and against central
         differences (h = 1e-6) of the vertex map on random coordinates of c, b and the A values,
         and a few instances' against central differences through the full solver.
`climbers` solves `count` copies of one LP (the config's) that differ in one variable's upper
         bound each with one cuOptSolveClimbers call (FP64), and a sample of the same copies one
         by one with cuOptSolve.  With --strong-branching: cuOptBatchPDLPStrongBranching on
         count / 2 fractional variables (a solve of the LP, then `count` warm-started branches),
         against the same branches solved one by one from the LP's solution.
`gather`  measures the random-gather ceiling (cuOptProfileGatherRate) for the config's two gathered
         vectors (y in the primal sweep, x_bar in the dual sweep) in FP32 and FP64.
Prints one JSON line with the timings.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

CONFIGS = {
    # name: (m, n, non-zeros per column (0: skewed generator), seed)
    "c0": (2_000, 5_000, 8, 0),
    "c1": (1_000_000, 2_000_000, 8, 1000),
    "c1_small": (750_000, 1_500_000, 8, 1000),
    "c2": (500_000, 1_500_000, 0, 2000),  # + one slack column per '<=' row (n = 1.75M)
    "c2_small": (50_000, 150_000, 0, 2000),
    "c4": (5_000, 10_000, 8, 4000),
}


def main() -> None:
    import numpy as np
    import torch

    from cuopt_b200 import generators as gen
    from cuopt_b200._lib import PDLPStatistics, lib, stats_dict

    ap = argparse.ArgumentParser()
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c1_small")
    ap.add_argument("--mode", choices=["solve", "sweeps", "batch", "adjoint", "climbers", "gather",
                                       "barrier"],
                    default="sweeps")
    ap.add_argument("--fd-solver", type=int, default=2,
                    help="adjoint mode: instances also differenced through the full solver")
    ap.add_argument("--fd-coords", type=int, default=32,
                    help="adjoint mode: coordinates per kind (c, b, A) and instance")
    ap.add_argument("--count", type=int, default=512, help="batch mode: instances")
    ap.add_argument("--sequential", type=int, default=64,
                    help="batch mode: instances also solved one by one (timing sample)")
    ap.add_argument("--repeats", type=int, default=2,
                    help="batch mode: batched solves, the first one untimed (warm-up)")
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="mixed")
    ap.add_argument("--batch-precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--iterations", type=int, default=3)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--time-limit", type=float, default=0.0)
    ap.add_argument("--iteration-limit", type=int, default=0,
                    help="solve and climbers modes: > 0 caps iterations")
    ap.add_argument("--strong-branching", action="store_true",
                    help="climbers mode: time cuOptBatchPDLPStrongBranching instead")
    ap.add_argument("--refine", type=int, default=0, help="> 0: continue a mixed-precision solve in FP64 to 1e-8")
    ap.add_argument("--tiled", type=int, default=-1, choices=[-1, 0, 1],
                    help="pdlp_tiled_sweeps: -1 autotuned, 0 sliced ELL only, 1 tiled where possible")
    ap.add_argument("--persistent", type=int, default=-1, choices=[-1, 0, 1, 2],
                    help="pdlp_persistent_iterations: -1 timed choice, 0 CUDA graphs, 1 persistent "
                         "kernel, 2 cluster-resident kernel")
    ap.add_argument("--solves", type=int, default=1,
                    help="solve mode: solves of the same LP (the statistics are the last one's)")
    a = ap.parse_args()

    if a.mode == "batch":
        print(json.dumps(run_batch(a)))
        return
    if a.mode == "adjoint":
        print(json.dumps(run_adjoint(a)))
        return
    if a.mode == "climbers":
        print(json.dumps(run_climbers(a)))
        return
    if a.mode == "gather":
        print(json.dumps(run_gather(a)))
        return
    if a.mode == "barrier":
        print(json.dumps(run_barrier()))
        return
    m, n, k, seed = CONFIGS[a.config]
    lp = (gen.constructed_lp(m, n, k, seed=seed) if k
          else gen.skewed_lp(m, n, seed=seed, explicit_slacks=True))
    m, n = lp.m, lp.n  # the skewed LP adds slack columns
    dev = torch.device("cuda", 0)
    t = lambda x, dt: torch.as_tensor(np.ascontiguousarray(x), device=dev, dtype=dt)
    arrs = [t(lp.c, torch.float64), t(lp.row_off, torch.int32), t(lp.col_idx, torch.int32),
            t(lp.val, torch.float64), t(lp.con_lo, torch.float64), t(lp.con_up, torch.float64),
            t(lp.var_lo, torch.float64), t(lp.var_up, torch.float64)]
    ptr = [C.c_void_p(x.data_ptr()) for x in arrs]
    L = lib()
    s = C.c_void_p()
    L.cuOptCreateSolverSettings(C.byref(s))
    for name in ("absolute_primal_tolerance", "relative_primal_tolerance", "absolute_dual_tolerance",
                 "relative_dual_tolerance", "absolute_gap_tolerance", "relative_gap_tolerance"):
        L.cuOptSetFloatParameter(s, name.encode(), a.tol)
    L.cuOptSetIntegerParameter(s, b"pdlp_precision", 1 if a.precision == "mixed" else 0)
    L.cuOptSetIntegerParameter(s, b"pdlp_tiled_sweeps", a.tiled)
    L.cuOptSetIntegerParameter(s, b"pdlp_persistent_iterations", a.persistent)
    L.cuOptSetParameter(s, b"log_to_console", b"false")
    if a.time_limit > 0:
        L.cuOptSetFloatParameter(s, b"time_limit", a.time_limit)
    if a.iteration_limit > 0:
        L.cuOptSetIntegerParameter(s, b"iteration_limit", a.iteration_limit)
    if a.refine:
        L.cuOptSetIntegerParameter(s, b"pdlp_refinement_passes", a.refine)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    out = {"config": a.config, "m": m, "n": n, "nnz": lp.nnz, "precision": a.precision, "mode": a.mode}
    if a.mode == "solve":
        x = torch.empty(n, device=dev, dtype=torch.float64)
        y = torch.empty(m, device=dev, dtype=torch.float64)
        rc = torch.empty(n, device=dev, dtype=torch.float64)
        st, status = PDLPStatistics(), C.c_int32()
        walls = []
        for _ in range(max(1, a.solves)):
            t0 = time.perf_counter()
            code = L.cuOptSolveDevice(m, n, 1, 0.0, *ptr, s, stream, C.c_void_p(x.data_ptr()),
                                      C.c_void_p(y.data_ptr()), C.c_void_p(rc.data_ptr()),
                                      C.byref(st), C.byref(status))
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - t0)
            if code != 0:
                break
        out.update({"rc": code, "status": status.value, "wall_s": walls[-1], "walls_s": walls})
        out.update(stats_dict(st))
        out["objective_rel_error"] = abs(st.primal_objective - lp.optimal_objective) / max(
            1.0, abs(lp.optimal_objective))
        if code != 0:
            print(json.dumps(out))
            sys.exit(1)
    else:
        vals = [C.c_double() for _ in range(4)]
        code = L.cuOptProfilePDHGSweeps(m, n, *ptr, s, stream, a.iterations, *[C.byref(v) for v in vals])
        out.update({"rc": code, "ms_primal": vals[0].value, "ms_dual": vals[1].value,
                    "bytes_primal": vals[2].value, "bytes_dual": vals[3].value})
        if code == 0:
            out["gbs_primal"] = vals[2].value / vals[0].value / 1e6
            out["gbs_dual"] = vals[3].value / vals[1].value / 1e6
            out["classes"] = sweep_classes(L, m, n, ptr, s, stream, a.iterations,
                                           4 if a.precision == "mixed" else 8)
        else:
            print(json.dumps(out))
            sys.exit(1)
    L.cuOptDestroySolverSettings(C.byref(s))
    print(json.dumps(out))


def sweep_classes(L, m, n, ptr, settings, stream, iterations, elem) -> dict:
    """The plain sweeps split by row-length class (cuOptProfileSweepClasses): per sweep and class,
    rows, non-zeros, padding, ms per launch, gathers/s and algorithmic GB/s (values + indices of
    the non-zeros, the row's offset and its epilogue vectors: primal 7, dual 5 elements)."""
    out_v = (C.c_double * 14)()
    code = L.cuOptProfileSweepClasses(m, n, *ptr, settings, stream, iterations, out_v)
    if code != 0:
        raise RuntimeError(f"cuOptProfileSweepClasses returned {code}")
    res = {}
    for s, (name, epi) in enumerate((("primal", 7), ("dual", 5))):
        v = list(out_v[7 * s:7 * s + 7])
        long_rows, long_nnz, long_ms, sl_rows, sl_nnz, sl_stored, sl_ms = v

        def cls(rows, nnz, ms, stored, offset_bytes):
            if rows == 0 or ms == 0:
                return {"rows": int(rows), "nnz": int(nnz)}
            byts = nnz * (elem + 4) + rows * (epi * elem + offset_bytes)
            return {"rows": int(rows), "nnz": int(nnz), "stored": int(stored),
                    "ms": ms, "gathers_per_s": nnz / (ms * 1e-3),
                    "algorithmic_gbs": byts / (ms * 1e-3) / 1e9}
        res[name] = {"long_rows": cls(long_rows, long_nnz, long_ms, long_nnz, 8),
                     "sliced_rows": cls(sl_rows, sl_nnz, sl_ms, sl_stored, 8 / 32)}
    return res


def gather_rates(m: int, n: int, nnz: int, stream) -> dict:
    """Best random-gather rates (gathers/s) for vectors of m and n elements, 4 and 8 bytes."""
    from cuopt_b200._lib import lib

    L = lib()
    out = {}
    for name, length in (("primal_gather_y", m), ("dual_gather_xbar", n)):
        for eb in (4, 8):
            rate, chunks = C.c_double(), C.c_int32()
            code = L.cuOptProfileGatherRate(length, 4 * nnz, eb, stream, C.byref(rate),
                                            C.byref(chunks))
            if code != 0:
                raise RuntimeError(f"cuOptProfileGatherRate returned {code}")
            out[f"{name}_fp{8 * eb}"] = {"gathers_per_s": rate.value, "chunks_in_flight": chunks.value}
    return out


def run_barrier() -> dict:
    """Cost of the persistent kernel's grid barrier (cuOptProbeGridBarrier): microseconds per
    barrier for grids of 8 to 1184 blocks, 5000 barriers each."""
    from cuopt_b200._lib import lib

    L = lib()
    out = {}
    for blocks, threads in ((8, 256), (16, 256), (8, 1024), (16, 1024), (2, 256)):
        ms = C.c_double()
        code = L.cuOptProbeClusterBarrier(blocks, threads, 5000, None, C.byref(ms))
        out[f"cluster_{blocks}x{threads}"] = ({"us_per_barrier": 1e3 * ms.value / 5000}
                                              if code == 0 else {"rc": code})
    for blocks in (8, 21, 57, 148, 296, 592, 740, 1184):
        st, ms = C.c_int32(), C.c_double()
        code = L.cuOptProbeGridBarrier(blocks, 5000, 0, 5000.0, None, C.byref(st), C.byref(ms))
        out[str(blocks)] = ({"us_per_barrier": 1e3 * ms.value / 5000, "status": st.value}
                            if code == 0 else {"rc": code})
    return out


def run_gather(a) -> dict:
    import torch

    m, n, k, _ = CONFIGS[a.config]
    nnz = n * k if k else 75_000_000
    stream = C.c_void_p(torch.cuda.current_stream(torch.device("cuda", 0)).cuda_stream)
    res = gather_rates(m, n, nnz, stream)
    from cuopt_b200._lib import lib
    L = lib()
    for name, length in (("primal_scatter_y", m), ("dual_scatter_ax", m)):
        for eb in (4, 8):
            rate, chunks = C.c_double(), C.c_int32()
            if L.cuOptProfileScatterRate(length, 4 * nnz, eb, stream, C.byref(rate),
                                         C.byref(chunks)) != 0:
                raise RuntimeError("cuOptProfileScatterRate failed")
            res[f"{name}_fp{8 * eb}"] = {"scatters_per_s": rate.value,
                                          "chunks_in_flight": chunks.value}
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    for v in res.values():
        rate = v.get("gathers_per_s", v.get("scatters_per_s"))
        v["per_sm_per_cycle_at_1965mhz"] = rate / sms / 1.965e9
    return {"config": a.config, "m": m, "n": n, "gathers": 4 * nnz, "sms": sms, "rates": res}


def batch_models(count: int = 512):
    """The 512-LP batch workload (generators.batch_lps) and its DataModels."""
    from cuopt_b200 import generators as gen
    from cuopt_b200 import linear_programming as lpm

    lps = gen.batch_lps(count, seed=3000)
    dms = []
    for lp in lps:
        dm = lpm.DataModel()
        dm.set_csr_constraint_matrix(lp.val, lp.col_idx, lp.row_off)
        dm.set_objective_coefficients(lp.c)
        dm.set_constraint_lower_bounds(lp.con_lo)
        dm.set_constraint_upper_bounds(lp.con_up)
        dm.set_variable_lower_bounds(lp.var_lo)
        dm.set_variable_upper_bounds(lp.var_up)
        dms.append(dm)
    return lps, dms


def run_batch(a, models=None) -> dict:
    """The 512-LP batch: one batched solve of `count` uneven LPs vs the same LPs one at a time.
    `models` (lps, dms) reuses generated instances; with a.per_instance the result also holds every
    instance's status, iteration count and primal objective."""
    import numpy as np

    from cuopt_b200 import linear_programming as lpm

    lps, dms = models if models is not None else batch_models(a.count)
    st = lpm.SolverSettings()
    st.set_optimality_tolerance(a.tol)
    st.set_parameter(lpm.CUOPT_METHOD, int(lpm.SolverMethod.PDLP))
    st.set_parameter(lpm.CUOPT_LOG_TO_CONSOLE, False)
    precision = getattr(a, "batch_precision", "fp64")
    st.set_parameter(lpm.CUOPT_PDLP_PRECISION, 1 if precision == "mixed" else 0)
    st.set_parameter(lpm.CUOPT_PDLP_PERSISTENT_ITERATIONS, getattr(a, "persistent", -1))
    if getattr(a, "refine", 0):
        st.set_parameter(lpm.CUOPT_PDLP_REFINEMENT_PASSES, a.refine)
    if a.time_limit > 0:
        st.set_parameter(lpm.CUOPT_TIME_LIMIT, a.time_limit)
    times = []
    for _ in range(max(1, a.repeats)):
        sols, t = lpm.BatchSolve(dms, st)
        times.append(t)
    batch_s = min(times[1:]) if len(times) > 1 else times[0]
    status = [int(s.get_termination_status()) for s in sols]
    iters = [s.get_lp_stats()["nb_iterations"] for s in sols]
    obj_err = [abs(s.get_primal_objective() - lp.optimal_objective) / max(1.0, abs(lp.optimal_objective))
               for s, lp in zip(sols, lps)]
    kkt = [max(s.stats.get("l2_relative_primal_residual", 0.0),
               s.stats.get("l2_relative_dual_residual", 0.0), s.stats.get("relative_gap", 0.0))
           for s in sols]
    worst = sorted(range(len(sols)), key=lambda i: -obj_err[i])[:8]
    out = {"config": "c3", "precision": precision, "count": a.count, "tolerance": a.tol,
           "refined_to": 1e-8 if (getattr(a, "refine", 0) and precision == "mixed") else None,
           "m_total": int(sum(lp.m for lp in lps)),
           "n_total": int(sum(lp.n for lp in lps)), "nnz_total": int(sum(lp.nnz for lp in lps)),
           "batch_s": batch_s, "batch_times_s": times, "batch_lps_per_s": a.count / batch_s,
           "optimal": status.count(1), "max_iterations": max(iters),
           "mean_iterations": float(np.mean(iters)), "max_objective_rel_error": max(obj_err),
           "batch_setup_s": sols[0].stats.get("setup_time"),
           "iterations_p50_p90_p99": [float(np.percentile(iters, q)) for q in (50, 90, 99)],
           "max_power_iterations": max(s.stats.get("power_iterations", 0) for s in sols),
           "fp64_resolved": sum(int(s.stats.get("refinement_passes", 0) > 0) for s in sols),
           "max_relative_kkt": max(kkt),
           "objective_rel_error_over_1e-6": sum(int(e > 1e-6) for e in obj_err),
           "plain_iterations": {
               "form": {0: "graphs", 1: "persistent"}.get(
                   sols[0].stats.get("plain_iteration_form"), "undecided"),
               "persistent_blocks": sols[0].stats.get("persistent_blocks"),
               "us_per_iteration_graphs": sols[0].stats.get("plain_iteration_us_graphs"),
               "us_per_iteration_persistent": sols[0].stats.get("plain_iteration_us_persistent"),
               "sweep_warps_per_block": [sols[0].stats.get("sweep_warps_per_block_primal"),
                                         sols[0].stats.get("sweep_warps_per_block_dual")],
               "sweep_block_shape_ms": sols[0].stats.get("sweep_block_shape_ms")},
           "worst_instances": [{"i": i, "m": lps[i].m, "status": status[i], "iterations": iters[i],
                                "objective_rel_error": obj_err[i], "relative_kkt": kkt[i],
                                "optimal_objective": lps[i].optimal_objective,
                                "fp64_continued": int(sols[i].stats.get("refinement_passes", 0) > 0)}
                               for i in worst]}
    if getattr(a, "per_instance", False):
        out["instances"] = {"status": status, "iterations": iters,
                            "primal_objective": [s.get_primal_objective() for s in sols],
                            "relative_kkt": kkt}
    if a.sequential > 0:
        pick = np.linspace(0, a.count - 1, min(a.sequential, a.count)).astype(int)
        lpm.Solve(dms[pick[0]], st)  # warm-up
        t0 = time.perf_counter()
        seq_iters_equal = 0
        for i in pick:
            s1 = lpm.Solve(dms[i], st)
            seq_iters_equal += int(s1.get_lp_stats()["nb_iterations"] == iters[i])
        seq_s = time.perf_counter() - t0
        out.update({"sequential_sample": int(len(pick)), "sequential_s": seq_s,
                    "sequential_s_per_lp": seq_s / len(pick),
                    "sequential_lps_per_s": len(pick) / seq_s,
                    "sequential_same_iterations": seq_iters_equal,
                    "speedup_batch_vs_sequential": (len(pick) / seq_s and
                                                    (a.count / batch_s) / (len(pick) / seq_s))})
    return out


def _vertex_map_oracle(lp, w, h, picks, dev):
    """Exact derivatives of L = w.x* at the vertex of a vertex_lp, and central differences of the
    vertex map x*(c, b, A) (the solution of the same basis under the perturbed data) at the picked
    coordinates.  Test oracle: a dense FP64 LU of the basis on the GPU (torch).  Each perturbed
    vertex is x0 + dx, with dx solved from the perturbation itself (B' dx = r0 + d_rhs - dB x0,
    r0 the unperturbed residual) by the LU plus three steps of iterative refinement against the
    perturbed basis, so the difference L(+h) - L(-h) = w.(dx+ - dx-) carries no cancellation of two
    full solves."""
    import numpy as np
    import scipy.sparse as sp
    import torch

    A = sp.csr_matrix((lp.val, lp.col_idx, lp.row_off), shape=(lp.m, lp.n))
    basic = lp.basic
    nonb = np.setdiff1d(np.arange(lp.n), basic)
    pos = np.full(lp.n, -1)
    pos[basic] = np.arange(lp.m)
    t = lambda v: torch.tensor(np.asarray(v, dtype=np.float64), device=dev)
    Bc = A[:, basic].tocoo()
    B = torch.zeros(lp.m, lp.m, dtype=torch.float64, device=dev)
    B[torch.tensor(Bc.row, device=dev, dtype=torch.int64),
      torch.tensor(Bc.col, device=dev, dtype=torch.int64)] = t(Bc.data)
    LU, piv = torch.linalg.lu_factor(B)
    solve = lambda R: torch.linalg.lu_solve(LU, piv, R)
    rhs0 = t(lp.con_lo - A[:, nonb] @ lp.x_star[nonb])
    x0 = solve(rhs0[:, None])
    for _ in range(2):
        x0 = x0 + solve(rhs0[:, None] - B @ x0)
    r0 = (rhs0[:, None] - B @ x0)[:, 0]
    x0 = x0[:, 0]
    wB = t(w[basic])
    lam = torch.linalg.lu_solve(LU, piv, wB[:, None], adjoint=True)[:, 0].cpu().numpy()
    rows = np.repeat(np.arange(lp.m), np.diff(lp.row_off))
    exact = {"c": np.zeros(lp.n), "b": lam, "A": -lam[rows] * lp.x_star[lp.col_idx]}
    x0h = x0.cpu().numpy()

    def diff(cols):
        """cols: (row i, basis position k or -1, delta d, rhs change g) per perturbed vertex;
        returns w_B . dx for each."""
        P = len(cols)
        R = r0[:, None].repeat(1, P).clone()
        ii = torch.tensor([c[0] for c in cols], device=dev, dtype=torch.int64)
        kk = torch.tensor([max(c[1], 0) for c in cols], device=dev, dtype=torch.int64)
        dd = torch.tensor([c[2] if c[1] >= 0 else 0.0 for c in cols], device=dev,
                          dtype=torch.float64)
        gg = torch.tensor([c[3] for c in cols], device=dev, dtype=torch.float64)
        ar = torch.arange(P, device=dev)
        R[ii, ar] += gg - dd * x0[kk]  # r0 + d_rhs - dB x0
        X = solve(R)
        for _ in range(3):
            res = R - B @ X
            res[ii, ar] -= dd * X[kk, ar]
            X = X + solve(res)
        return wB @ X

    fd = {"c": np.zeros(len(picks["c"]))}  # the vertex does not depend on c
    cols = []
    for i in picks["b"]:
        cols += [(int(i), -1, 0.0, h), (int(i), -1, 0.0, -h)]
    L = diff(cols)
    fd["b"] = ((L[0::2] - L[1::2]) / (2 * h)).cpu().numpy()
    cols = []
    for e in picks["A"]:
        i, j = int(rows[e]), int(lp.col_idx[e])
        for sgn in (1.0, -1.0):
            if pos[j] < 0:
                cols.append((i, -1, 0.0, -sgn * h * lp.x_star[j]))
            else:
                cols.append((i, int(pos[j]), sgn * h, 0.0))
    L = diff(cols)
    fd["A"] = ((L[0::2] - L[1::2]) / (2 * h)).cpu().numpy()
    return exact, fd, x0h


def run_adjoint(a) -> dict:
    """64 x (5000 x 10000) vertex LPs: batched forward solve with crossover, the matrix-free KKT
    adjoint backward (cuOptSolutionAdjointBatch), checked against the exact derivatives of every
    instance's vertex and against central differences (h = 1e-6) of the vertex map on
    a.fd_coords coordinates of each of c, b and the A values of every instance; a.fd_solver
    instances are also differenced through the full solver (perturbed LPs re-solved with
    crossover)."""
    import numpy as np
    import torch

    from cuopt_b200 import generators as gen
    from cuopt_b200 import linear_programming as lpm
    from cuopt_b200.torch_layer import LPInstance, lp_solve_batch

    count = a.count
    lps = [gen.vertex_lp(5000, 10000, 8, seed=4000 + i) for i in range(count)]
    rng = np.random.default_rng(4)
    ws = [rng.standard_normal(lp.n) for lp in lps]
    dev = torch.device("cuda", 0)
    f = lambda v: torch.tensor(v, device=dev, dtype=torch.float64)
    i32 = lambda v: torch.tensor(v, device=dev, dtype=torch.int32)

    def instance(lp, c=None, lo=None, up=None, val=None, grad=False):
        t = LPInstance(f(lp.c if c is None else c), f(lp.con_lo if lo is None else lo),
                       f(lp.con_up if up is None else up), f(lp.val if val is None else val),
                       i32(lp.row_off), i32(lp.col_idx), f(lp.var_lo), f(lp.var_up))
        if grad:
            for x in (t.c, t.con_lo, t.con_up, t.values):
                x.requires_grad_()
        return t

    st = lpm.SolverSettings()
    st.set_optimality_tolerance(a.tol)
    st.set_parameter(lpm.CUOPT_METHOD, int(lpm.SolverMethod.PDLP))
    st.set_parameter(lpm.CUOPT_CROSSOVER, True)
    st.set_parameter(lpm.CUOPT_LOG_TO_CONSOLE, False)
    insts = [instance(lp, grad=True) for lp in lps]
    warm = instance(lps[0], grad=True)
    (x0, _), = lp_solve_batch([warm], st)  # warm-up (forward and backward)
    (f(ws[0]) * x0).sum().backward()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    outs = lp_solve_batch(insts, st)
    torch.cuda.synchronize()
    forward_s = time.perf_counter() - t0
    loss = sum((f(w) * x).sum() for w, (x, _) in zip(ws, outs))
    t0 = time.perf_counter()
    loss.backward()
    torch.cuda.synchronize()
    backward_s = time.perf_counter() - t0

    h = 1e-6
    vertex_err, basis_err, fd_err, checked = 0.0, {"c": 0.0, "b": 0.0, "A": 0.0}, 0.0, 0
    worst = None
    picks_all = []
    for q, (lp, w, t) in enumerate(zip(lps, ws, insts)):
        picks = {"c": rng.choice(lp.n, a.fd_coords, replace=False),
                 "b": rng.choice(lp.m, a.fd_coords, replace=False),
                 "A": rng.choice(lp.nnz, a.fd_coords, replace=False)}
        picks_all.append(picks)
        exact, fd, xB = _vertex_map_oracle(lp, w, h, picks, dev)
        x = outs[q][0].detach().cpu().numpy()
        vertex_err = max(vertex_err, float(np.abs(x[lp.basic] - xB).max() / max(1.0, np.abs(xB).max())))
        grads = {"c": t.c.grad.cpu().numpy(), "b": (t.con_lo.grad + t.con_up.grad).cpu().numpy(),
                 "A": t.values.grad.cpu().numpy()}
        for kind in ("c", "b", "A"):
            e = exact[kind]
            basis_err[kind] = max(basis_err[kind],
                                  float(np.abs(grads[kind] - e).max() / max(1.0, np.abs(e).max())))
            for k, d in zip(picks[kind], fd[kind]):
                g = grads[kind][k]
                err = abs(d - g) / (1.0 + abs(g))
                if err > fd_err:
                    fd_err, worst = err, {"instance": q, "kind": kind, "coordinate": int(k),
                                          "fd": float(d), "gradient": float(g)}
                checked += 1

    # Central differences through the solver (perturbed LPs re-solved with crossover, in one
    # batched call) on the first a.fd_solver instances, a few coordinates each.
    solver_err, solver_checked = 0.0, 0
    pert, keys = [], []
    for q in range(min(a.fd_solver, count)):
        lp = lps[q]
        for kind in ("c", "b", "A"):
            for k in picks_all[q][kind][:4]:
                for sgn in (1.0, -1.0):
                    c, lo, up, val = lp.c.copy(), lp.con_lo.copy(), lp.con_up.copy(), lp.val.copy()
                    if kind == "c":
                        c[k] += sgn * h
                    elif kind == "b":
                        lo[k] += sgn * h
                        up[k] += sgn * h
                    else:
                        val[k] += sgn * h
                    pert.append(instance(lp, c, lo, up, val))
                    keys.append((q, kind, int(k), sgn))
    if pert:
        res = lp_solve_batch(pert, st)
        vals = {key: float(x.detach().cpu().numpy() @ ws[key[0]]) for key, (x, _) in zip(keys, res)}
        for (q, kind, k, sgn) in keys:
            if sgn < 0:
                continue
            fdv = (vals[(q, kind, k, 1.0)] - vals[(q, kind, k, -1.0)]) / (2 * h)
            t = insts[q]
            g = {"c": t.c.grad, "b": t.con_lo.grad + t.con_up.grad, "A": t.values.grad}[kind][k].item()
            solver_err = max(solver_err, abs(fdv - g) / (1.0 + abs(g)))
            solver_checked += 1
    return {"config": "c4", "count": count, "m": 5000, "n": 10000, "forward_s": forward_s,
            "backward_s": backward_s, "adjoint_ms_per_instance": backward_s * 1e3 / count,
            "backward": "matrix-free LSQR on the GPU (cuOptSolutionAdjointBatch), one thread block "
                        "per active-set system; no dense factorisation",
            "crossover_vertex_max_rel_error": vertex_err,
            "grad_vs_exact_max_rel_error": basis_err, "exact_checked_instances": count,
            "fd_h": h, "fd_checked": checked, "fd_max_rel_error": fd_err, "fd_worst": worst,
            "fd_of": "the vertex map (perturbed vertices solved by a dense FP64 LU with refinement "
                     "on the GPU, a test oracle)",
            "fd_through_solver_checked": solver_checked,
            "fd_through_solver_max_rel_error": solver_err}


def run_climbers(a) -> dict:
    """Strong-branching shape: `count` climbers of one LP in one call vs the same LPs one by one."""
    import numpy as np

    from cuopt_b200 import generators as gen
    from cuopt_b200 import linear_programming as lpm

    m, n, k, seed = CONFIGS[a.config]
    lp = (gen.constructed_lp(m, n, k, seed=seed) if k
          else gen.skewed_lp(m, n, seed=seed, explicit_slacks=True))
    m, n = lp.m, lp.n
    rng = np.random.default_rng(7)
    var = rng.choice(n, a.count, replace=False).astype(np.int32)
    lo = lp.var_lo[var].copy()
    up = np.minimum(lp.var_up[var], rng.uniform(0.5, 3.0, a.count))

    def model(j=None, l=None, u=None):
        dm = lpm.DataModel()
        dm.set_csr_constraint_matrix(lp.val, lp.col_idx, lp.row_off)
        dm.set_objective_coefficients(lp.c)
        dm.set_constraint_lower_bounds(lp.con_lo)
        dm.set_constraint_upper_bounds(lp.con_up)
        vl, vu = lp.var_lo.copy(), lp.var_up.copy()
        if j is not None:
            vl[j], vu[j] = l, u
        dm.set_variable_lower_bounds(vl)
        dm.set_variable_upper_bounds(vu)
        return dm

    st = lpm.SolverSettings()
    st.set_optimality_tolerance(a.tol)
    st.set_parameter(lpm.CUOPT_METHOD, int(lpm.SolverMethod.PDLP))
    st.set_parameter(lpm.CUOPT_LOG_TO_CONSOLE, False)
    if a.time_limit > 0:
        st.set_parameter(lpm.CUOPT_TIME_LIMIT, a.time_limit)
    if a.iteration_limit > 0:
        st.set_parameter(lpm.CUOPT_ITERATION_LIMIT, a.iteration_limit)
    base = model()
    if a.strong_branching:
        frac = var[: a.count // 2]
        root = np.minimum(lp.x_star[frac], lp.var_up[frac] - 1.0) + 0.5
        var = np.concatenate([frac, frac])
        lo = np.concatenate([lp.var_lo[frac], np.ceil(root)])
        up = np.concatenate([np.floor(root), lp.var_up[frac]])
        run = lambda: lpm.BatchPDLPStrongBranching(base, frac, root, st)
    else:
        run = lambda: lpm.SolveClimbers(base, var, lo, up, st)
    times = []
    for _ in range(max(1, a.repeats)):
        sols, t = run()
        times.append(t)
    batch_s = min(times[1:]) if len(times) > 1 else times[0]
    status = [int(s.get_termination_status()) for s in sols]
    iters = [s.get_lp_stats()["nb_iterations"] for s in sols]
    out = {"config": a.config, "m": m, "n": n, "nnz": lp.nnz, "climbers": len(sols),
           "strong_branching": bool(a.strong_branching),
           "climbers_s": batch_s, "climbers_times_s": times, "climbers_per_s": len(sols) / batch_s,
           "optimal": status.count(1), "max_iterations": max(iters),
           "mean_iterations": float(np.mean(iters))}
    if a.sequential > 0:
        pick = np.linspace(0, len(sols) - 1, min(a.sequential, len(sols))).astype(int)
        dms = [model(var[i], lo[i], up[i]) for i in pick]
        t0 = time.perf_counter()
        if a.strong_branching:
            # One solve of the LP, then each branch from its solution (single solves recompute the
            # step size and start at primal weight 1).
            root_sol = lpm.Solve(base, st)
            for dm in dms:
                dm.set_initial_primal_solution(root_sol.get_primal_solution())
                dm.set_initial_dual_solution(root_sol.get_dual_solution())
        else:
            lpm.Solve(dms[0], st)  # warm-up
            t0 = time.perf_counter()
        same, seq_iters = 0, []
        for i, dm in zip(pick, dms):
            s1 = lpm.Solve(dm, st)
            seq_iters.append(s1.get_lp_stats()["nb_iterations"])
            same += int(seq_iters[-1] == iters[i])
        seq_s = time.perf_counter() - t0
        out.update({"sequential_sample": int(len(pick)), "sequential_s_per_lp": seq_s / len(pick),
                    "sequential_lps_per_s": len(pick) / seq_s,
                    "sequential_same_iterations": same,
                    "sequential_mean_iterations": float(np.mean(seq_iters)),
                    "speedup_climbers_vs_sequential": (len(sols) / batch_s) / (len(pick) / seq_s)})
    return out


if __name__ == "__main__":
    main()
