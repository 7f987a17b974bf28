#!/usr/bin/env python
"""PDLP benchmark on one B200 (or N replicas under torchrun).

Workload (default, c1): the seeded 1,000,000 x 2,000,000 LP with 8 non-zeros per column
(16M non-zeros), equality rows, bounds [0, 10], optimum known by construction.  One "step" is one
full solve to 1e-6 relative KKT (all six tolerances 1e-6), mixed precision (FP32 matrix and
iterates, FP64 termination / restart / step ratio).  The same solve in plain FP64 is timed beside it.

  value   LPs solved per second from device-resident inputs (cuOptSolveDevice), CUDA events on the
          solve's stream, max over ranks; the matrices (>= 200 MB each) exceed the 126 MB L2.
  e2e     the same through the reference-compatible C API with host buffers
          (cuOptCreateRangedProblem + cuOptSolve + cuOptGet* including the H2D / D2H copies).
  roofline  the dominant fused PDHG sweep, timed per launch with CUDA events
            (cuOptProfilePDHGSweeps), against the measured HBM copy bandwidth; beside it, the
            sweep's gathers per second against the measured random-gather ceiling
            (cuOptProfileGatherRate), the bound of sweeps over uniformly random sparsity.
  parity  every leg reports its relative KKT, its objective error against the optimum known by
          construction, and its gap to the FP64 oracle (the CPU restatement of the reference's
          algorithm: solved live for the CPU baseline, else tests/golden/oracle_results.json).
          An objective within 1e-6 is met by the legs refined to 1e-8 relative KKT; 1e-6 KKT
          alone does not bound it.
  cpu_baseline  whole FP64 oracle solves of the workload on all host threads (scaling, step size,
            termination checks, restarts; no extrapolation).
  c0      the 2000 x 5000 LP (L2-resident, launch-bound): time to 1e-6, iterations/s, time and
          launches per iteration (plain iterations replay CUDA graphs), against the reference's own
          CPU dual simplex (time-limited) and the oracle.
  batch_c3  512 seeded LPs of uneven sizes (m log-uniform in [200, 20000], n = 2.5 m,
            6-12 non-zeros per column) in one cuOptBatchSolve call, against all 512 solved one by
            one with cuOptSolve: FP64 at 1e-6 and 1e-8, mixed precision at 1e-6 and refined in
            FP64 to 1e-8.
  adjoint_c4  64 non-degenerate 5000 x 10000 LPs solved in one batched call with
            crossover, L = sum w * x* back-propagated through the matrix-free KKT adjoint,
            gradients checked against every instance's exact derivatives and central differences
            (h = 1e-6, 32 coordinates of each of c, b and A per instance).

`--impl reference` times the CPU oracle alone (rank 0) on the same workload and metric.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "time-to-1e-6 KKT & PDHG iter/s (mixed vs FP64); batched LPs/s; SpMV GB/s"
UNIT = "LPs/s to 1e-6 rel. KKT"
CONFIGS = {
    # name: (m, n, nnz per column, seed)
    "c1": (1_000_000, 2_000_000, 8, 1000),
    "c0": (2_000, 5_000, 8, 0),
    "c1_small": (750_000, 1_500_000, 8, 1000),
}
ORACLE_FIXTURE = ROOT / "tests" / "golden" / "oracle_results.json"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic(kernel: str, precision: str):
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return d.get(f"{kernel}_{precision}")


def _oracle_fixture():
    return json.loads(ORACLE_FIXTURE.read_text()) if ORACLE_FIXTURE.exists() else None


def rel_err(a: float, b: float) -> float:
    return abs(a - b) / max(1.0, abs(b))


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_lp(cfg: str):
    from cuopt_b200 import generators as gen
    m, n, k, seed = CONFIGS[cfg]
    return gen.constructed_lp(m, n, k, seed=seed, name=cfg)


def settings_handle(L, tol, precision, iteration_limit=None, refine_passes=0, refine_tol=1e-8,
                    time_limit=None):
    h = C.c_void_p()
    assert L.cuOptCreateSolverSettings(C.byref(h)) == 0
    for name in ("absolute_primal_tolerance", "relative_primal_tolerance", "absolute_dual_tolerance",
                 "relative_dual_tolerance", "absolute_gap_tolerance", "relative_gap_tolerance"):
        assert L.cuOptSetFloatParameter(h, name.encode(), tol) == 0
    assert L.cuOptSetIntegerParameter(h, b"method", 1) == 0
    assert L.cuOptSetIntegerParameter(h, b"pdlp_precision", precision) == 0
    assert L.cuOptSetParameter(h, b"log_to_console", b"false") == 0
    if iteration_limit is not None:
        assert L.cuOptSetIntegerParameter(h, b"iteration_limit", int(iteration_limit)) == 0
    if time_limit is not None:
        assert L.cuOptSetFloatParameter(h, b"time_limit", float(time_limit)) == 0
    if refine_passes:
        assert L.cuOptSetIntegerParameter(h, b"pdlp_refinement_passes", int(refine_passes)) == 0
        assert L.cuOptSetFloatParameter(h, b"pdlp_refinement_tolerance", float(refine_tol)) == 0
    return h


class DeviceLP:
    """The LP in device memory (torch tensors), user order."""

    def __init__(self, lp, torch, device):
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), device=device, dtype=dt)
        self.m, self.n = lp.m, lp.n
        self.off = t(lp.row_off, torch.int32)
        self.idx = t(lp.col_idx, torch.int32)
        self.val = t(lp.val, torch.float64)
        self.c = t(lp.c, torch.float64)
        self.lo = t(lp.con_lo, torch.float64)
        self.up = t(lp.con_up, torch.float64)
        self.vl = t(lp.var_lo, torch.float64)
        self.vu = t(lp.var_up, torch.float64)
        self.x = torch.empty(lp.n, device=device, dtype=torch.float64)
        self.y = torch.empty(lp.m, device=device, dtype=torch.float64)
        self.rc = torch.empty(lp.n, device=device, dtype=torch.float64)

    def ptrs(self):
        return [C.c_void_p(a.data_ptr()) for a in
                (self.c, self.off, self.idx, self.val, self.lo, self.up, self.vl, self.vu)]


def solve_device(L, dlp, settings, stream_ptr):
    from cuopt_b200._lib import PDLPStatistics, stats_dict
    st = PDLPStatistics()
    status = C.c_int32()
    rc = L.cuOptSolveDevice(dlp.m, dlp.n, 1, 0.0, *dlp.ptrs(), settings, C.c_void_p(stream_ptr),
                            C.c_void_p(dlp.x.data_ptr()), C.c_void_p(dlp.y.data_ptr()),
                            C.c_void_p(dlp.rc.data_ptr()), C.byref(st), C.byref(status))
    if rc != 0:
        raise RuntimeError(f"cuOptSolveDevice returned {rc}")
    return status.value, stats_dict(st)


def form_info(st):
    """The tuned choices of a solve: the form of the plain iterations and the cycle timings it was
    chosen on (pdlp_persistent_iterations = -1: CUDA graphs, the persistent cooperative kernel and,
    for small LPs, the cluster-resident kernel), and the plain sweeps' warps per block with the ms
    per launch of 4, 8 and 16 (pdlp_sweep_warps_per_block = 0)."""
    ms = list(st["sweep_block_shape_ms"])
    return {"form": {0: "graphs", 1: "persistent", 2: "cluster"}.get(st["plain_iteration_form"],
                                                                       "undecided"),
            "persistent_blocks": st["persistent_blocks"],
            "us_per_iteration_graphs": st["plain_iteration_us_graphs"],
            "us_per_iteration_persistent": st["plain_iteration_us_persistent"],
            "us_per_iteration_cluster": st["plain_iteration_us_cluster"],
            "sweep_warps_per_block": {"primal": st["sweep_warps_per_block_primal"],
                                      "dual": st["sweep_warps_per_block_dual"]},
            "sweep_ms_by_warps_per_block": {"primal": dict(zip(("4", "8", "16"), ms[:3])),
                                            "dual": dict(zip(("4", "8", "16"), ms[3:]))}}


def grid_barrier_costs(L):
    """Microseconds per grid barrier of the persistent kernel, alone (cuOptProbeGridBarrier)."""
    out = {}
    for blocks in (20, 148, 296, 740):
        st, ms = C.c_int32(), C.c_double()
        if L.cuOptProbeGridBarrier(blocks, 2000, 0, 5000.0, None, C.byref(st), C.byref(ms)) == 0:
            out[str(blocks)] = 1e3 * ms.value / 2000 if st.value == 0 else None
    return out


def solve_e2e(L, lp, pinned, settings):
    """One solve through the reference-compatible C API from (pinned) host buffers."""
    h = C.c_void_p()
    p = lambda a: C.c_void_p(a.ctypes.data)
    rc = L.cuOptCreateRangedProblem(lp.m, lp.n, 1, 0.0, p(pinned["c"]), p(pinned["off"]),
                                    p(pinned["idx"]), p(pinned["val"]), p(pinned["lo"]),
                                    p(pinned["up"]), p(pinned["vl"]), p(pinned["vu"]),
                                    b"C" * lp.n, C.byref(h))
    assert rc == 0, rc
    sol = C.c_void_p()
    L.cuOptSolve(h, settings, C.byref(sol))
    status = C.c_int32()
    L.cuOptGetTerminationStatus(sol, C.byref(status))
    L.cuOptGetPrimalSolution(sol, p(pinned["x"]))
    L.cuOptGetDualSolution(sol, p(pinned["y"]))
    L.cuOptGetReducedCosts(sol, p(pinned["rc"]))
    L.cuOptDestroySolution(C.byref(sol))
    L.cuOptDestroyProblem(C.byref(h))
    return status.value


def oracle_solves(lp, steps: int, warmup: int, budget_s: float, threads: int, tol: float = 1e-6):
    """Whole FP64 oracle solves of `lp` to `tol` (scaling, step size, termination checks,
    restarts) on `threads` host threads.  Warm-up: `warmup` bounded runs of 20 iterations.  Timed:
    up to `steps` solves, stopping early once the next one would end past `budget_s` (the first
    always runs).  Returns (seconds per solve, solves timed, last result dict)."""
    from oracle import oracle as O
    for _ in range(warmup):
        O.solve(lp, tol=tol, iteration_limit=20, threads=threads)
    times, res = [], None
    t_all = time.perf_counter()
    for _ in range(max(1, steps)):
        t0 = time.perf_counter()
        res, _, _, _ = O.solve(lp, tol=tol, threads=threads)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_all + times[-1] > budget_s:
            break
    return float(np.mean(times)), len(times), res


def bench_config(args, lp, world):
    """The workload both arms report (the reference arm times the same one on the host); the
    arithmetic each arm uses is in its own `dtype` / `precision` keys."""
    return {"workload": f"{args.config}: {lp.m}x{lp.n} LP, {lp.nnz} nnz, Stable3 PDLP to 1e-6 "
                        "relative KKT", "replicas": world,
            "l2": "inputs larger than L2 (matrix 16M nnz, >= 190 MB per copy)",
            "parallelism": f"replicas x{world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    lp = make_lp(args.config)
    threads = O.max_threads()
    s, timed, res = oracle_solves(lp, args.steps, args.warmup, args.reference_seconds, threads)
    value = 1.0 / s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": timed, "steps_requested": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * s, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "precision": "fp64",
        "data": "synthetic (seeded generator, optimum known by construction)",
        "config": bench_config(args, lp, 1),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{timed} whole FP64 oracle solve(s) of the workload to 1e-6 "
                                   f"relative KKT on {threads} threads ({s:.2f} s each; warm-up: "
                                   f"{args.warmup} runs of 20 iterations); steps past a "
                                   f"{args.reference_seconds:.0f} s budget are not run"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "status": res["status"], "iterations": res["iterations"],
        "pdhg_iter_per_s": res["iterations"] / s,
        "objective_rel_error": rel_err(res["primal_obj"], lp.optimal_objective),
    }
    print(json.dumps(line), flush=True)


class Replicas:
    """Replica plumbing (one process per GPU, every rank solves its own copy of the workload, no
    data-path collective): a barrier around the timed region and the max over ranks of a time.
    backend "nccl" with a CUDA device on the GPU box, "gloo" on CPU (tests)."""

    def __init__(self, world: int, rank: int, device=None, backend: str = "nccl",
                 timeout_s: float = 600.0):
        import torch
        import torch.distributed as dist
        self.world, self.rank, self.device = world, rank, device
        self._torch, self._dist = torch, dist
        if world > 1:
            import datetime
            kw = {"device_id": device} if backend == "nccl" else {}
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s),
                                    world_size=world, rank=rank, **kw)

    def barrier(self):
        if self.world > 1:
            self._dist.barrier()

    def max(self, v: float) -> float:
        if self.world == 1:
            return v
        t = self._torch.tensor([v], device=self.device, dtype=self._torch.float64)
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.world > 1:
            self._dist.destroy_process_group()


def parity(lp, st, oracle=None):
    """Per-result correctness record: relative KKT (reported by the solver), objective error
    against the constructed optimum, and (when the oracle's result at the same tolerance is given)
    the gap to the FP64 oracle's objective, status and iteration count."""
    out = {"status": st[0], "iterations": st[1]["number_of_steps_taken"],
           "relative_kkt": max(st[1]["l2_relative_primal_residual"],
                               st[1]["l2_relative_dual_residual"], st[1]["relative_gap"]),
           "objective_rel_error": rel_err(st[1]["primal_objective"], lp.optimal_objective)}
    if oracle is not None:
        out["objective_rel_error_vs_oracle"] = rel_err(st[1]["primal_objective"],
                                                       oracle["primal_objective"])
        out["oracle_status"] = oracle["status"]
        out["oracle_iterations"] = oracle["iterations"]
    return out


def batch_parity(res: dict, lps, oracle_batch, tol_key: str) -> dict:
    """Summary of a batch's per-instance results against the oracle fixture at its tolerance."""
    inst = res.pop("instances")
    out = {"instances": len(lps)}
    if oracle_batch is None:
        return out
    want = [o[tol_key] for o in oracle_batch]
    out["status_equal_oracle"] = sum(int(a == w["status"]) for a, w in zip(inst["status"], want))
    out["iterations_equal_oracle"] = sum(int(a == w["iterations"])
                                         for a, w in zip(inst["iterations"], want))
    out["max_objective_rel_error_vs_oracle"] = max(
        rel_err(a, w["primal_objective"]) for a, w in zip(inst["primal_objective"], want))
    return out


def run_c0(L, torch, device, sptr, args, O=None):
    """The 2000 x 5000 LP: time to 1e-6 (FP64 and mixed) from device-resident inputs, iterations
    per second, and the per-iteration overhead beyond the sweeps' device time."""
    lp = make_lp("c0")
    dlp = DeviceLP(lp, torch, device)
    stream = torch.cuda.current_stream(device)
    ref = None
    out = {"config": "c0", "m": lp.m, "n": lp.n, "nnz": lp.nnz}
    if O is not None:
        r, _, _, _ = O.solve(lp, tol=1e-6)
        ref = {"status": r["status"], "iterations": r["iterations"], "primal_objective": r["primal_obj"]}
    for prec, name in ((0, "fp64"), (1, "mixed")):
        sh = settings_handle(L, 1e-6, prec)
        for _ in range(3):
            solve_device(L, dlp, sh, sptr)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sts = [solve_device(L, dlp, sh, sptr) for _ in range(args.c0_steps)]
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.c0_steps
        L.cuOptDestroySolverSettings(C.byref(sh))
        st = sts[-1][1]
        it = st["number_of_steps_taken"]
        out[name] = {"ms_per_solve": ms, "lps_per_s": 1000.0 / ms,
                     "pdhg_iter_per_s": it / (st["loop_time"] or 1e-9),
                     "setup_ms": 1e3 * st["setup_time"],
                     "us_per_iteration": 1e6 * st["loop_time"] / max(it, 1),
                     "kernel_launches_per_iteration": st["kernel_launches"] / max(it, 1),
                     "iteration_loop": form_info(st),
                     **parity(lp, sts[-1], ref if name == "fp64" else None)}
    if O is not None:
        s, timed, _ = oracle_solves(lp, 3, 1, 30.0, O.max_threads())
        out["cpu_baseline_port"] = {"value": 1.0 / s, "unit": UNIT, "cores": O.max_threads(),
                                    "kind": "port",
                                    "sample": f"{timed} whole FP64 oracle PDLP solves "
                                              f"({s * 1e3:.0f} ms each)"}
        from oracle import ref_simplex as R
        if R.available():
            # The reference's own CPU dual simplex (solve_linear_program), compiled from its
            # sources, under a time limit: its status, time, residual and objective error.
            res, _ = R.solve(lp, time_limit=args.simplex_seconds,
                             timeout=args.simplex_seconds + 120)
            out["cpu_baseline"] = {
                "value": (1.0 / res["solve_seconds"]) if res["status"] == "OPTIMAL" else 0.0,
                "unit": UNIT, "cores": res["threads"], "kind": "reference",
                "sample": f"one solve_linear_program call (the reference's CPU dual simplex) "
                          f"with a {args.simplex_seconds:.0f} s time limit",
                "status": res["status"], "solve_seconds": res["solve_seconds"],
                "primal_residual": res["primal_residual"],
                "objective_rel_error": rel_err(res["objective"], lp.optimal_objective)}
        else:
            out["cpu_baseline"] = {**out["cpu_baseline_port"],
                                   "note": "oracle/_ref/ref_dual_simplex not built"}
    return out


def run_c2(L, torch, device, sptr, args):
    """The skewed-sparsity LP (500k x 1.5M, Zipf(1.3) row lengths capped at 5000, slacks added):
    the plain sweeps' time and rates per row-length class (FP64 and mixed), and a solve sample of
    a fixed iteration count (iterations per second and the relative KKT it reaches).  The full
    solve to 1e-6 takes far longer than a bench run (its evidence is a separate measurement)."""
    from cuopt_b200 import generators as gen
    from cuopt_b200.profile import sweep_classes
    from cuopt_b200.profile import CONFIGS as PCONF

    m0, n0, _, seed = PCONF["c2"]
    lp = gen.skewed_lp(m0, n0, seed=seed, explicit_slacks=True)
    dlp = DeviceLP(lp, torch, device)
    out = {"config": "c2", "m": lp.m, "n": lp.n, "nnz": lp.nnz}
    for prec, name, elem in ((0, "fp64", 8), (1, "mixed", 4)):
        sh = settings_handle(L, 1e-6, prec)
        vals = [C.c_double() for _ in range(4)]
        code = L.cuOptProfilePDHGSweeps(lp.m, lp.n, *dlp.ptrs(), sh, C.c_void_p(sptr), 10,
                                        *[C.byref(v) for v in vals])
        if code != 0:
            raise RuntimeError(f"cuOptProfilePDHGSweeps returned {code}")
        leg = {"primal_sweep_ms": vals[0].value, "dual_sweep_ms": vals[1].value,
               "primal_gbs": vals[2].value / vals[0].value / 1e6,
               "dual_gbs": vals[3].value / vals[1].value / 1e6,
               "classes": sweep_classes(L, lp.m, lp.n, dlp.ptrs(), sh, C.c_void_p(sptr), 10, elem)}
        L.cuOptDestroySolverSettings(C.byref(sh))
        sh = settings_handle(L, 1e-6, prec, iteration_limit=args.c2_iterations)
        status, st = solve_device(L, dlp, sh, sptr)
        L.cuOptDestroySolverSettings(C.byref(sh))
        it = st["number_of_steps_taken"]
        leg["solve_sample"] = {"iterations": it, "status": status,
                               "continued_in_fp64": int(st["refinement_passes"] > 0),
                               "pdhg_iter_per_s": it / (st["loop_time"] or 1e-9),
                               "setup_s": st["setup_time"], "relative_kkt": max(
                                   st["l2_relative_primal_residual"],
                                   st["l2_relative_dual_residual"], st["relative_gap"])}
        out[name] = leg
    return out


def run_b200(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    replicas = Replicas(world, rank, device, "nccl")
    barrier, max_over_ranks = replicas.barrier, replicas.max

    from cuopt_b200._lib import lib
    L = lib()
    lp = make_lp(args.config)
    dlp = DeviceLP(lp, torch, device)
    stream = torch.cuda.current_stream(device)
    sptr = stream.cuda_stream
    tol = 1e-6
    s_mixed = settings_handle(L, tol, 1)
    s_fp64 = settings_handle(L, tol, 0)
    fixture = _oracle_fixture()
    fx_single = (fixture or {}).get("single", {}).get(args.config)
    lone = rank == 0 and world == 1

    def timed(settings, steps, warmup):
        for _ in range(warmup):
            solve_device(L, dlp, settings, sptr)
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []
        with ClockSampler(local) as clk:
            ev0.record(stream)
            for _ in range(steps):
                stats.append(solve_device(L, dlp, settings, sptr))
            ev1.record(stream)
            torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1) / steps
        return max_over_ranks(ms), stats, clk.summary()

    ms_mixed, st_mixed, clocks = timed(s_mixed, args.steps, args.warmup)
    last_mixed = st_mixed[-1][1]
    fx6 = fx_single["1e-06"] if fx_single else None
    fx8 = fx_single["1e-08"] if fx_single else None
    mixed = parity(lp, st_mixed[-1], fx6)

    fp64 = None
    if not args.no_fp64:
        ms_fp64, st_fp64, _ = timed(s_fp64, max(1, args.fp64_steps), max(1, args.fp64_warmup))
        last_fp64 = st_fp64[-1][1]
        fp64 = {"ms_per_solve": ms_fp64,
                "pdhg_iter_per_s": last_fp64["number_of_steps_taken"] / (last_fp64["loop_time"] or 1e-9),
                "setup_s": last_fp64["setup_time"], "speedup_mixed_vs_fp64": ms_fp64 / ms_mixed,
                **parity(lp, st_fp64[-1], fx6)}

    # 1e-8 relative KKT: mixed precision to 1e-6 continued in FP64, and FP64 from the start.
    refine = fp64_8 = None
    if not args.no_refine:
        s_ref = settings_handle(L, tol, 1, refine_passes=1, refine_tol=1e-8, time_limit=60.0)
        ms_ref, st_ref, _ = timed(s_ref, 1, 1)
        L.cuOptDestroySolverSettings(C.byref(s_ref))
        refine = {"ms_per_solve": ms_ref, "refinement_passes": st_ref[-1][1]["refinement_passes"],
                  **parity(lp, st_ref[-1], fx8)}
        s_f8 = settings_handle(L, 1e-8, 0, time_limit=60.0)
        ms_f8, st_f8, _ = timed(s_f8, 1, 1)
        L.cuOptDestroySolverSettings(C.byref(s_f8))
        fp64_8 = {"ms_per_solve": ms_f8, **parity(lp, st_f8[-1], fx8)}
        refine["speedup_vs_fp64_to_1e-8"] = ms_f8 / ms_ref

    # Roofline of the dominant fused sweep (mixed precision = the headline path)
    prof = {}
    for prec, name in ((1, "mixed"), (0, "fp64")):
        a, b, ba, bb = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        sh = settings_handle(L, tol, prec)
        rc = L.cuOptProfilePDHGSweeps(lp.m, lp.n, *dlp.ptrs(), sh, C.c_void_p(sptr),
                                      args.profile_iters, C.byref(a), C.byref(b), C.byref(ba),
                                      C.byref(bb))
        L.cuOptDestroySolverSettings(C.byref(sh))
        assert rc == 0, rc
        prof[name] = {"primal_sweep_ms": a.value, "dual_sweep_ms": b.value,
                      "primal_sweep_bytes": ba.value, "dual_sweep_bytes": bb.value}
    peak, peak_kind = _peaks()
    pm = prof["mixed"]
    dom = "dual" if pm["dual_sweep_ms"] >= pm["primal_sweep_ms"] else "primal"
    achieved = pm[f"{dom}_sweep_bytes"] / (pm[f"{dom}_sweep_ms"] * 1e-3) / 1e9
    from cuopt_b200.profile import gather_rates
    rates = gather_rates(lp.m, lp.n, lp.nnz, C.c_void_p(sptr))
    g_peak = rates["dual_gather_xbar_fp32" if dom == "dual" else "primal_gather_y_fp32"]["gathers_per_s"]
    g_ach = lp.nnz / (pm[f"{dom}_sweep_ms"] * 1e-3)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "kernel": f"{dom} sweep (sell_map_kernel, mixed precision)",
                "traffic": _traffic(dom, "mixed"),
                "gather": {"achieved": g_ach / 1e9, "peak": g_peak / 1e9, "unit": "G gathers/s",
                           "frac": g_ach / g_peak, "peak_kind": "measured live (cuOptProfileGatherRate)",
                           "hbm_frac_at_gather_peak": pm[f"{dom}_sweep_bytes"] / (lp.nnz / g_peak) / 1e9 / peak},
                "gather_ceilings": rates,
                "iteration_achieved_gbs_mixed": (pm["primal_sweep_bytes"] + pm["dual_sweep_bytes"])
                / ((pm["primal_sweep_ms"] + pm["dual_sweep_ms"]) * 1e-3) / 1e9,
                "iteration_achieved_gbs_fp64": (prof["fp64"]["primal_sweep_bytes"] + prof["fp64"]["dual_sweep_bytes"])
                / ((prof["fp64"]["primal_sweep_ms"] + prof["fp64"]["dual_sweep_ms"]) * 1e-3) / 1e9,
                "sweeps": prof}

    # e2e through the C API with host buffers (pinned), mixed precision
    pin = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a, dtype=dt)).pin_memory().numpy()
    pinned = {"c": pin(lp.c, np.float64), "off": pin(lp.row_off, np.int32),
              "idx": pin(lp.col_idx, np.int32), "val": pin(lp.val, np.float64),
              "lo": pin(lp.con_lo, np.float64), "up": pin(lp.con_up, np.float64),
              "vl": pin(lp.var_lo, np.float64), "vu": pin(lp.var_up, np.float64),
              "x": pin(np.zeros(lp.n), np.float64), "y": pin(np.zeros(lp.m), np.float64),
              "rc": pin(np.zeros(lp.n), np.float64)}
    solve_e2e(L, lp, pinned, s_mixed)
    barrier()
    torch.cuda.synchronize()
    e2e_steps = args.e2e_steps or args.steps
    t0 = time.perf_counter()
    e2e_status = [solve_e2e(L, lp, pinned, s_mixed) for _ in range(e2e_steps)]
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / e2e_steps)
    h2d = (lp.m + 1) * 4 + lp.nnz * 12 + lp.n * 8 * 3 + lp.m * 8 * 2
    d2h = (2 * lp.n + lp.m) * 8

    O = None
    if lone and not args.no_cpu:
        from oracle import oracle as O

    # CPU baseline (rank 0, N = 1 only): whole FP64 oracle solves of the workload.
    cpu = None
    if O is not None:
        threads = O.max_threads()
        s, timed_n, res = oracle_solves(lp, 1, 1, args.cpu_seconds, threads)
        cpu = {"value": 1.0 / s, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{timed_n} whole FP64 oracle solve(s) of the workload to 1e-6 relative "
                         f"KKT on {threads} threads ({s:.2f} s each)",
               "status": res["status"], "iterations": res["iterations"],
               "pdhg_iter_per_s": res["iterations"] / s}
        live = {"status": res["status"], "iterations": res["iterations"],
                "primal_objective": res["primal_obj"]}
        if fp64 is not None:
            fp64["live_oracle"] = {k: parity(lp, st_fp64[-1], live)[k] for k in
                                   ("objective_rel_error_vs_oracle", "oracle_status",
                                    "oracle_iterations")}
        mixed["objective_rel_error_vs_live_oracle"] = rel_err(last_mixed["primal_objective"],
                                                              res["primal_obj"])

    c0 = run_c0(L, torch, device, sptr, args, O) if lone and not args.no_c0 else None
    c2 = run_c2(L, torch, device, sptr, args) if lone and not args.no_c2 else None

    # 512 uneven LPs in one batched call vs all of them one by one (rank 0, N = 1): FP64 at 1e-6
    # and 1e-8, mixed precision at 1e-6 and refined in FP64 to 1e-8.
    batch = batch_mixed = None
    if lone and not args.no_batch:
        from cuopt_b200.profile import batch_models, run_batch
        models = batch_models(512)
        ob = (fixture or {}).get("batch")
        ns = lambda **kw: argparse.Namespace(count=512, time_limit=120.0, per_instance=True, **kw)
        batch = run_batch(ns(sequential=args.batch_sequential, repeats=3, tol=1e-6,
                             batch_precision="fp64"), models)
        batch["parity"] = batch_parity(batch, models[0], ob, "1e-06")
        b8 = run_batch(ns(sequential=0, repeats=2, tol=1e-8, batch_precision="fp64"), models)
        b8["parity"] = batch_parity(b8, models[0], ob, "1e-08")
        batch["fp64_to_1e-8"] = b8
        batch_mixed = run_batch(ns(sequential=args.batch_sequential, repeats=3, tol=1e-6,
                                   batch_precision="mixed"), models)
        batch_mixed["parity"] = batch_parity(batch_mixed, models[0], None, "1e-06")
        br = run_batch(ns(sequential=0, repeats=2, tol=1e-6, batch_precision="mixed", refine=1),
                       models)
        br["parity"] = batch_parity(br, models[0], ob, "1e-08")
        batch_mixed["refined_to_1e-8"] = br
        # The batch as specified: the FP32-bulk batch against plain FP64 solves one by one.
        if batch.get("sequential_lps_per_s"):
            batch_mixed["speedup_vs_sequential_fp64"] = (batch_mixed["batch_lps_per_s"] /
                                                         batch["sequential_lps_per_s"])
    # 64 non-degenerate 5000 x 10000 LPs, batched forward (crossover) + KKT adjoint.
    adjoint = None
    if lone and not args.no_adjoint:
        from cuopt_b200.profile import run_adjoint
        adjoint = run_adjoint(argparse.Namespace(count=64, tol=1e-6,
                                                 fd_coords=args.adjoint_fd_coords, fd_solver=2))

    value = world * 1000.0 / ms_mixed
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 mixed",
        "precision": "mixed (FP32 matrix and iterates, FP64 termination / restart / step ratio)",
        "data": "synthetic (seeded generator, optimum known by construction)",
        "config": bench_config(args, lp, world),
        "pdhg_iter_per_s": last_mixed["number_of_steps_taken"] / (last_mixed["loop_time"] or 1e-9),
        "setup_s": last_mixed["setup_time"], "loop_s": last_mixed["loop_time"],
        **mixed, "fp64": fp64, "mixed_refined_to_1e-8": refine, "fp64_to_1e-8": fp64_8,
        "objective_bound": "1e-6 relative KKT does not bound the objective error by 1e-6 (the "
                           "oracle itself is 6.8e-6 off on batch instance 284 at 1e-6); the legs "
                           "refined to 1e-8 are the ones held to 1e-6",
        "iteration_loop": {**form_info(last_mixed), "grid_barrier_us": grid_barrier_costs(L)},
        "c0": c0, "c2": c2, "batch_c3": batch, "batch_c3_mixed": batch_mixed,
        "adjoint_c4": adjoint,
        "roofline": roofline, "cpu_baseline": cpu,
        "e2e": {"value": world * 1000.0 / e2e_ms, "unit": UNIT,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "steps": e2e_steps, "status": e2e_status},
        "clocks": clocks, "gpu_launches": int(sum(st["kernel_launches"] for _, st in st_mixed)),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    L.cuOptDestroySolverSettings(C.byref(s_mixed))
    L.cuOptDestroySolverSettings(C.byref(s_fp64))
    replicas.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c1")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--fp64-warmup", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=0, help="0: as many as --steps")
    ap.add_argument("--c0-steps", type=int, default=10)
    ap.add_argument("--simplex-seconds", type=float, default=60.0,
                    help="c0 leg: time limit of the reference's CPU dual simplex")
    ap.add_argument("--profile-iters", type=int, default=50)
    ap.add_argument("--cpu-seconds", type=float, default=60.0,
                    help="GPU arm: time budget of the whole-solve CPU baseline")
    ap.add_argument("--reference-seconds", type=float, default=120.0,
                    help="reference arm: time budget of its timed whole solves")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-refine", action="store_true")
    ap.add_argument("--no-c0", action="store_true")
    ap.add_argument("--no-c2", action="store_true")
    ap.add_argument("--c2-iterations", type=int, default=4000,
                    help="iteration count of the config-2 solve sample")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adjoint-fd-coords", type=int, default=32,
                    help="adjoint batch: coordinates per kind checked by central differences")
    ap.add_argument("--batch-sequential", type=int, default=512,
                    help="512-LP batch: instances also solved one by one")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
