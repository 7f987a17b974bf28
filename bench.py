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
  roofline  the dominant fused PDHG sweep, timed per launch with CUDA events (cuOptProfilePDHGSweeps)
            against the measured HBM copy bandwidth.
  cpu_baseline  the oracle (FP64 restatement of the same algorithm) on the host cores: a bounded
            number of PDHG iterations, scaled by the iterations the solve needs.
  batch_c3  512 seeded LPs of uneven sizes (m log-uniform in [200, 20000], n = 2.5 m,
            6-12 non-zeros per column) solved in FP64 to 1e-6 by one cuOptBatchSolve call, against
            a sample of the same LPs solved one by one with cuOptSolve.
  batch_c3_mixed  the same in mixed precision (batch and single solves): Lanczos step sizes, FP32
            sweeps; an instance whose FP32 iterates stall continues in FP64.  The batch as
            specified (FP32 bulk against plain FP64 solves one by one) is its
            speedup_vs_sequential_fp64.
  adjoint_c4  64 non-degenerate 5000 x 10000 LPs solved in one batched call with
            crossover, L = sum w * x* back-propagated through the KKT adjoint, gradients checked
            against the exact basis derivatives and central differences (h = 1e-6).

`--impl reference` times that CPU implementation alone (rank 0) on the same workload and metric.
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
CONFIGS = {
    # name: (m, n, nnz per column, seed)
    "c1": (1_000_000, 2_000_000, 8, 1000),
    "c0": (2_000, 5_000, 8, 0),
    "c1_small": (750_000, 1_500_000, 8, 1000),
}
# FP64 Stable3 iterations to 1e-6 on the 1M x 2M LP (the oracle and the GPU FP64 path follow the same
# iterates; measured by the FP64 leg of this benchmark on a B200).  Used only to scale the CPU
# per-iteration time of the reference arm into the LPs/s unit.
FP64_ITERATIONS_C1 = 1700


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
    from cuopt_b200._lib import PDLPStatistics
    st = PDLPStatistics()
    status = C.c_int32()
    rc = L.cuOptSolveDevice(dlp.m, dlp.n, 1, 0.0, *dlp.ptrs(), settings, C.c_void_p(stream_ptr),
                            C.c_void_p(dlp.x.data_ptr()), C.c_void_p(dlp.y.data_ptr()),
                            C.c_void_p(dlp.rc.data_ptr()), C.byref(st), C.byref(status))
    if rc != 0:
        raise RuntimeError(f"cuOptSolveDevice returned {rc}")
    return status.value, {f: getattr(st, f) for f, _ in PDLPStatistics._fields_}


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


def cpu_sample(lp, target_s: float, threads: int):
    """Seconds per PDHG iteration of the oracle on the host cores (bounded sample)."""
    from oracle import oracle as O
    t2 = O.pdhg_seconds(lp, 2, threads)
    iters = int(max(3, min(200, target_s / max(t2 / 2, 1e-6))))
    t = O.pdhg_seconds(lp, iters, threads)
    return t / iters, iters


def bench_config(args, lp, world):
    """The workload both arms report (the reference arm times the same one on the host)."""
    return {"workload": f"{args.config}: {lp.m}x{lp.n} LP, {lp.nnz} nnz, Stable3 PDLP to 1e-6 "
                        "relative KKT, mixed precision", "replicas": world,
            "l2": "inputs larger than L2 (matrix 16M nnz, >= 190 MB per copy)",
            "parallelism": f"replicas x{world}"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle import oracle as O
    lp = make_lp(args.config)
    threads = O.max_threads()
    iters_needed = args.cpu_iterations or FP64_ITERATIONS_C1 or 10000
    samples = []
    for i in range(args.warmup + args.steps):
        s_per_iter, n = cpu_sample(lp, args.cpu_seconds / max(1, args.warmup + args.steps), threads)
        if i >= args.warmup:
            samples.append(s_per_iter)
    s_iter = float(np.mean(samples))
    value = 1.0 / (s_iter * iters_needed)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "LPs/s to 1e-6 rel. KKT",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * s_iter * iters_needed, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(args, lp, 1),
        "cpu_baseline": {"value": value, "unit": "LPs/s to 1e-6 rel. KKT", "cores": threads,
                         "kind": "port",
                         "sample": f"oracle FP64 PDHG, {n} iterations per step on {threads} threads, "
                                   f"{s_iter * 1e3:.1f} ms/iteration x {iters_needed} iterations"},
        "e2e": {"value": value, "unit": "LPs/s to 1e-6 rel. KKT", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "pdhg_iter_per_s": 1.0 / s_iter,
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
    from cuopt_b200 import generators as gen
    L = lib()
    lp = make_lp(args.config)
    dlp = DeviceLP(lp, torch, device)
    stream = torch.cuda.current_stream(device)
    sptr = stream.cuda_stream
    tol = 1e-6
    s_mixed = settings_handle(L, tol, 1)
    s_fp64 = settings_handle(L, tol, 0)

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
                status, st = solve_device(L, dlp, settings, sptr)
                stats.append((status, st))
            ev1.record(stream)
            torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1) / steps
        return max_over_ranks(ms), stats, clk.summary()

    ms_mixed, st_mixed, clocks = timed(s_mixed, args.steps, args.warmup)
    status_mixed, last_mixed = st_mixed[-1]
    kkt_mixed = gen.kkt_relative_error(lp, dlp.x.cpu().numpy(), dlp.y.cpu().numpy())
    obj_err_mixed = abs(last_mixed["primal_objective"] - lp.optimal_objective) / abs(lp.optimal_objective)
    fp64 = None
    if not args.no_fp64:
        ms_fp64, st_fp64, _ = timed(s_fp64, max(1, args.fp64_steps), max(1, args.fp64_warmup))
        status_fp64, last_fp64 = st_fp64[-1]
        fp64 = {
            "ms_per_solve": ms_fp64, "status": status_fp64,
            "iterations": last_fp64["number_of_steps_taken"],
            "pdhg_iter_per_s": last_fp64["number_of_steps_taken"] / (last_fp64["loop_time"] or 1e-9),
            "setup_s": last_fp64["setup_time"],
            "objective_rel_error": abs(last_fp64["primal_objective"] - lp.optimal_objective)
            / abs(lp.optimal_objective),
            "speedup_mixed_vs_fp64": ms_fp64 / ms_mixed,
        }

    # Mixed precision to 1e-6, then FP64 continuation from that solution to 1e-8 relative KKT
    refine = None
    if not args.no_refine:
        s_ref = settings_handle(L, tol, 1, refine_passes=8, refine_tol=1e-8, time_limit=20.0)
        ms_ref, st_ref, _ = timed(s_ref, 1, 1)
        L.cuOptDestroySolverSettings(C.byref(s_ref))
        status_ref, last_ref = st_ref[-1]
        kkt_ref = gen.kkt_relative_error(lp, dlp.x.cpu().numpy(), dlp.y.cpu().numpy())
        refine = {"ms_per_solve": ms_ref, "status": status_ref,
                  "iterations": last_ref["number_of_steps_taken"],
                  "refinement_passes": last_ref["refinement_passes"],
                  "rel_primal": last_ref["l2_relative_primal_residual"],
                  "rel_dual": last_ref["l2_relative_dual_residual"],
                  "rel_gap": last_ref["relative_gap"], "kkt_check": kkt_ref,
                  "objective_rel_error": abs(last_ref["primal_objective"] - lp.optimal_objective)
                  / abs(lp.optimal_objective)}

    # Roofline of the dominant fused sweep (mixed precision = the headline path)
    prof = {}
    for prec, name in ((1, "mixed"), (0, "fp64")):
        a, b, ba, bb = C.c_double(), C.c_double(), C.c_double(), C.c_double()
        sh = settings_handle(L, tol, prec)
        p = dlp.ptrs()
        rc = L.cuOptProfilePDHGSweeps(lp.m, lp.n, *p, sh, C.c_void_p(sptr), args.profile_iters,
                                      C.byref(a), C.byref(b), C.byref(ba), C.byref(bb))
        L.cuOptDestroySolverSettings(C.byref(sh))
        assert rc == 0, rc
        prof[name] = {"primal_sweep_ms": a.value, "dual_sweep_ms": b.value,
                      "primal_sweep_bytes": ba.value, "dual_sweep_bytes": bb.value}
    peak, peak_kind = _peaks()
    pm = prof["mixed"]
    dom = "dual" if pm["dual_sweep_ms"] >= pm["primal_sweep_ms"] else "primal"
    achieved = pm[f"{dom}_sweep_bytes"] / (pm[f"{dom}_sweep_ms"] * 1e-3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": peak_kind,
                "kernel": f"{dom} sweep (sell_map_kernel, mixed precision)",
                "traffic": _traffic(dom, "mixed"),
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
    t0 = time.perf_counter()
    e2e_status = [solve_e2e(L, lp, pinned, s_mixed) for _ in range(args.e2e_steps)]
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks((time.perf_counter() - t0) * 1e3 / args.e2e_steps)
    h2d = (lp.m + 1) * 4 + lp.nnz * 12 + lp.n * 8 * 3 + lp.m * 8 * 2
    d2h = (2 * lp.n + lp.m) * 8

    # CPU baseline (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle as O
        threads = O.max_threads()
        s_iter, n = cpu_sample(lp, args.cpu_seconds, threads)
        iters = fp64["iterations"] if fp64 else last_mixed["number_of_steps_taken"]
        cpu = {"value": 1.0 / (s_iter * iters), "unit": "LPs/s to 1e-6 rel. KKT", "cores": threads,
               "kind": "port",
               "sample": f"oracle FP64 PDHG iterations: {n} on {threads} threads "
                         f"({s_iter * 1e3:.1f} ms each), scaled by the {iters} iterations of the FP64 solve",
               "pdhg_iter_per_s": 1.0 / s_iter}

    # 512 uneven FP64 LPs in one batched call vs the same LPs one by one (rank 0, N = 1),
    # then the same in mixed precision.
    batch = batch_mixed = None
    if rank == 0 and world == 1 and not args.no_batch:
        from cuopt_b200.profile import run_batch
        batch = run_batch(argparse.Namespace(count=512, sequential=args.batch_sequential,
                                             repeats=3, tol=1e-6, time_limit=120.0))
        batch_mixed = run_batch(argparse.Namespace(count=512, sequential=args.batch_sequential,
                                                   repeats=3, tol=1e-6, time_limit=120.0,
                                                   batch_precision="mixed"))
        # The batch as specified: the FP32-bulk batch against plain FP64 solves one by one.
        if batch.get("sequential_lps_per_s"):
            batch_mixed["speedup_vs_sequential_fp64"] = (batch_mixed["batch_lps_per_s"] /
                                                         batch["sequential_lps_per_s"])
    # 64 non-degenerate 5000 x 10000 LPs, batched forward (crossover) + KKT adjoint.
    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        from cuopt_b200.profile import run_adjoint
        adjoint = run_adjoint(argparse.Namespace(count=64, tol=1e-6, fd_instances=1,
                                                 fd_coords=args.adjoint_fd_coords,
                                                 basis_checks=2))

    value = world * 1000.0 / ms_mixed
    line = {
        "metric": METRIC, "value": value, "unit": "LPs/s to 1e-6 rel. KKT", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_mixed,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64 mixed",
        "data": "synthetic (seeded generator, optimum known by construction)",
        "config": bench_config(args, lp, world),
        "status": status_mixed, "iterations": last_mixed["number_of_steps_taken"],
        "pdhg_iter_per_s": last_mixed["number_of_steps_taken"] / (last_mixed["loop_time"] or 1e-9),
        "setup_s": last_mixed["setup_time"], "loop_s": last_mixed["loop_time"],
        "objective_rel_error": obj_err_mixed, "kkt": kkt_mixed, "fp64": fp64,
        "mixed_refined_to_1e-8": refine, "batch_c3": batch, "batch_c3_mixed": batch_mixed,
        "adjoint_c4": adjoint,
        "roofline": roofline, "cpu_baseline": cpu,
        "e2e": {"value": world * 1000.0 / e2e_ms, "unit": "LPs/s to 1e-6 rel. KKT",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "status": e2e_status},
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
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--config", choices=sorted(CONFIGS), default="c1")
    ap.add_argument("--fp64-steps", type=int, default=2)
    ap.add_argument("--fp64-warmup", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--profile-iters", type=int, default=50)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--cpu-iterations", type=int, default=0)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-refine", action="store_true")
    ap.add_argument("--no-batch", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--adjoint-fd-coords", type=int, default=16,
                    help="adjoint batch: coordinates per kind checked by central differences")
    ap.add_argument("--batch-sequential", type=int, default=32,
                    help="512-LP batch: instances also solved one by one (timing sample)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
