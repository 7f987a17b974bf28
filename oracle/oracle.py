"""ctypes wrapper of the CPU oracle (oracle/liboracle_pdlp.so) — TEST INFRASTRUCTURE ONLY.

Used by tests/, __graft_entry__.smoke() and the CPU leg of bench.py to check the CUDA product path;
never by the product library.  Build with `make -C oracle`.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle_pdlp.so"


class _LP(C.Structure):
    _fields_ = [("m", C.c_int), ("n", C.c_int), ("nnz", C.c_int),
                ("row_off", C.c_void_p), ("col_idx", C.c_void_p), ("val", C.c_void_p),
                ("c", C.c_void_p), ("con_lo", C.c_void_p), ("con_up", C.c_void_p),
                ("var_lo", C.c_void_p), ("var_up", C.c_void_p),
                ("obj_offset", C.c_double), ("maximize", C.c_int),
                ("initial_primal", C.c_void_p), ("initial_dual", C.c_void_p),
                ("initial_step_size", C.c_double), ("initial_primal_weight", C.c_double)]


class _Settings(C.Structure):
    _fields_ = [("abs_primal", C.c_double), ("rel_primal", C.c_double),
                ("abs_dual", C.c_double), ("rel_dual", C.c_double),
                ("abs_gap", C.c_double), ("rel_gap", C.c_double),
                ("iteration_limit", C.c_long), ("time_limit", C.c_double), ("threads", C.c_int),
                ("detect_infeasibility", C.c_int), ("primal_infeasible_tolerance", C.c_double),
                ("dual_infeasible_tolerance", C.c_double), ("per_constraint_residual", C.c_int)]


class _Result(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int),
                ("primal_obj", C.c_double), ("dual_obj", C.c_double),
                ("l2_primal", C.c_double), ("l2_dual", C.c_double),
                ("rel_primal", C.c_double), ("rel_dual", C.c_double),
                ("gap", C.c_double), ("rel_gap", C.c_double),
                ("step_size", C.c_double), ("primal_weight", C.c_double),
                ("restarts", C.c_int), ("power_iterations", C.c_int), ("solve_time", C.c_double)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH} missing: run `make -C oracle`")
        _lib = C.CDLL(str(LIB_PATH))
        _lib.oracle_pdlp_solve.argtypes = [C.POINTER(_LP), C.POINTER(_Settings), C.POINTER(_Result),
                                           C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_pdlp_solve.restype = C.c_int
        _lib.oracle_initial_step_and_weight.argtypes = [C.POINTER(_LP), C.c_int,
                                                        C.POINTER(C.c_double), C.POINTER(C.c_double)]
        _lib.oracle_pdhg_iterations.argtypes = [C.POINTER(_LP), C.c_int, C.c_int]
        _lib.oracle_pdhg_iterations.restype = C.c_double
        _lib.oracle_max_threads.restype = C.c_int
    return _lib


class _Holder:
    """Keeps the numpy arrays alive while the C struct points at them."""

    def __init__(self, row_off, col_idx, val, c, con_lo, con_up, var_lo, var_up, obj_offset=0.0,
                 maximize=False, initial_primal=None, initial_dual=None, initial_step_size=None,
                 initial_primal_weight=None):
        self.a = [np.ascontiguousarray(row_off, np.int32), np.ascontiguousarray(col_idx, np.int32)]
        self.a += [np.ascontiguousarray(v, np.float64) for v in (val, c, con_lo, con_up, var_lo, var_up)]
        p = [x.ctypes.data for x in self.a]
        m = len(self.a[0]) - 1
        self.init = [None if v is None else np.ascontiguousarray(v, np.float64)
                     for v in (initial_primal, initial_dual)]
        self.s = _LP(m, len(self.a[3]), int(self.a[0][-1]) if m >= 0 else 0, *p,
                     float(obj_offset), int(bool(maximize)),
                     *[None if v is None else v.ctypes.data for v in self.init],
                     *[float("nan") if v is None else float(v)
                       for v in (initial_step_size, initial_primal_weight)])


def _holder(lp, initial_primal=None, initial_dual=None, initial_step_size=None,
            initial_primal_weight=None):
    return _Holder(lp.row_off, lp.col_idx, lp.val, lp.c, lp.con_lo, lp.con_up, lp.var_lo, lp.var_up,
                   getattr(lp, "obj_offset", 0.0), getattr(lp, "maximize", False),
                   initial_primal, initial_dual, initial_step_size, initial_primal_weight)


def solve(lp, tol=1e-4, iteration_limit=2**31 - 1, time_limit=1e300, threads=0,
          detect_infeasibility=False, infeasible_tol=1e-10, initial_primal=None, initial_dual=None,
          initial_step_size=None, initial_primal_weight=None, per_constraint_residual=False,
          abs_tol=None, rel_tol=None):
    """Runs the FP64 Stable3 restatement (optionally warm-started from an initial primal and / or
    dual solution in the user's order, and from a given step size and primal weight).  `tol` sets
    the six absolute and relative tolerances; `abs_tol` / `rel_tol` override the absolute or the
    relative ones.  Returns (result dict, x, y, reduced_cost)."""
    h = _holder(lp, initial_primal, initial_dual, initial_step_size, initial_primal_weight)
    m, n = h.s.m, h.s.n
    at = tol if abs_tol is None else abs_tol
    rt = tol if rel_tol is None else rel_tol
    st = _Settings(at, rt, at, rt, at, rt, int(iteration_limit), float(time_limit), int(threads),
                   int(bool(detect_infeasibility)), float(infeasible_tol), float(infeasible_tol),
                   int(bool(per_constraint_residual)))
    r = _Result()
    x, y, rc = np.zeros(n), np.zeros(m), np.zeros(n)
    lib().oracle_pdlp_solve(C.byref(h.s), C.byref(st), C.byref(r), x.ctypes.data, y.ctypes.data,
                            rc.ctypes.data)
    res = {f: getattr(r, f) for f, _ in _Result._fields_}
    return res, x, y, rc


def strong_branching(lp, fractional, root, tol=1e-4, time_limit=1e300, threads=0):
    """The reference's batch_pdlp_solve (solve.cu:743-919) restated on the oracle: the LP solved
    once (iteration limit 100000, no infeasibility detection), then every down branch
    (x_j <= floor(root)) and up branch (x_j >= ceil(root)) solved from that solution, its step size
    and its primal weight under the same limits.  Returns a list of (result, x, y, rc), down
    branches first."""
    import copy
    base, x0, y0, _ = solve(lp, tol=tol, iteration_limit=100000, time_limit=time_limit,
                            threads=threads)
    out = []
    for down in (True, False):
        for j, r in zip(fractional, root):
            q = copy.copy(lp)
            q.var_lo = np.array(lp.var_lo, dtype=np.float64)
            q.var_up = np.array(lp.var_up, dtype=np.float64)
            if down:
                q.var_up[j] = np.floor(r)
            else:
                q.var_lo[j] = np.ceil(r)
            out.append(solve(q, tol=tol, iteration_limit=100000, time_limit=time_limit,
                             threads=threads, initial_primal=x0, initial_dual=y0,
                             initial_step_size=base["step_size"],
                             initial_primal_weight=base["primal_weight"]))
    return out


def initial_step_and_weight(lp, mode: int = 4):
    """(step size, primal weight) before the first iteration; mode 4 Stable3, 2 Methodical1."""
    h = _holder(lp)
    step, w = C.c_double(), C.c_double()
    lib().oracle_initial_step_and_weight(C.byref(h.s), mode, C.byref(step), C.byref(w))
    return step.value, w.value


def pdhg_seconds(lp, iterations: int, threads: int = 0) -> float:
    """Wall time of `iterations` reflected PDHG steps on the CPU."""
    h = _holder(lp)
    return lib().oracle_pdhg_iterations(C.byref(h.s), int(iterations), int(threads))


def max_threads() -> int:
    return lib().oracle_max_threads()
