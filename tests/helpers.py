"""Shared helpers for the tests: LP <-> DataModel conversion and the oracle adapter."""
from __future__ import annotations

from types import SimpleNamespace

import numpy as np

from cuopt_b200 import linear_programming as lpm


def datamodel_from_lp(lp, maximize=False, offset=0.0) -> lpm.DataModel:
    dm = lpm.DataModel()
    dm.set_maximize(maximize)
    dm.set_objective_offset(offset)
    dm.set_csr_constraint_matrix(lp.val, lp.col_idx, lp.row_off)
    dm.set_objective_coefficients(lp.c)
    dm.set_constraint_lower_bounds(lp.con_lo)
    dm.set_constraint_upper_bounds(lp.con_up)
    dm.set_variable_lower_bounds(lp.var_lo)
    dm.set_variable_upper_bounds(lp.var_up)
    return dm


def oracle_view(dm: lpm.DataModel):
    """The arrays of a DataModel in the layout the oracle takes."""
    m, n = dm.n_constraints, dm.n_variables
    lo = dm.constraint_lower_bounds
    up = dm.constraint_upper_bounds
    if lo is None:
        rt = dm.row_types.astype(str)
        b = dm.b
        lo = np.where(rt == "L", -np.inf, b)
        up = np.where(rt == "G", np.inf, b)
    return SimpleNamespace(
        row_off=dm.A_offsets, col_idx=dm.A_indices, val=dm.A_values, c=dm.c, con_lo=lo, con_up=up,
        var_lo=dm.variable_lower_bounds if dm.variable_lower_bounds is not None else np.zeros(n),
        var_up=dm.variable_upper_bounds if dm.variable_upper_bounds is not None else np.full(n, np.inf),
        obj_offset=dm.objective_offset, maximize=dm.maximize, m=m, n=n)


def settings(tol=1e-4, iteration_limit=None, time_limit=None, precision=None, method=None,
             quiet=True) -> lpm.SolverSettings:
    s = lpm.SolverSettings()
    s.set_optimality_tolerance(tol)
    if iteration_limit is not None:
        s.set_parameter(lpm.CUOPT_ITERATION_LIMIT, int(iteration_limit))
    if time_limit is not None:
        s.set_parameter(lpm.CUOPT_TIME_LIMIT, float(time_limit))
    if precision is not None:
        s.set_parameter(lpm.CUOPT_PDLP_PRECISION, int(precision))
    s.set_parameter(lpm.CUOPT_METHOD, int(method if method is not None else lpm.SolverMethod.PDLP))
    if quiet:
        s.set_parameter(lpm.CUOPT_LOG_TO_CONSOLE, False)
    return s


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


# The objective bound the results are held to: within 1e-6 relative (to max(1, |optimum|)) of the
# optimum known by construction and of the FP64 oracle.  A solve to 1e-6 relative KKT does not
# imply it: the residuals are relative to |b| and |c| while the objective can be far smaller, so
# the oracle itself ends 6.8e-6 off on instance 284 of the 512-LP batch at 1e-6 (pinned in
# test_oracle.py).  Tests of the bound therefore solve to 1e-8 relative KKT: FP64 at 1e-8, or
# mixed precision at 1e-6 continued in FP64 to 1e-8 (refined_settings).
OBJ_RTOL = 1e-6
REFINED_TOL = 1e-8


def refined_settings(**kw) -> lpm.SolverSettings:
    """Mixed precision to 1e-6 relative KKT, then the FP64 continuation to 1e-8."""
    s = settings(tol=1e-6, precision=1, **kw)
    s.set_parameter(lpm.CUOPT_PDLP_REFINEMENT_PASSES, 1)
    s.set_parameter(lpm.CUOPT_PDLP_REFINEMENT_TOLERANCE, REFINED_TOL)
    return s


def relative_kkt(sol) -> float:
    """Largest of the three relative KKT errors a solution reports."""
    st = sol.stats
    return max(st["l2_relative_primal_residual"], st["l2_relative_dual_residual"],
               st["relative_gap"])


def oracle_results():
    """The oracle's results on the benchmark workloads (tests/golden/oracle_results.json, written
    by tests/golden/make_oracle_fixtures.py)."""
    import json
    from pathlib import Path
    return json.loads((Path(__file__).resolve().parent / "golden" / "oracle_results.json").read_text())


def small_lp(rows, c, con_lo, con_up, var_lo, var_up):
    """An LP view (as the oracle and datamodel_from_lp take it) from dense row lists
    [[(column, value), ...], ...]."""
    from types import SimpleNamespace
    off, idx, val = [0], [], []
    for r in rows:
        for j, v in r:
            idx.append(j)
            val.append(v)
        off.append(len(idx))
    return SimpleNamespace(m=len(rows), n=len(c), row_off=np.array(off, np.int32),
                           col_idx=np.array(idx, np.int32), val=np.array(val, float),
                           c=np.array(c, float), con_lo=np.array(con_lo, float),
                           con_up=np.array(con_up, float), var_lo=np.array(var_lo, float),
                           var_up=np.array(var_up, float), obj_offset=0.0, maximize=False)


def infeasible_cases(golden_dir):
    """(name, lp view) pairs: a 2-row LP with no feasible point, and afiro with the variable bounds
    of the reference's (disabled) infeasibility test (pdlp_test.cu:1289-1313: variables 1-7 in
    [7, 8], variables 13-26 in [1, 5])."""
    inf = np.inf
    tiny = small_lp([[(0, 1.0), (1, 1.0)], [(0, 1.0), (1, -1.0)]], [1.0, 1.0], [-inf, -inf],
                    [-1.0, 0.0], [0.0, 0.0], [inf, inf])
    afiro = oracle_view(lpm.ReadMps(golden_dir / "afiro_original.mps"))
    afiro.var_lo = afiro.var_lo.copy()
    afiro.var_up = afiro.var_up.copy()
    afiro.var_lo[1:8], afiro.var_up[1:8] = 7.0, 8.0
    afiro.var_lo[13:27], afiro.var_up[13:27] = 1.0, 5.0
    return [("two_rows", tiny), ("afiro_new_bounds", afiro)]


# Small LPs written out in the reference's own tests, restated as DataModels.

def reference_ranged_lp() -> lpm.DataModel:
    """max 5x + 8y  s.t.  2x + 3y <= 12,  3x + y <= 6,  2 <= x + 2y <= 8,  0 <= x, y <= 10
    (cpp/tests/linear_programming/c_api_tests/c_api_test.c:927-1041; optimum 32)."""
    dm = lpm.DataModel()
    dm.set_maximize(True)
    dm.set_csr_constraint_matrix([2.0, 3.0, 3.0, 1.0, 1.0, 2.0], [0, 1, 0, 1, 0, 1], [0, 2, 4, 6])
    dm.set_objective_coefficients([5.0, 8.0])
    dm.set_constraint_lower_bounds([-np.inf, -np.inf, 2.0])
    dm.set_constraint_upper_bounds([12.0, 6.0, 8.0])
    dm.set_variable_lower_bounds([0.0, 0.0])
    dm.set_variable_upper_bounds([10.0, 10.0])
    return dm


MAXIMIZE_DUAL_RHS = np.array([1.0, 55.0, 3.0])


def reference_maximize_dual_lp() -> lpm.DataModel:
    """max 4x1 + x2 + 5x3 + 3x4  s.t.  x1 - x2 - x3 + 3x4 <= 1,  5x1 + x2 + 3x3 + 8x4 <= 55,
    -x1 + 2x2 + 3x3 - 5x4 <= 3,  x >= 0 (c_api_test.c:1461-1614: the objective equals the dual
    objective sum_i y_i rhs_i)."""
    dm = lpm.DataModel()
    dm.set_maximize(True)
    dm.set_csr_constraint_matrix([1.0, -1.0, -1.0, 3.0, 5.0, 1.0, 3.0, 8.0, -1.0, 2.0, 3.0, -5.0],
                                 [0, 1, 2, 3] * 3, [0, 4, 8, 12])
    dm.set_objective_coefficients([4.0, 1.0, 5.0, 3.0])
    dm.set_constraint_bounds(MAXIMIZE_DUAL_RHS)
    dm.set_row_types(["L", "L", "L"])
    dm.set_variable_lower_bounds([0.0] * 4)
    dm.set_variable_upper_bounds([np.inf] * 4)
    return dm


def chess_set_lp() -> lpm.DataModel:
    """max 5xs + 20xl  s.t.  xs + 3xl <= 200,  3xs + 2xl <= 160,  x >= 0
    (cpp/tests/dual_simplex/unit_tests/solve.cpp:23-94; optimum 1333.33 at (0, 66.6667))."""
    dm = lpm.DataModel()
    dm.set_maximize(True)
    dm.set_csr_constraint_matrix([1.0, 3.0, 3.0, 2.0], [0, 1, 0, 1], [0, 2, 4])
    dm.set_objective_coefficients([5.0, 20.0])
    dm.set_constraint_bounds([200.0, 160.0])
    dm.set_row_types(["L", "L"])
    return dm


def trivial_two_row_lp() -> lpm.DataModel:
    """min x  s.t.  x <= 1 (twice),  x >= 0: the LP of the reference's Python solver test
    (python/cuopt/cuopt/tests/linear_programming/test_lp_solver.py:46-79), which expects Optimal with
    x = 0, zero residuals, zero objectives and zero gap at tolerance 1e-2."""
    dm = lpm.DataModel()
    dm.set_csr_constraint_matrix([1.0, 1.0], [0, 0], [0, 1, 2])
    dm.set_constraint_bounds([1.0, 1.0])
    dm.set_objective_coefficients([1.0])
    dm.set_row_types(["L", "L"])
    return dm


def with_variable_bounds(view, j, lo, up):
    """A copy of an oracle view whose variable j has the bounds [lo, up] (a climber's LP)."""
    import copy
    q = copy.copy(view)
    q.var_lo = np.array(view.var_lo, dtype=np.float64)
    q.var_up = np.array(view.var_up, dtype=np.float64)
    q.var_lo[j], q.var_up[j] = lo, up
    return q


def highs_objective(view):
    """Optimal objective of an oracle view by SciPy HiGHS (a third-party cross-check)."""
    from scipy.optimize import linprog
    from scipy.sparse import csr_matrix

    A = csr_matrix((view.val, view.col_idx, view.row_off), shape=(view.m, view.n))
    lo, up = np.asarray(view.con_lo), np.asarray(view.con_up)
    eq = lo == up
    ub_rows = np.isfinite(up) & ~eq
    lb_rows = np.isfinite(lo) & ~eq
    from scipy.sparse import vstack
    A_ub = vstack([A[ub_rows], -A[lb_rows]])
    b_ub = np.concatenate([up[ub_rows], -lo[lb_rows]])
    bounds = [(l, None if np.isinf(u) else u) for l, u in zip(view.var_lo, view.var_up)]
    sign = -1.0 if view.maximize else 1.0
    r = linprog(sign * np.asarray(view.c), A_ub=A_ub, b_ub=b_ub, A_eq=A[eq], b_eq=lo[eq],
                bounds=bounds, method="highs")
    assert r.status == 0, r.message
    return sign * r.fun + view.obj_offset
