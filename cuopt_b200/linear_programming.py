"""Python mirror of the reference's `cuopt.linear_programming` LP API, on top of the C-ABI.

Counterparts (python/cuopt/cuopt/linear_programming/ in the reference):
  DataModel       data_model/data_model.py:154-683   (setters / getters of the LP arrays)
  SolverSettings  solver_settings/solver_settings.py:102-183 (set_parameter, set_optimality_tolerance)
  Solve           solver/solver.py:13-106
  BatchSolve      solver/solver.py:109-160
  Solution        solution/solution.py:55-393         (getters, get_lp_stats)
  PDLPWarmStartData  cpp/include/cuopt/linear_programming/pdlp/pdlp_warm_start_data.hpp
                  (returned; rejected by the Stable3 solve as in pdlp.cu:176-181)
Every call goes through libcuopt_b200.so; arrays are copied into the library, as in the reference.
"""
from __future__ import annotations

import ctypes as C
from enum import IntEnum

import numpy as np

from ._lib import PDLPStatistics, handle_t, lib, stats_dict

# Parameter names (reference constants.h:23-76)
CUOPT_ABSOLUTE_DUAL_TOLERANCE = "absolute_dual_tolerance"
CUOPT_RELATIVE_DUAL_TOLERANCE = "relative_dual_tolerance"
CUOPT_ABSOLUTE_PRIMAL_TOLERANCE = "absolute_primal_tolerance"
CUOPT_RELATIVE_PRIMAL_TOLERANCE = "relative_primal_tolerance"
CUOPT_ABSOLUTE_GAP_TOLERANCE = "absolute_gap_tolerance"
CUOPT_RELATIVE_GAP_TOLERANCE = "relative_gap_tolerance"
CUOPT_ITERATION_LIMIT = "iteration_limit"
CUOPT_TIME_LIMIT = "time_limit"
CUOPT_PDLP_SOLVER_MODE = "pdlp_solver_mode"
CUOPT_METHOD = "method"
CUOPT_PRESOLVE = "presolve"
CUOPT_LOG_TO_CONSOLE = "log_to_console"
CUOPT_INFEASIBILITY_DETECTION = "infeasibility_detection"
CUOPT_PER_CONSTRAINT_RESIDUAL = "per_constraint_residual"
CUOPT_CROSSOVER = "crossover"
# Additions of this library
CUOPT_PDLP_PRECISION = "pdlp_precision"
CUOPT_PDLP_REFINEMENT_PASSES = "pdlp_refinement_passes"
CUOPT_PDLP_REFINEMENT_TOLERANCE = "pdlp_refinement_tolerance"
CUOPT_PDLP_TILED_SWEEPS = "pdlp_tiled_sweeps"
CUOPT_PDLP_PERSISTENT_ITERATIONS = "pdlp_persistent_iterations"
CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK = "pdlp_sweep_warps_per_block"

_TOLERANCE_NAMES = (CUOPT_ABSOLUTE_DUAL_TOLERANCE, CUOPT_RELATIVE_DUAL_TOLERANCE,
                    CUOPT_ABSOLUTE_PRIMAL_TOLERANCE, CUOPT_RELATIVE_PRIMAL_TOLERANCE,
                    CUOPT_ABSOLUTE_GAP_TOLERANCE, CUOPT_RELATIVE_GAP_TOLERANCE)


class SolverMethod(IntEnum):
    Concurrent = 0
    PDLP = 1
    DualSimplex = 2
    Barrier = 3


class PDLPSolverMode(IntEnum):
    Stable1 = 0
    Stable2 = 1
    Methodical1 = 2
    Fast1 = 3
    Stable3 = 4


class PDLPPrecision(IntEnum):
    FP64 = 0
    Mixed = 1


class LPTerminationStatus(IntEnum):
    NoTermination = 0
    Optimal = 1
    PrimalInfeasible = 2
    DualInfeasible = 3
    IterationLimit = 4
    TimeLimit = 5
    NumericalError = 6
    PrimalFeasible = 7
    ConcurrentLimit = 9


class ErrorStatus(IntEnum):
    Success = 0
    InvalidArgument = 1
    MPSFileError = 2
    MPSParseError = 3
    ValidationError = 4
    OutOfMemoryError = 5
    RuntimeError = 6


class CuOptError(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where} returned {ErrorStatus(code).name} ({code})")
        self.code = code


def _check(code: int, where: str) -> None:
    if code != 0:
        raise CuOptError(code, where)


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class DataModel:
    """LP data: minimise/maximise c.x + offset s.t. lower <= A x <= upper (or row types + rhs),
    variable_lower <= x <= variable_upper.  A is CSR (values, column indices, row offsets)."""

    def __init__(self):
        self.maximize = False
        self.A_values = np.zeros(0)
        self.A_indices = np.zeros(0, np.int32)
        self.A_offsets = np.zeros(1, np.int32)
        self.c = np.zeros(0)
        self.objective_offset = 0.0
        self.b = None
        self.row_types = None
        self.constraint_lower_bounds = None
        self.constraint_upper_bounds = None
        self.variable_lower_bounds = None
        self.variable_upper_bounds = None
        self.variable_types = None
        self.initial_primal_solution = None
        self.initial_dual_solution = None

    # setters (reference data_model.py:154-469)
    def set_maximize(self, maximize):
        self.maximize = bool(maximize)

    def set_csr_constraint_matrix(self, A_values, A_indices, A_offsets):
        self.A_values, self.A_indices, self.A_offsets = _f64(A_values), _i32(A_indices), _i32(A_offsets)

    def set_constraint_bounds(self, b):
        self.b = _f64(b)

    def set_objective_coefficients(self, c):
        self.c = _f64(c)

    def set_objective_offset(self, objective_offset):
        self.objective_offset = float(objective_offset)

    def set_variable_lower_bounds(self, v):
        self.variable_lower_bounds = _f64(v)

    def set_variable_upper_bounds(self, v):
        self.variable_upper_bounds = _f64(v)

    def set_constraint_lower_bounds(self, v):
        self.constraint_lower_bounds = _f64(v)

    def set_constraint_upper_bounds(self, v):
        self.constraint_upper_bounds = _f64(v)

    def set_row_types(self, row_types):
        self.row_types = np.asarray(row_types, dtype="S1")

    def set_variable_types(self, variable_types):
        self.variable_types = np.asarray(variable_types, dtype="S1")

    def set_initial_primal_solution(self, v):
        self.initial_primal_solution = _f64(v)

    def set_initial_dual_solution(self, v):
        self.initial_dual_solution = _f64(v)

    # getters
    def get_sense(self):
        return self.maximize

    def get_constraint_matrix_values(self):
        return self.A_values

    def get_constraint_matrix_indices(self):
        return self.A_indices

    def get_constraint_matrix_offsets(self):
        return self.A_offsets

    def get_objective_coefficients(self):
        return self.c

    def get_objective_offset(self):
        return self.objective_offset

    def get_constraint_bounds(self):
        return self.b

    def get_constraint_lower_bounds(self):
        return self.constraint_lower_bounds

    def get_constraint_upper_bounds(self):
        return self.constraint_upper_bounds

    def get_variable_lower_bounds(self):
        return self.variable_lower_bounds

    def get_variable_upper_bounds(self):
        return self.variable_upper_bounds

    def get_row_types(self):
        return self.row_types

    @property
    def n_constraints(self) -> int:
        return len(self.A_offsets) - 1

    @property
    def n_variables(self) -> int:
        return len(self.c)

    def _create(self) -> handle_t:
        """Creates the C problem handle (cuOptCreateRangedProblem / cuOptCreateProblem)."""
        L = lib()
        m, n = self.n_constraints, self.n_variables
        vl = self.variable_lower_bounds if self.variable_lower_bounds is not None else np.zeros(n)
        vu = (self.variable_upper_bounds if self.variable_upper_bounds is not None
              else np.full(n, np.inf))
        vt = (self.variable_types.tobytes() if self.variable_types is not None
              else b"C" * max(n, 1))
        h = handle_t()
        sense = -1 if self.maximize else 1
        if self.constraint_lower_bounds is not None or self.constraint_upper_bounds is not None:
            lo = (self.constraint_lower_bounds if self.constraint_lower_bounds is not None
                  else np.full(m, -np.inf))
            up = (self.constraint_upper_bounds if self.constraint_upper_bounds is not None
                  else np.full(m, np.inf))
            keep = (vl, vu, lo, up)
            rc = L.cuOptCreateRangedProblem(m, n, sense, self.objective_offset, _ptr(self.c),
                                            _ptr(self.A_offsets), _ptr(self.A_indices),
                                            _ptr(self.A_values), _ptr(lo), _ptr(up), _ptr(vl),
                                            _ptr(vu), vt, C.byref(h))
        else:
            if self.row_types is None or self.b is None:
                raise CuOptError(4, "DataModel (constraint bounds or row types + rhs must be set)")
            keep = (vl, vu)
            rc = L.cuOptCreateProblem(m, n, sense, self.objective_offset, _ptr(self.c),
                                      _ptr(self.A_offsets), _ptr(self.A_indices),
                                      _ptr(self.A_values), self.row_types.tobytes() or b"E",
                                      _ptr(self.b), _ptr(vl), _ptr(vu), vt, C.byref(h))
        del keep
        _check(rc, "cuOptCreateProblem")
        return h


class SolverSettings:
    """Parameter bag applied to a C settings handle at solve time (reference solver_settings.py)."""

    def __init__(self):
        self.params: dict[str, object] = {}

    def set_parameter(self, name, value):
        self.params[name] = value

    def get_parameter(self, name):
        return self.params.get(name)

    def set_optimality_tolerance(self, eps_optimal):
        for n in _TOLERANCE_NAMES:
            self.params[n] = float(eps_optimal)

    def set_pdlp_warm_start_data(self, pdlp_warm_start_data):
        """PDLP solver state from a previous solve (reference solver_settings.py:183-207).  The
        reference resumes from it in Stable2 only (pdlp.cu:176-181); this library runs every mode
        as Stable3, so a solve given it ends NoTermination with a validation error, as a Stable3
        solve does in the reference.  Start from a previous solution with
        DataModel.set_initial_primal_solution / set_initial_dual_solution instead."""
        self.pdlp_warm_start_data = pdlp_warm_start_data

    def get_pdlp_warm_start_data(self):
        return getattr(self, "pdlp_warm_start_data", None)

    def _create(self) -> handle_t:
        L = lib()
        h = handle_t()
        _check(L.cuOptCreateSolverSettings(C.byref(h)), "cuOptCreateSolverSettings")
        for name, value in self.params.items():
            if isinstance(value, bool):
                rc = L.cuOptSetParameter(h, name.encode(), b"true" if value else b"false")
            elif isinstance(value, (int, np.integer)):
                rc = L.cuOptSetIntegerParameter(h, name.encode(), int(value))
            elif isinstance(value, (float, np.floating)):
                rc = L.cuOptSetFloatParameter(h, name.encode(), float(value))
            else:
                rc = L.cuOptSetParameter(h, name.encode(), str(value).encode())
            if rc != 0:
                L.cuOptDestroySolverSettings(C.byref(h))
                _check(rc, f"set parameter {name}")
        return h


class PDLPWarmStartData:
    """The PDLP state a solve ends with (reference pdlp_warm_start_data.hpp): the current
    iterates, the step size, the primal weight and the iteration counts.  The restart-state
    vectors are those iterates."""

    def __init__(self, primal, dual, step_size, primal_weight, iterations):
        self.current_primal_solution = np.asarray(primal, dtype=np.float64)
        self.current_dual_solution = np.asarray(dual, dtype=np.float64)
        self.initial_primal_average = self.current_primal_solution
        self.initial_dual_average = self.current_dual_solution
        self.last_restart_duality_gap_primal_solution = self.current_primal_solution
        self.last_restart_duality_gap_dual_solution = self.current_dual_solution
        self.initial_step_size = float(step_size)
        self.initial_primal_weight = float(primal_weight)
        self.total_pdlp_iterations = int(iterations)
        self.total_pdhg_iterations = int(iterations)


class Solution:
    """Solution of an LP (reference solution/solution.py:55-393)."""

    def __init__(self, primal, dual, reduced_cost, status, error_status, error_message, stats):
        self.primal_solution = primal
        self.dual_solution = dual
        self.reduced_cost = reduced_cost
        self.termination_status = LPTerminationStatus(status)
        self.error_status = ErrorStatus(error_status)
        self.error_message = error_message
        self.stats = stats
        self.solve_time = stats.get("solve_time", 0.0)
        self.primal_objective = stats.get("primal_objective", 0.0)
        self.dual_objective = stats.get("dual_objective", 0.0)
        self.solved_by_pdlp = bool(stats.get("solved_by_pdlp", 1))

    def get_primal_solution(self):
        return self.primal_solution

    def get_dual_solution(self):
        return self.dual_solution

    def get_reduced_cost(self):
        return self.reduced_cost

    def get_primal_objective(self):
        return self.primal_objective

    def get_dual_objective(self):
        return self.dual_objective

    def get_termination_status(self):
        return self.termination_status

    def get_termination_reason(self):
        return self.termination_status.name

    def get_error_status(self):
        return self.error_status

    def get_error_message(self):
        return self.error_message

    def get_solve_time(self):
        return self.solve_time

    def get_solved_by_pdlp(self):
        return self.solved_by_pdlp

    def get_pdlp_warm_start_data(self):
        """The solve's final PDLP state (reference solution.py:338-346); None when the LP was not
        solved by PDLP."""
        if not self.solved_by_pdlp or self.error_status != ErrorStatus.Success:
            return None
        return PDLPWarmStartData(self.primal_solution, self.dual_solution,
                                 self.stats.get("step_size", 0.0),
                                 self.stats.get("primal_weight", 0.0),
                                 self.stats.get("number_of_steps_taken", 0))

    def get_lp_stats(self):
        return {
            "primal_residual": self.stats.get("l2_primal_residual"),
            "dual_residual": self.stats.get("l2_dual_residual"),
            "gap": self.stats.get("gap"),
            "nb_iterations": self.stats.get("number_of_steps_taken"),
        }


def _read_solution(sol: handle_t, m: int, n: int) -> Solution:
    L = lib()
    status, err = C.c_int32(), C.c_int32()
    L.cuOptGetTerminationStatus(sol, C.byref(status))
    L.cuOptGetErrorStatus(sol, C.byref(err))
    buf = C.create_string_buffer(1024)
    L.cuOptGetErrorString(sol, buf, 1024)
    st = PDLPStatistics()
    L.cuOptGetPDLPStatistics(sol, C.byref(st))
    stats = stats_dict(st)
    x, y, rc = np.zeros(n), np.zeros(m), np.zeros(n)
    if err.value == 0:
        L.cuOptGetPrimalSolution(sol, _ptr(x))
        L.cuOptGetDualSolution(sol, _ptr(y))
        L.cuOptGetReducedCosts(sol, _ptr(rc))
    return Solution(x, y, rc, status.value, err.value, buf.value.decode(), stats)


def _apply_initial(settings_h: handle_t, data_model: DataModel) -> None:
    L = lib()
    if data_model.initial_primal_solution is not None:
        v = data_model.initial_primal_solution
        _check(L.cuOptSetInitialPrimalSolution(settings_h, _ptr(v), len(v)),
               "cuOptSetInitialPrimalSolution")
    if data_model.initial_dual_solution is not None:
        v = data_model.initial_dual_solution
        _check(L.cuOptSetInitialDualSolution(settings_h, _ptr(v), len(v)),
               "cuOptSetInitialDualSolution")


def _warm_start_rejected(data_model: DataModel) -> Solution:
    """The reference's answer to PDLP warm-start data outside Stable2 (pdlp.cu:179-181): a
    validation error, termination status NoTermination, zero vectors."""
    m, n = data_model.n_constraints, data_model.n_variables
    return Solution(np.zeros(n), np.zeros(m), np.zeros(n), int(LPTerminationStatus.NoTermination),
                    int(ErrorStatus.ValidationError),
                    "Only Stable2 mode supported for warm start (this library runs Stable3; start "
                    "from a solution with set_initial_primal_solution / "
                    "set_initial_dual_solution)", {"solved_by_pdlp": 0})


def Solve(data_model: DataModel, solver_settings: SolverSettings | None = None) -> Solution:
    """Solves one LP (reference solver.py:13-106)."""
    L = lib()
    settings = solver_settings or SolverSettings()
    if settings.get_pdlp_warm_start_data() is not None:
        return _warm_start_rejected(data_model)
    p = data_model._create()
    s = settings._create()
    sol = handle_t()
    try:
        _apply_initial(s, data_model)
        L.cuOptSolve(p, s, C.byref(sol))
        return _read_solution(sol, data_model.n_constraints, data_model.n_variables)
    finally:
        L.cuOptDestroySolution(C.byref(sol))
        L.cuOptDestroySolverSettings(C.byref(s))
        L.cuOptDestroyProblem(C.byref(p))


def BatchSolve(data_model_list, solver_settings: SolverSettings | None = None):
    """Solves a list of LPs in one call (reference solver.py:109-160).  Returns (solutions, time)."""
    import time

    L = lib()
    settings = solver_settings or SolverSettings()
    if settings.get_pdlp_warm_start_data() is not None:
        raise CuOptError(int(ErrorStatus.ValidationError),
                         "BatchSolve (PDLP warm-start data cannot be used with a batch)")
    probs = (handle_t * len(data_model_list))()
    sols = (handle_t * len(data_model_list))()
    for i, dm in enumerate(data_model_list):
        probs[i] = dm._create()
    s = settings._create()
    try:
        t0 = time.perf_counter()
        L.cuOptBatchSolve(probs, len(data_model_list), s, sols)
        elapsed = time.perf_counter() - t0
        out = [_read_solution(handle_t(sols[i]), dm.n_constraints, dm.n_variables)
               for i, dm in enumerate(data_model_list)]
        return out, elapsed
    finally:
        for i in range(len(data_model_list)):
            h = handle_t(sols[i])
            L.cuOptDestroySolution(C.byref(h))
            h = handle_t(probs[i])
            L.cuOptDestroyProblem(C.byref(h))
        L.cuOptDestroySolverSettings(C.byref(s))


def ReadMps(path: str) -> DataModel:
    """Reads an MPS file through cuOptReadProblem into a DataModel."""
    L = lib()
    h = handle_t()
    _check(L.cuOptReadProblem(str(path).encode(), C.byref(h)), "cuOptReadProblem")
    try:
        m, n, nnz, sense = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        off = C.c_double()
        L.cuOptGetNumConstraints(h, C.byref(m))
        L.cuOptGetNumVariables(h, C.byref(n))
        L.cuOptGetNumNonZeros(h, C.byref(nnz))
        L.cuOptGetObjectiveSense(h, C.byref(sense))
        L.cuOptGetObjectiveOffset(h, C.byref(off))
        m, n, nnz = m.value, n.value, nnz.value
        vals, idx, offs = np.zeros(nnz), np.zeros(nnz, np.int32), np.zeros(m + 1, np.int32)
        L.cuOptGetConstraintMatrix(h, _ptr(offs), _ptr(idx), _ptr(vals))
        c, lo, up, vl, vu = np.zeros(n), np.zeros(m), np.zeros(m), np.zeros(n), np.zeros(n)
        L.cuOptGetObjectiveCoefficients(h, _ptr(c))
        L.cuOptGetConstraintLowerBounds(h, _ptr(lo))
        L.cuOptGetConstraintUpperBounds(h, _ptr(up))
        L.cuOptGetVariableLowerBounds(h, _ptr(vl))
        L.cuOptGetVariableUpperBounds(h, _ptr(vu))
        dm = DataModel()
        dm.set_maximize(sense.value == -1)
        dm.set_objective_offset(off.value)
        dm.set_csr_constraint_matrix(vals, idx, offs)
        dm.set_objective_coefficients(c)
        dm.set_constraint_lower_bounds(lo)
        dm.set_constraint_upper_bounds(up)
        dm.set_variable_lower_bounds(vl)
        dm.set_variable_upper_bounds(vu)
        return dm
    finally:
        L.cuOptDestroyProblem(C.byref(h))


def _solve_climbers(call, data_model, count, arrays, solver_settings):
    import time

    L = lib()
    settings = solver_settings or SolverSettings()
    if settings.get_pdlp_warm_start_data() is not None:
        raise CuOptError(int(ErrorStatus.ValidationError),
                         "climber batch (batch mode not supported for PDLP warm-start data)")
    prob = data_model._create()
    s = settings._create()
    sols = (handle_t * count)()
    keep = [np.ascontiguousarray(a) for a in arrays]
    try:
        _apply_initial(s, data_model)
        t0 = time.perf_counter()
        call(L, prob, s, sols, [C.c_void_p(a.ctypes.data) for a in keep])
        elapsed = time.perf_counter() - t0
        out = [_read_solution(handle_t(sols[i]), data_model.n_constraints, data_model.n_variables)
               if sols[i] else None for i in range(count)]
        return out, elapsed
    finally:
        for i in range(count):
            h = handle_t(sols[i])
            if h:
                L.cuOptDestroySolution(C.byref(h))
        L.cuOptDestroyProblem(C.byref(prob))
        L.cuOptDestroySolverSettings(C.byref(s))


def SolveClimbers(data_model, variable_indices, lower_bounds, upper_bounds,
                  solver_settings: SolverSettings | None = None):
    """Solves copies of one LP that differ only in one variable's bounds each (the reference's
    new_bounds batch, solve.cu:740-882): copy i bounds variable_indices[i] by
    [lower_bounds[i], upper_bounds[i]].  An initial solution set on the data model is every copy's
    starting point.  Returns (solutions, time)."""
    idx = np.asarray(variable_indices, dtype=np.int32)
    lo = np.asarray(lower_bounds, dtype=np.float64)
    up = np.asarray(upper_bounds, dtype=np.float64)
    n = len(idx)
    return _solve_climbers(
        lambda L, p, s, sols, a: L.cuOptSolveClimbers(p, s, n, a[0], a[1], a[2], sols),
        data_model, n, [idx, lo, up], solver_settings)


def BatchPDLPStrongBranching(data_model, fractional, root_solution,
                             solver_settings: SolverSettings | None = None):
    """Strong branching (the reference's batch_pdlp_solve, solve.cu:743-919): the down branches
    (x_j <= floor(root_j)) of every fractional variable, then the up branches (x_j >= ceil(root_j)),
    all started from a solve of the LP itself (its solution, step size and primal weight; iteration
    limit 100000, no infeasibility detection).  Returns (solutions, time) with 2 * len(fractional)
    solutions."""
    frac = np.asarray(fractional, dtype=np.int32)
    root = np.asarray(root_solution, dtype=np.float64)
    n = len(frac)
    return _solve_climbers(
        lambda L, p, s, sols, a: L.cuOptBatchPDLPStrongBranching(p, s, n, a[0], a[1], sols),
        data_model, 2 * n, [frac, root], solver_settings)
