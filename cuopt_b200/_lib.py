"""ctypes binding of libcuopt_b200.so — the C-ABI declared in include/cuopt/linear_programming/cuopt_c.h
and include/cuopt_b200.h.

The library is loaded from the package directory.  If it is missing the import fails loudly: there
is no Python or CPU fallback for the solver.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libcuopt_b200.so"

cuopt_int_t = C.c_int32
cuopt_float_t = C.c_double
handle_t = C.c_void_p
_P_int = C.POINTER(cuopt_int_t)
_P_float = C.POINTER(cuopt_float_t)


class PDLPStatistics(C.Structure):
    """Mirror of cuOptPDLPStatistics (include/cuopt_b200.h)."""

    _fields_ = [
        ("number_of_steps_taken", cuopt_int_t),
        ("total_number_of_attempted_steps", cuopt_int_t),
        ("l2_primal_residual", cuopt_float_t),
        ("l2_relative_primal_residual", cuopt_float_t),
        ("l2_dual_residual", cuopt_float_t),
        ("l2_relative_dual_residual", cuopt_float_t),
        ("primal_objective", cuopt_float_t),
        ("dual_objective", cuopt_float_t),
        ("gap", cuopt_float_t),
        ("relative_gap", cuopt_float_t),
        ("solve_time", cuopt_float_t),
        ("solved_by_pdlp", cuopt_int_t),
        ("restarts", cuopt_int_t),
        ("power_iterations", cuopt_int_t),
        ("refinement_passes", cuopt_int_t),
        ("step_size", cuopt_float_t),
        ("primal_weight", cuopt_float_t),
        ("setup_time", cuopt_float_t),
        ("loop_time", cuopt_float_t),
        ("kernel_launches", cuopt_float_t),
        ("crossover", cuopt_int_t),
        ("plain_iteration_form", cuopt_int_t),
        ("persistent_blocks", cuopt_int_t),
        ("plain_iteration_us_graphs", cuopt_float_t),
        ("plain_iteration_us_persistent", cuopt_float_t),
        ("plain_iteration_us_cluster", cuopt_float_t),
        ("sweep_warps_per_block_primal", cuopt_int_t),
        ("sweep_warps_per_block_dual", cuopt_int_t),
        ("sweep_block_shape_ms", cuopt_float_t * 6),
    ]


def stats_dict(st) -> dict:
    """A PDLPStatistics as a dict of Python numbers (array fields as lists)."""
    out = {}
    for f, _ in PDLPStatistics._fields_:
        v = getattr(st, f)
        out[f] = list(v) if isinstance(v, C.Array) else v
    return out


# name -> (restype, argtypes)
SIGNATURES = {
    "cuOptGetFloatSize": (C.c_int8, []),
    "cuOptGetIntSize": (C.c_int8, []),
    "cuOptGetVersion": (cuopt_int_t, [_P_int, _P_int, _P_int]),
    "cuOptReadProblem": (cuopt_int_t, [C.c_char_p, C.POINTER(handle_t)]),
    "cuOptWriteProblem": (cuopt_int_t, [handle_t, C.c_char_p, cuopt_int_t]),
    "cuOptCreateProblem": (cuopt_int_t, [cuopt_int_t, cuopt_int_t, cuopt_int_t, cuopt_float_t,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p,
                                         C.POINTER(handle_t)]),
    "cuOptCreateRangedProblem": (cuopt_int_t, [cuopt_int_t, cuopt_int_t, cuopt_int_t, cuopt_float_t,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                               C.c_char_p, C.POINTER(handle_t)]),
    "cuOptCreateQuadraticProblem": (cuopt_int_t, [cuopt_int_t, cuopt_int_t, cuopt_int_t,
                                                  cuopt_float_t] + [C.c_void_p] * 7 +
                                    [C.c_char_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.POINTER(handle_t)]),
    "cuOptCreateQuadraticRangedProblem": (cuopt_int_t, [cuopt_int_t, cuopt_int_t, cuopt_int_t,
                                                        cuopt_float_t] + [C.c_void_p] * 11 +
                                          [C.POINTER(handle_t)]),
    "cuOptDestroyProblem": (None, [C.POINTER(handle_t)]),
    "cuOptGetNumConstraints": (cuopt_int_t, [handle_t, _P_int]),
    "cuOptGetNumVariables": (cuopt_int_t, [handle_t, _P_int]),
    "cuOptGetObjectiveSense": (cuopt_int_t, [handle_t, _P_int]),
    "cuOptGetObjectiveOffset": (cuopt_int_t, [handle_t, _P_float]),
    "cuOptGetObjectiveCoefficients": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetNumNonZeros": (cuopt_int_t, [handle_t, _P_int]),
    "cuOptGetConstraintMatrix": (cuopt_int_t, [handle_t, C.c_void_p, C.c_void_p, C.c_void_p]),
    "cuOptGetConstraintSense": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetConstraintRightHandSide": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetConstraintLowerBounds": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetConstraintUpperBounds": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetVariableLowerBounds": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetVariableUpperBounds": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetVariableTypes": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptCreateSolverSettings": (cuopt_int_t, [C.POINTER(handle_t)]),
    "cuOptDestroySolverSettings": (None, [C.POINTER(handle_t)]),
    "cuOptSetParameter": (cuopt_int_t, [handle_t, C.c_char_p, C.c_char_p]),
    "cuOptGetParameter": (cuopt_int_t, [handle_t, C.c_char_p, cuopt_int_t, C.c_char_p]),
    "cuOptSetIntegerParameter": (cuopt_int_t, [handle_t, C.c_char_p, cuopt_int_t]),
    "cuOptGetIntegerParameter": (cuopt_int_t, [handle_t, C.c_char_p, _P_int]),
    "cuOptSetFloatParameter": (cuopt_int_t, [handle_t, C.c_char_p, cuopt_float_t]),
    "cuOptGetFloatParameter": (cuopt_int_t, [handle_t, C.c_char_p, _P_float]),
    "cuOptSetMIPGetSolutionCallback": (cuopt_int_t, [handle_t, C.c_void_p, C.c_void_p]),
    "cuOptSetMIPSetSolutionCallback": (cuopt_int_t, [handle_t, C.c_void_p, C.c_void_p]),
    "cuOptSetInitialPrimalSolution": (cuopt_int_t, [handle_t, C.c_void_p, cuopt_int_t]),
    "cuOptSetInitialDualSolution": (cuopt_int_t, [handle_t, C.c_void_p, cuopt_int_t]),
    "cuOptAddMIPStart": (cuopt_int_t, [handle_t, C.c_void_p, cuopt_int_t]),
    "cuOptIsMIP": (cuopt_int_t, [handle_t, _P_int]),
    "cuOptSolve": (cuopt_int_t, [handle_t, handle_t, C.POINTER(handle_t)]),
    "cuOptDestroySolution": (None, [C.POINTER(handle_t)]),
    "cuOptGetTerminationStatus": (cuopt_int_t, [handle_t, _P_int]),
    "cuOptGetErrorStatus": (cuopt_int_t, [handle_t, _P_int]),
    "cuOptGetErrorString": (cuopt_int_t, [handle_t, C.c_char_p, cuopt_int_t]),
    "cuOptGetPrimalSolution": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetObjectiveValue": (cuopt_int_t, [handle_t, _P_float]),
    "cuOptGetSolveTime": (cuopt_int_t, [handle_t, _P_float]),
    "cuOptGetMIPGap": (cuopt_int_t, [handle_t, _P_float]),
    "cuOptGetSolutionBound": (cuopt_int_t, [handle_t, _P_float]),
    "cuOptGetDualSolution": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetDualObjectiveValue": (cuopt_int_t, [handle_t, _P_float]),
    "cuOptGetReducedCosts": (cuopt_int_t, [handle_t, C.c_void_p]),
    "cuOptGetPDLPStatistics": (cuopt_int_t, [handle_t, C.POINTER(PDLPStatistics)]),
    "cuOptSolveDevice": (cuopt_int_t, [cuopt_int_t, cuopt_int_t, cuopt_int_t, cuopt_float_t] +
                         [C.c_void_p] * 8 + [handle_t, C.c_void_p] + [C.c_void_p] * 3 +
                         [C.POINTER(PDLPStatistics), C.POINTER(cuopt_int_t)]),
    "cuOptProfilePDHGSweeps": (cuopt_int_t, [cuopt_int_t, cuopt_int_t] + [C.c_void_p] * 8 +
                               [handle_t, C.c_void_p, cuopt_int_t] +
                               [C.POINTER(C.c_double)] * 4),
    "cuOptProfileSweepClasses": (cuopt_int_t, [cuopt_int_t, cuopt_int_t] + [C.c_void_p] * 8 +
                                 [handle_t, C.c_void_p, cuopt_int_t, C.POINTER(C.c_double)]),
    "cuOptProfileGatherRate": (cuopt_int_t, [cuopt_int_t, C.c_int64, cuopt_int_t, C.c_void_p,
                                             C.POINTER(C.c_double), C.POINTER(cuopt_int_t)]),
    "cuOptProfileScatterRate": (cuopt_int_t, [cuopt_int_t, C.c_int64, cuopt_int_t, C.c_void_p,
                                              C.POINTER(C.c_double), C.POINTER(cuopt_int_t)]),
    "cuOptProbeClusterBarrier": (cuopt_int_t, [cuopt_int_t, cuopt_int_t, cuopt_int_t, C.c_void_p,
                                               C.POINTER(C.c_double)]),
    "cuOptProbeGridBarrier": (cuopt_int_t, [cuopt_int_t, cuopt_int_t, cuopt_int_t, C.c_double,
                                            C.c_void_p, C.POINTER(cuopt_int_t),
                                            C.POINTER(C.c_double)]),
    "cuOptBatchSolve": (cuopt_int_t, [C.POINTER(handle_t), cuopt_int_t, handle_t,
                                      C.POINTER(handle_t)]),
    "cuOptSolutionAdjoint": (cuopt_int_t, [handle_t, handle_t] + [C.c_void_p] * 6),
    "cuOptSolutionAdjointBatch": (cuopt_int_t, [cuopt_int_t] + [C.c_void_p] * 8),
    "cuOptSolveClimbers": (cuopt_int_t, [handle_t, handle_t, cuopt_int_t] + [C.c_void_p] * 3 +
                           [C.POINTER(handle_t)]),
    "cuOptBatchPDLPStrongBranching": (cuopt_int_t, [handle_t, handle_t, cuopt_int_t] +
                                      [C.c_void_p] * 2 + [C.POINTER(handle_t)]),
    "cuOptComputeKKTErrorsNoAlloc": (cuopt_int_t, [cuopt_int_t, cuopt_int_t, cuopt_int_t,
                                                   cuopt_float_t] + [C.c_void_p] * 11),
}

_lib = None


def lib() -> C.CDLL:
    """Loads libcuopt_b200.so once and attaches the signatures above."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(
                f"{LIB_PATH} is missing: build it with `python -m cuopt_b200.build` "
                "(no CPU fallback exists for the PDLP solver)")
        handle = C.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib
