"""CPU tests of the Python mirror's host logic that needs no solve: PDLP warm-start data, which
the reference accepts only in Stable2 (pdlp.cu:176-181) and never in a batch
(solver_wrapper.pyx:528).  This library runs every mode as Stable3, so a solve given the data
ends as the reference's Stable3 solve does (pdlp_test.cu:880-901: NoTermination)."""
from __future__ import annotations

import numpy as np
import pytest

from cuopt_b200 import linear_programming as lpm
from tests.helpers import chess_set_lp


def _solution(error=0, by_pdlp=1):
    stats = {"number_of_steps_taken": 610, "step_size": 0.25, "primal_weight": 1.5,
             "solved_by_pdlp": by_pdlp}
    return lpm.Solution(np.array([0.0, 66.6]), np.array([6.6, 0.0]), np.array([-1.6, 0.0]),
                        1, error, "", stats)


def test_warm_start_data_carries_the_final_state():
    d = _solution().get_pdlp_warm_start_data()
    assert isinstance(d, lpm.PDLPWarmStartData)
    assert np.array_equal(d.current_primal_solution, [0.0, 66.6])
    assert np.array_equal(d.last_restart_duality_gap_dual_solution, [6.6, 0.0])
    assert (d.initial_step_size, d.initial_primal_weight, d.total_pdlp_iterations) == (0.25, 1.5, 610)
    assert _solution(error=6).get_pdlp_warm_start_data() is None
    assert _solution(by_pdlp=0).get_pdlp_warm_start_data() is None


def test_solve_with_warm_start_data_ends_without_termination():
    s = lpm.SolverSettings()
    assert s.get_pdlp_warm_start_data() is None
    s.set_pdlp_warm_start_data(_solution().get_pdlp_warm_start_data())
    sol = lpm.Solve(chess_set_lp(), s)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.NoTermination
    assert sol.get_error_status() == lpm.ErrorStatus.ValidationError
    assert "Stable2" in sol.get_error_message()
    assert not np.any(sol.get_primal_solution()) and len(sol.get_dual_solution()) == 2


def test_batch_solve_with_warm_start_data_raises():
    s = lpm.SolverSettings()
    s.set_pdlp_warm_start_data(_solution().get_pdlp_warm_start_data())
    with pytest.raises(lpm.CuOptError):
        lpm.BatchSolve([chess_set_lp(), chess_set_lp()], s)
    with pytest.raises(lpm.CuOptError):
        lpm.SolveClimbers(chess_set_lp(), [0], [0.0], [1.0], s)


@pytest.mark.parametrize("mode,name", [(0, "Stable1"), (1, "Stable2"), (2, "Methodical1"),
                                       (3, "Fast1")])
def test_unbuilt_solver_modes_are_rejected(mode, name):
    """Only Stable3 is built: a solve or a batch that asks for another mode ends with a validation
    error naming the mode (before any device work), instead of being solved as Stable3."""
    s = lpm.SolverSettings()
    s.set_parameter(lpm.CUOPT_PDLP_SOLVER_MODE, mode)
    s.set_parameter(lpm.CUOPT_LOG_TO_CONSOLE, False)
    sol = lpm.Solve(chess_set_lp(), s)
    assert sol.get_error_status() == lpm.ErrorStatus.ValidationError
    assert sol.get_termination_status() == lpm.LPTerminationStatus.NoTermination
    assert name in sol.get_error_message()
    sols, _ = lpm.BatchSolve([chess_set_lp(), chess_set_lp()], s)
    assert all(x.get_error_status() == lpm.ErrorStatus.ValidationError for x in sols)


@pytest.mark.parametrize("w", [1, 5, 12])
def test_sweep_block_shape_must_be_a_built_one(w):
    """pdlp_sweep_warps_per_block accepts 0 (timed choice), 4, 8 and 16; other values end with a
    validation error before any device work."""
    s = lpm.SolverSettings()
    s.set_parameter(lpm.CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK, w)
    s.set_parameter(lpm.CUOPT_LOG_TO_CONSOLE, False)
    sol = lpm.Solve(chess_set_lp(), s)
    assert sol.get_error_status() == lpm.ErrorStatus.ValidationError
    assert "pdlp_sweep_warps_per_block" in sol.get_error_message()
