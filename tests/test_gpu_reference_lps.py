"""GPU tests on the small LPs written out in the reference's own tests: the ranged C API problem
(c_api_tests.cpp:105-112), the maximisation whose objective must equal its dual objective
(c_api_tests.cpp:149-165), the chess-set LP (dual_simplex/unit_tests/solve.cpp:23-94) and the
trivial two-row LP of the Python solver test (test_lp_solver.py:46-79).

Each is solved through the C-ABI and checked against the golden values of those tests (with their
tolerances) and against the oracle: same status and iteration count, objective within 1e-9
relative (FP64 path; summation order differs).
"""
from __future__ import annotations

import pytest

from cuopt_b200 import linear_programming as lpm
from oracle import oracle as O
from tests.helpers import (MAXIMIZE_DUAL_RHS, chess_set_lp, oracle_view, reference_maximize_dual_lp,
                           reference_ranged_lp, rel, settings, trivial_two_row_lp)

pytestmark = pytest.mark.gpu


def _solve_both(dm, tol, method=None):
    sol = lpm.Solve(dm, settings(tol=tol, method=method))
    res, x, y, _ = O.solve(oracle_view(dm), tol=tol)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert res["status"] == 1
    assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
    assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-9
    return sol


@pytest.mark.parametrize("tol", [1e-4, 1e-8])
def test_reference_ranged_problem(golden, tol):
    g = golden["ranged_problem_objective"]
    sol = _solve_both(reference_ranged_lp(), tol)
    assert abs(sol.get_primal_objective() - g["value"]) <= g["abs_tol"]


@pytest.mark.parametrize("method", [lpm.SolverMethod.Concurrent, lpm.SolverMethod.PDLP])
def test_reference_maximize_dual_variables(golden, method):
    g = golden["maximize_dual_objective_match"]
    sol = _solve_both(reference_maximize_dual_lp(), 1e-4, method)
    dual_objective = sol.get_dual_solution() @ MAXIMIZE_DUAL_RHS
    assert abs(sol.get_primal_objective() - dual_objective) <= g["abs_tol"]


def test_chess_set(golden):
    g = golden["chess_set_dual_simplex"]
    sol = _solve_both(chess_set_lp(), 1e-8)
    x = sol.get_primal_solution()
    assert abs(sol.get_primal_objective() - g["objective"]) <= 1e-2
    assert abs(x[0] - g["x"][0]) <= 1e-6 and abs(x[1] - g["x"][1]) <= 1e-3


def test_trivial_two_row_lp():
    """The reference runs this LP in Stable2 with a note that its Stable3 does not terminate on it;
    Stable3 here (and in the oracle) ends Optimal, with the values that test asserts: x = 0, zero
    residuals, objectives and gap, solved by PDLP."""
    sol = _solve_both(trivial_two_row_lp(), 1e-2)
    st = sol.get_lp_stats()
    assert sol.get_termination_reason() == "Optimal"
    assert sol.get_primal_solution()[0] == pytest.approx(0.0)
    assert st["primal_residual"] == pytest.approx(0.0)
    assert st["dual_residual"] == pytest.approx(0.0)
    assert sol.get_primal_objective() == pytest.approx(0.0)
    assert sol.get_dual_objective() == pytest.approx(0.0)
    assert st["gap"] == pytest.approx(0.0)
    assert sol.get_solved_by_pdlp()


def test_afiro_climbers_with_different_bounds_like_the_reference(golden, golden_dir):
    """pdlp_test.cu:1194-1287 (more_complex_batch_different_bounds): five afiro climbers, #1 with
    variable 5 in [4, 5] and #3 with variable 1 in [-7, 13], the others unchanged.  All are
    Optimal; #0, #2 and #4 have the same objective, at afiro's; #1 and #3 stop where the oracle's
    solves of their LPs stop, at the same objective (1e-8 relative)."""
    import numpy as np

    from tests.helpers import with_variable_bounds

    dm = lpm.ReadMps(golden_dir / "afiro_original.mps")
    v = oracle_view(dm)
    var = np.array([0, 5, 0, 1, 0], np.int32)
    lo = np.array([v.var_lo[0], 4.0, v.var_lo[0], -7.0, v.var_lo[0]])
    up = np.array([v.var_up[0], 5.0, v.var_up[0], 13.0, v.var_up[0]])
    sols, _ = lpm.SolveClimbers(dm, var, lo, up, settings(tol=1e-4))
    for sol in sols:
        assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    g = golden["afiro_objective"]
    assert rel(sols[0].get_primal_objective(), g["value"]) <= g["rel_tol"]
    assert sols[0].get_primal_objective() == sols[2].get_primal_objective() == \
        sols[4].get_primal_objective()
    for b in (1, 3):
        res, _, _, _ = O.solve(with_variable_bounds(v, var[b], lo[b], up[b]), tol=1e-4)
        assert res["status"] == 1
        assert sols[b].get_lp_stats()["nb_iterations"] == res["iterations"]
        assert rel(sols[b].get_primal_objective(), res["primal_obj"]) <= 1e-8


def _variant_bounds(view, g):
    import numpy as np
    j = g["variable"]
    lo = np.array([view.var_lo[j] if v is None else v for v in g["lower"]])
    up = np.array([view.var_up[j] if v is None else g["upper"] for v in g["lower"]])
    return np.full(len(lo), j, np.int32), lo, up


def test_many_different_bounds_climbers(golden, golden_dir):
    """pdlp_test.cu:1720-1804: 13 climbers of good-mps-some-var-bounds (two groups of eight, from
    210 to about 16 000 iterations) each end as the oracle's solve of its LP does: same status,
    iteration count within 5 %, the optimum (HiGHS) within 1e-3 relative, constraint violations
    under 1e-8."""
    import numpy as np
    from scipy.sparse import csr_matrix

    from tests.helpers import highs_objective, with_variable_bounds

    g = golden["many_different_bounds"]
    dm = lpm.ReadMps(golden_dir / "good-mps-some-var-bounds.mps")
    v = oracle_view(dm)
    var, lo, up = _variant_bounds(v, g)
    sols, _ = lpm.SolveClimbers(dm, var, lo, up, settings(tol=1e-4))
    A = csr_matrix((v.val, v.col_idx, v.row_off), shape=(v.m, v.n))
    for b, sol in enumerate(sols):
        q = with_variable_bounds(v, var[b], lo[b], up[b])
        res, _, _, _ = O.solve(q, tol=1e-4)
        assert int(sol.get_termination_status()) == res["status"] == 1
        it = sol.get_lp_stats()["nb_iterations"]
        assert abs(it - res["iterations"]) <= 0.05 * res["iterations"] + 10
        assert rel(sol.get_primal_objective(), highs_objective(q)) <= 1e-3
        x = sol.get_primal_solution()
        ax = A @ x
        viol = max(np.max(np.maximum(0.0, ax - q.con_up)), np.max(np.maximum(0.0, q.con_lo - ax)),
                   np.max(np.maximum(0.0, q.var_lo - x)), np.max(np.maximum(0.0, x - q.var_up)))
        assert viol <= g["constraint_tol"]


def test_some_climber_hits_the_iteration_limit(golden, golden_dir):
    """pdlp_test.cu:1806-1885: at 500 iterations one climber hits the limit and the other is
    Optimal, with the oracle's iteration count and objective (1e-8 relative)."""
    from tests.helpers import with_variable_bounds

    g = golden["some_climber_hit_iteration_limit"]
    dm = lpm.ReadMps(golden_dir / "good-mps-some-var-bounds.mps")
    v = oracle_view(dm)
    var, lo, up = _variant_bounds(v, g)
    sols, _ = lpm.SolveClimbers(dm, var, lo, up,
                                settings(tol=1e-4, iteration_limit=g["iteration_limit"]))
    for b, (sol, status) in enumerate(zip(sols, g["statuses"])):
        assert sol.get_termination_status() == lpm.LPTerminationStatus[status]
        if status == "Optimal":
            res, _, _, _ = O.solve(with_variable_bounds(v, var[b], lo[b], up[b]), tol=1e-4,
                                   iteration_limit=g["iteration_limit"])
            assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
            assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-8


def _afiro(golden_dir):
    return lpm.ReadMps(golden_dir / "afiro_original.mps")


def test_afiro_at_the_minimal_absolute_tolerance(golden, golden_dir):
    """pdlp_test.cu:76-100: absolute tolerances 1e-12, relative 0: Optimal at afiro's objective
    (1 %)."""
    s = settings(tol=1e-4)
    for name in ("absolute_primal_tolerance", "absolute_dual_tolerance", "absolute_gap_tolerance"):
        s.set_parameter(name, 1e-12)
    for name in ("relative_primal_tolerance", "relative_dual_tolerance", "relative_gap_tolerance"):
        s.set_parameter(name, 0.0)
    s.set_parameter(lpm.CUOPT_TIME_LIMIT, 120.0)
    sol = lpm.Solve(_afiro(golden_dir), s)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert rel(sol.get_primal_objective(), golden["afiro_objective"]["value"]) <= 0.01


def test_afiro_from_an_all_ones_primal(golden, golden_dir):
    """pdlp_test.cu:102-122: started from x = 1: Optimal at afiro's objective (1 %), where the
    oracle's warm-started solve stops."""
    import numpy as np

    dm = _afiro(golden_dir)
    dm.set_initial_primal_solution(np.ones(dm.n_variables))
    sol = lpm.Solve(dm, settings(tol=1e-4))
    res, _, _, _ = O.solve(oracle_view(dm), initial_primal=np.ones(dm.n_variables))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert rel(sol.get_primal_objective(), golden["afiro_objective"]["value"]) <= 0.01
    assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]


def test_afiro_iteration_limit_returns_the_current_iterate(golden_dir):
    """pdlp_test.cu:124-147: 10 iterations at tolerance 0 end IterationLimit with the current primal
    iterate, the oracle's to 1e-9."""
    import numpy as np

    dm = _afiro(golden_dir)
    sol = lpm.Solve(dm, settings(tol=0.0, iteration_limit=10))
    res, x, _, _ = O.solve(oracle_view(dm), tol=0.0, iteration_limit=10)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.IterationLimit
    got = sol.get_primal_solution()
    assert np.any(got != 0.0)
    assert np.max(np.abs(got - x)) <= 1e-9 * (1 + np.abs(x).max())
