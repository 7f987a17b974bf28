"""GPU tests of the climber batch (cuOptSolveClimbers / cuOptBatchPDLPStrongBranching): copies of
one LP that differ in one variable's bounds each, swept together through one matrix read.

Reference for every expectation: the CPU oracle solving each modified LP alone (for strong
branching, its restatement of batch_pdlp_solve: a solve of the LP, then warm-started branches), and
the reference's own batch test (pdlp_test.cu:1450-1535: identical climbers on afiro give bitwise
identical results, all Optimal at afiro's objective).  Tolerances: iterates after the same number
of iterations agree with the oracle to 1e-9 relative to the vector's magnitude; solutions at the
1e-6 termination of a strong-branching batch to 1e-7.
"""
from __future__ import annotations

import numpy as np
import pytest

from cuopt_b200 import generators as gen
from cuopt_b200 import linear_programming as lpm
from oracle import oracle as O
from tests.helpers import datamodel_from_lp, oracle_view, rel, settings

pytestmark = pytest.mark.gpu

ITERATE_RTOL = 1e-9


def _climbers(lp, count, seed):
    rng = np.random.default_rng(seed)
    var = rng.choice(lp.n, count, replace=False)
    lo = lp.var_lo[var].copy()
    up = np.minimum(lp.var_up[var], rng.uniform(0.5, 3.0, count))  # tighter upper bounds
    return var, lo, up


def _modified(lp, j, lo, up):
    import copy
    q = copy.copy(lp)
    q.var_lo, q.var_up = np.array(lp.var_lo, dtype=np.float64), np.array(lp.var_up, dtype=np.float64)
    q.var_lo[j], q.var_up[j] = lo, up
    return q


@pytest.fixture(scope="module")
def base_lp():
    return gen.constructed_lp(200, 500, 8, seed=11)


@pytest.mark.parametrize("k", [10, 200, 600])
def test_climber_iterates_match_single_oracle(base_lp, k):
    """11 climbers (two groups of eight, one partly filled) follow the oracle's solves of their
    modified LPs."""
    var, lo, up = _climbers(base_lp, 11, seed=3)
    sols, _ = lpm.SolveClimbers(datamodel_from_lp(base_lp), var, lo, up,
                                settings(tol=1e-12, iteration_limit=k))
    for b, sol in enumerate(sols):
        res, x, y, rc = O.solve(_modified(base_lp, var[b], lo[b], up[b]), tol=1e-12,
                                iteration_limit=k)
        assert sol.get_termination_status() == lpm.LPTerminationStatus.IterationLimit
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        assert np.max(np.abs(sol.get_primal_solution() - x)) <= ITERATE_RTOL * (1 + np.abs(x).max())
        assert np.max(np.abs(sol.get_dual_solution() - y)) <= ITERATE_RTOL * (1 + np.abs(y).max())
        assert np.max(np.abs(sol.get_reduced_cost() - rc)) <= ITERATE_RTOL * (1 + np.abs(rc).max())


def test_climbers_solve_to_tolerance_like_single_solves(base_lp):
    """12 climbers in two groups of eight whose upper bounds cut into the optimum: the second
    group is done at 610 iterations while two climbers of the first need 620 and 640, so the
    sweeps drop a group mid-solve.  Each climber stops where the oracle's solve of its LP stops."""
    rng = np.random.default_rng(5)
    var = rng.choice(np.where(base_lp.x_star > 2.0)[0], 12, replace=False)
    lo = base_lp.var_lo[var].copy()
    up = base_lp.x_star[var] * rng.uniform(0.05, 0.6, 12)
    sols, _ = lpm.SolveClimbers(datamodel_from_lp(base_lp), var, lo, up, settings(tol=1e-6))
    for b, sol in enumerate(sols):
        res, _, _, _ = O.solve(_modified(base_lp, var[b], lo[b], up[b]), tol=1e-6)
        assert int(sol.get_termination_status()) == res["status"] == 1
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-8


def test_identical_afiro_climbers_are_bitwise_identical(golden, golden_dir):
    """pdlp_test.cu:1450-1535 (big_batch_afiro, here 24 climbers): every climber keeps variable 0's
    own bounds; all are Optimal at afiro's objective with bitwise identical results."""
    dm = lpm.ReadMps(golden_dir / "afiro_original.mps")
    v = oracle_view(dm)
    count = 24
    sols, _ = lpm.SolveClimbers(dm, np.zeros(count, np.int32), np.full(count, v.var_lo[0]),
                                np.full(count, v.var_up[0]), settings(tol=1e-4))
    g = golden["afiro_objective"]
    ref = sols[0]
    assert ref.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert rel(ref.get_primal_objective(), g["value"]) <= g["rel_tol"]
    for sol in sols[1:]:
        assert sol.get_termination_status() == ref.get_termination_status()
        assert sol.get_primal_objective() == ref.get_primal_objective()
        assert sol.get_dual_objective() == ref.get_dual_objective()
        assert sol.get_lp_stats()["nb_iterations"] == ref.get_lp_stats()["nb_iterations"]
        assert np.array_equal(sol.get_primal_solution(), ref.get_primal_solution())
        assert np.array_equal(sol.get_dual_solution(), ref.get_dual_solution())
    single = lpm.Solve(dm, settings(tol=1e-4))
    assert single.get_lp_stats()["nb_iterations"] == ref.get_lp_stats()["nb_iterations"]


def test_strong_branching_builds_down_then_up_branches(base_lp):
    """batch_pdlp_solve / run_batch_pdlp (solve.cu:743-919): the LP is solved first, then
    x_j <= floor(root_j) for every fractional j and x_j >= ceil(root_j), each started from that
    solution, its step size and primal weight; each matches the oracle's restatement."""
    rng = np.random.default_rng(5)
    frac = rng.choice(base_lp.n, 3, replace=False)
    root = base_lp.x_star[frac] + 0.5
    sols, _ = lpm.BatchPDLPStrongBranching(datamodel_from_lp(base_lp), frac, root,
                                           settings(tol=1e-6))
    ref = O.strong_branching(base_lp, frac, root, tol=1e-6)
    assert len(sols) == len(ref) == 6
    for i, (sol, (res, x, y, _)) in enumerate(zip(sols, ref)):
        j = frac[i % 3]
        xj = sol.get_primal_solution()[j]
        assert int(sol.get_termination_status()) == res["status"] == 1
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        assert sol.stats["power_iterations"] == 0
        assert np.max(np.abs(sol.get_primal_solution() - x)) <= 1e-7 * (1 + np.abs(x).max())
        assert np.max(np.abs(sol.get_dual_solution() - y)) <= 1e-7 * (1 + np.abs(y).max())
        if i < 3:
            assert xj <= np.floor(root[i]) + 1e-6
        else:
            assert xj >= np.ceil(root[i - 3]) - 1e-6


@pytest.mark.parametrize("k", [10, 400])
def test_climbers_start_from_the_initial_solution(base_lp, k):
    """An initial solution on the data model starts every climber (as new_bounds with an initial
    solution does in the reference's batch): iterates follow the oracle's warm-started solves."""
    rng = np.random.default_rng(8)
    x0 = base_lp.x_star + 0.05 * rng.standard_normal(base_lp.n)
    y0 = base_lp.y_star + 0.05 * rng.standard_normal(base_lp.m)
    var, lo, up = _climbers(base_lp, 9, seed=6)
    dm = datamodel_from_lp(base_lp)
    dm.set_initial_primal_solution(x0)
    dm.set_initial_dual_solution(y0)
    sols, _ = lpm.SolveClimbers(dm, var, lo, up, settings(tol=1e-12, iteration_limit=k))
    for b, sol in enumerate(sols):
        res, x, y, _ = O.solve(_modified(base_lp, var[b], lo[b], up[b]), tol=1e-12,
                               iteration_limit=k, initial_primal=x0, initial_dual=y0)
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        assert np.max(np.abs(sol.get_primal_solution() - x)) <= ITERATE_RTOL * (1 + np.abs(x).max())
        assert np.max(np.abs(sol.get_dual_solution() - y)) <= ITERATE_RTOL * (1 + np.abs(y).max())


def test_crossing_climber_is_infeasible(base_lp):
    sols, _ = lpm.SolveClimbers(datamodel_from_lp(base_lp), [0, 1], [5.0, base_lp.var_lo[1]],
                                [1.0, base_lp.var_up[1]], settings(tol=1e-6))
    assert sols[0].get_termination_status() == lpm.LPTerminationStatus.PrimalInfeasible
    assert sols[1].get_termination_status() == lpm.LPTerminationStatus.Optimal


def test_afiro_strong_branching_like_the_reference(golden_dir):
    """pdlp_test.cu:1615-1720 (strong_branching_test): afiro, fractional {1, 2, 4} at
    {0.891, 0.109, 0.636429}.  Every branch has the status of the single solve of its LP and an
    objective within 1e-1 of it (the reference's tolerance), consistent with its own x; the
    new_bounds batch (cuOptSolveClimbers, cold start) agrees the same way.  Beyond the reference:
    each branch takes the oracle's iteration count."""
    dm = lpm.ReadMps(golden_dir / "afiro_original.mps")
    v = oracle_view(dm)
    frac, root = [1, 2, 4], [0.891, 0.109, 0.636429]
    s = settings(tol=1e-4)
    sols, _ = lpm.BatchPDLPStrongBranching(dm, frac, root, s)
    var = frac + frac
    lo = [v.var_lo[j] for j in frac] + [np.ceil(r) for r in root]
    up = [np.floor(r) for r in root] + [v.var_up[j] for j in frac]
    cold, _ = lpm.SolveClimbers(dm, var, lo, up, s)
    ref = O.strong_branching(v, frac, root, tol=1e-4)
    assert len(sols) == len(cold) == 6
    for i in range(6):
        q = _modified(v, var[i], lo[i], up[i])
        single = lpm.Solve(datamodel_from_lp(q, offset=v.obj_offset), s)
        for sol in (sols[i], cold[i]):
            assert sol.get_termination_status() == single.get_termination_status()
            assert abs(sol.get_primal_objective() - single.get_primal_objective()) <= 1e-1
            x = sol.get_primal_solution()
            assert abs(float(v.c @ x) + v.obj_offset - sol.get_primal_objective()) <= \
                1e-9 * (1 + abs(sol.get_primal_objective()))
            assert lo[i] - 1e-9 <= x[var[i]] <= up[i] + 1e-9
        assert sols[i].get_lp_stats()["nb_iterations"] == ref[i][0]["iterations"]
