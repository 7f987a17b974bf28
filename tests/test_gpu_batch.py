"""GPU parity tests of the batched PDLP (cuOptBatchSolve / BatchSolve): every instance of a
block-diagonal batch must follow its own single-LP Stable3 trajectory.

Reference for every expectation: the CPU oracle solving each instance alone (an FP64 restatement of
the reference's Stable3 PDLP) and the optima known by construction.  Tolerances: iterates after the
same number of iterations agree with the oracle to 1e-9 relative to the vector's magnitude
(summation order differs); solved instances reach the relative KKT targets asked for, and on solves
to 1e-8 relative KKT (FP64, or mixed precision refined in FP64) the objectives are within
OBJ_RTOL = 1e-6 of the constructed optima and of the oracle's.
"""
from __future__ import annotations

import numpy as np
import pytest

from cuopt_b200 import generators as gen
from cuopt_b200 import linear_programming as lpm
from oracle import oracle as O
from tests.helpers import (OBJ_RTOL, REFINED_TOL, datamodel_from_lp, oracle_results, oracle_view,
                           refined_settings, rel, relative_kkt, settings)

pytestmark = pytest.mark.gpu

ITERATE_RTOL = 1e-9


@pytest.fixture(scope="module")
def instances():
    """Uneven sizes, a maximisation with an offset, and one instance with long rows."""
    lps = [gen.constructed_lp(m, int(2.5 * m), k, seed=50 + i)
           for i, (m, k) in enumerate([(200, 6), (1300, 12), (450, 8), (3000, 9)])]
    lps.append(gen.skewed_lp(400, 3000, seed=7, cap=3000))
    return lps


def _models(lps, maximize_index=None):
    dms = []
    for i, lp in enumerate(lps):
        if i == maximize_index:
            dm = datamodel_from_lp(lp, maximize=True, offset=1.25)
            dm.set_objective_coefficients(-lp.c)
        else:
            dm = datamodel_from_lp(lp)
        dms.append(dm)
    return dms


@pytest.mark.parametrize("k", [10, 200, 1000])
def test_batch_iterates_match_single_oracle(instances, k):
    dms = _models(instances)
    sols, _ = lpm.BatchSolve(dms, settings(tol=1e-12, iteration_limit=k))
    for lp, sol in zip(instances, sols):
        res, x, y, rc = O.solve(lp, tol=1e-12, iteration_limit=k)
        assert sol.get_termination_status() == lpm.LPTerminationStatus.IterationLimit
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        assert np.max(np.abs(sol.get_primal_solution() - x)) <= ITERATE_RTOL * (1 + np.abs(x).max())
        assert np.max(np.abs(sol.get_dual_solution() - y)) <= ITERATE_RTOL * (1 + np.abs(y).max())
        assert np.max(np.abs(sol.get_reduced_cost() - rc)) <= ITERATE_RTOL * (1 + np.abs(rc).max())
        assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-9


def test_batch_solves_to_tolerance_like_single_solves(instances):
    """Each instance terminates Optimal at 1e-6 at the oracle's iteration count with the oracle's
    objective (1e-9), with its own restarts; at 1e-8 the constructed optima are recovered within
    OBJ_RTOL."""
    lps = instances[:4]
    dms = _models(lps, maximize_index=2)
    sols, _ = lpm.BatchSolve(dms, settings(tol=1e-6))
    tight, _ = lpm.BatchSolve(dms, settings(tol=REFINED_TOL))
    for i, (lp, dm, sol, t) in enumerate(zip(lps, dms, sols, tight)):
        res, _, _, _ = O.solve(oracle_view(dm), tol=1e-6)
        assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
        assert res["status"] == 1
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-9
        want = -lp.optimal_objective + 1.25 if i == 2 else lp.optimal_objective
        assert t.get_termination_status() == lpm.LPTerminationStatus.Optimal
        assert relative_kkt(t) <= REFINED_TOL
        assert rel(t.get_primal_objective(), want) <= OBJ_RTOL


def test_batch_is_deterministic(instances):
    dms = _models(instances)
    a, _ = lpm.BatchSolve(dms, settings(tol=1e-12, iteration_limit=300))
    b, _ = lpm.BatchSolve(dms, settings(tol=1e-12, iteration_limit=300))
    for sa, sb in zip(a, b):
        assert np.array_equal(sa.get_primal_solution(), sb.get_primal_solution())
        assert np.array_equal(sa.get_dual_solution(), sb.get_dual_solution())


def test_batch_mixes_special_cases(golden, golden_dir, instances):
    """Problems that never reach PDLP (no constraints) are answered as single solves would."""
    dms = [datamodel_from_lp(instances[0]),
           lpm.ReadMps(golden_dir / "lp-model-no-constraints.mps"),
           datamodel_from_lp(instances[2])]
    s = settings(tol=1e-6, method=lpm.SolverMethod.Concurrent)
    sols, _ = lpm.BatchSolve(dms, s)
    assert sols[0].get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert sols[2].get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert sols[1].get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert not sols[1].get_solved_by_pdlp()
    assert abs(sols[1].get_primal_objective() - golden["no_constraints_objective"]["value"]) <= 1e-4
    single = lpm.Solve(datamodel_from_lp(instances[2]), s)
    assert sols[2].get_lp_stats()["nb_iterations"] == single.get_lp_stats()["nb_iterations"]


def test_mixed_batch_follows_single_mixed_solves(instances):
    """In mixed precision every instance takes its step size from Golub-Kahan-Lanczos, as a single
    mixed solve does: the same number of Lanczos steps and the same step size (1e-12 relative;
    summation order differs), Optimal at 1e-6 with the single solve's iteration count (±5 %) and
    relative KKT <= 1e-6; refined in FP64 to 1e-8, the constructed optima within OBJ_RTOL."""
    lps = instances[:4]
    dms = _models(lps)
    s = settings(tol=1e-6, precision=1)
    sols, _ = lpm.BatchSolve(dms, s)
    for lp, dm, sol in zip(lps, dms, sols):
        single = lpm.Solve(dm, s)
        assert sol.get_termination_status() == single.get_termination_status() == \
            lpm.LPTerminationStatus.Optimal
        assert sol.stats["power_iterations"] == single.stats["power_iterations"] > 0
        assert rel(sol.stats["step_size"], single.stats["step_size"]) <= 1e-12
        si, bi = single.get_lp_stats()["nb_iterations"], sol.get_lp_stats()["nb_iterations"]
        assert abs(bi - si) <= 0.05 * si + 10
        assert relative_kkt(sol) <= 1e-6
    refined, _ = lpm.BatchSolve(dms, refined_settings())
    for lp, sol in zip(lps, refined):
        assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
        assert sol.stats["refinement_passes"] == 1
        assert relative_kkt(sol) <= REFINED_TOL
        assert rel(sol.get_primal_objective(), lp.optimal_objective) <= OBJ_RTOL


def _c3_subset(count=32):
    """`count` instances of the 512-LP batch spread over its size range (every 16th by size)."""
    fx = oracle_results()["batch"]
    order = sorted(range(len(fx)), key=lambda i: fx[i]["m"])
    return [order[int(q)] for q in np.linspace(0, len(order) - 1, count)], fx


def test_c3_subset_fp64_matches_oracle_fixture():
    """32 instances of the 512-LP batch (200 to 20 000 rows) in one FP64 batch at 1e-6: every
    instance ends with the oracle's status and iteration count and its objective within 1e-9
    relative (tests/golden/oracle_results.json); at 1e-8, every objective is within OBJ_RTOL of the
    constructed optimum and of the oracle's 1e-8 objective."""
    ids, fx = _c3_subset()
    lps = [gen.batch_instance(i) for i in ids]
    dms = [datamodel_from_lp(lp) for lp in lps]
    sols, _ = lpm.BatchSolve(dms, settings(tol=1e-6))
    for i, lp, sol in zip(ids, lps, sols):
        want = fx[i]["1e-06"]
        assert int(sol.get_termination_status()) == want["status"] == 1
        assert sol.get_lp_stats()["nb_iterations"] == want["iterations"], i
        assert rel(sol.get_primal_objective(), want["primal_objective"]) <= 1e-9, i
        assert relative_kkt(sol) <= 1e-6
    tight, _ = lpm.BatchSolve(dms, settings(tol=REFINED_TOL))
    for i, lp, sol in zip(ids, lps, tight):
        want = fx[i]["1e-08"]
        assert int(sol.get_termination_status()) == want["status"] == 1
        assert rel(sol.get_primal_objective(), want["primal_objective"]) <= 1e-9, i
        assert rel(sol.get_primal_objective(), lp.optimal_objective) <= OBJ_RTOL, i


def test_c3_subset_mixed_refined_meets_objective_bound():
    """The same 32 instances in one mixed-precision batch: Optimal at 1e-6 relative KKT; refined in
    FP64 to 1e-8, every objective within OBJ_RTOL of the constructed optimum and of the oracle's
    1e-8 objective."""
    ids, fx = _c3_subset()
    lps = [gen.batch_instance(i) for i in ids]
    dms = [datamodel_from_lp(lp) for lp in lps]
    sols, _ = lpm.BatchSolve(dms, settings(tol=1e-6, precision=1))
    assert all(int(s.get_termination_status()) == 1 for s in sols)
    assert max(relative_kkt(s) for s in sols) <= 1e-6
    refined, _ = lpm.BatchSolve(dms, refined_settings())
    for i, lp, sol in zip(ids, lps, refined):
        assert int(sol.get_termination_status()) == 1
        assert relative_kkt(sol) <= REFINED_TOL
        assert rel(sol.get_primal_objective(), lp.optimal_objective) <= OBJ_RTOL, i
        assert rel(sol.get_primal_objective(), fx[i]["1e-08"]["primal_objective"]) <= OBJ_RTOL, i
