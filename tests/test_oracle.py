"""The CPU oracle pinned against the reference's golden values and against constructed optima.

The oracle (oracle/pdlp_oracle.cpp) is the FP64 restatement of the reference's Stable3 PDLP path.
These tests run on the CPU only.
"""
from __future__ import annotations

import numpy as np
import pytest

from cuopt_b200 import generators as gen
from cuopt_b200 import linear_programming as lpm
from oracle import oracle as O
from tests.helpers import (MAXIMIZE_DUAL_RHS, chess_set_lp, oracle_view, reference_maximize_dual_lp,
                           reference_ranged_lp, rel, trivial_two_row_lp)


def test_methodical1_initial_step_and_weight_match_reference_golden(golden, golden_dir):
    """pdlp_test.cu:243-286: Methodical1 initial step size 1.4893 and primal weight 0.0141652 on
    afiro.  Pins Ruiz (5 passes), Pock-Chambolle (alpha 1), max-|A| step size and the
    combined-bounds primal weight."""
    dm = lpm.ReadMps(golden_dir / "afiro_original.mps")
    step, weight = O.initial_step_and_weight(oracle_view(dm), mode=2)
    g1 = golden["afiro_methodical1_initial_step_size"]
    g2 = golden["afiro_methodical1_initial_primal_weight"]
    assert abs(step - g1["value"]) <= g1["abs_tol"]
    assert abs(weight - g2["value"]) <= g2["abs_tol"]


def test_stable3_initial_weight_is_one(golden_dir):
    """Stable3 with bound/objective rescaling uses primal weight 1 (pdlp.cu:2799-2810)."""
    dm = lpm.ReadMps(golden_dir / "afiro_original.mps")
    step, weight = O.initial_step_and_weight(oracle_view(dm), mode=4)
    assert weight == 1.0
    assert 0.0 < step < 10.0


def test_afiro_objective(golden, golden_dir):
    g = golden["afiro_objective"]
    dm = lpm.ReadMps(golden_dir / "afiro_original.mps")
    res, x, y, _ = O.solve(oracle_view(dm), tol=1e-4)
    assert res["status"] == 1
    assert rel(res["primal_obj"], g["value"]) <= g["rel_tol"]
    res8, _, _, _ = O.solve(oracle_view(dm), tol=1e-8)
    assert abs(res8["primal_obj"] - g["value"]) <= 1e-4


@pytest.mark.parametrize("name,key", [("max_offset.mps", "max_offset_objective"),
                                      ("good-max.mps", "good_max_objective")])
def test_maximize_fixtures(golden, golden_dir, name, key):
    dm = lpm.ReadMps(golden_dir / name)
    res, _, _, _ = O.solve(oracle_view(dm), tol=1e-8)
    assert res["status"] == 1
    assert abs(res["primal_obj"] - golden[key]["value"]) <= golden[key]["abs_tol"]


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_constructed_optimum_small(seed):
    lp = gen.constructed_lp(200, 500, 8, seed=seed)
    res, x, y, _ = O.solve(lp, tol=1e-7)
    assert res["status"] == 1
    assert rel(res["primal_obj"], lp.optimal_objective) <= 1e-6
    kkt = gen.kkt_relative_error(lp, x, y)
    assert kkt["rel_primal"] <= 1e-7 and kkt["rel_gap"] <= 1e-7


def test_constructed_optimum_2000x5000():
    """The 2000 x 5000 LP to 1e-6: objective within 1e-6 relative of the constructed optimum."""
    lp = gen.constructed_lp(2000, 5000, 8, seed=0)
    res, x, y, _ = O.solve(lp, tol=1e-6)
    assert res["status"] == 1
    assert rel(res["primal_obj"], lp.optimal_objective) <= 1e-5
    assert gen.kkt_relative_error(lp, x, y)["rel_primal"] <= 1e-6


def test_skewed_generator_is_consistent():
    lp = gen.skewed_lp(400, 1200, seed=3, cap=300)
    kkt = gen.kkt_relative_error(lp, lp.x_star, lp.y_star)
    assert kkt["rel_primal"] < 1e-12 and kkt["rel_dual"] < 1e-12 and kkt["rel_gap"] < 1e-9
    res, x, y, _ = O.solve(lp, tol=1e-6)
    assert res["status"] == 1
    assert rel(res["primal_obj"], lp.optimal_objective) <= 1e-4


def test_constructed_generator_kkt_exact():
    lp = gen.constructed_lp(300, 800, 8, seed=4)
    kkt = gen.kkt_relative_error(lp, lp.x_star, lp.y_star)
    assert max(kkt["rel_primal"], kkt["rel_dual"], kkt["rel_gap"]) < 1e-12


def test_iteration_limit_and_no_constraints():
    lp = gen.constructed_lp(100, 250, 8, seed=9)
    res, _, _, _ = O.solve(lp, tol=1e-12, iteration_limit=1)
    assert res["status"] == 4 and res["iterations"] == 10  # limit checked at conditional majors
    res0, _, _, _ = O.solve(lp, tol=1e-12, iteration_limit=0)
    assert res0["status"] == 4 and res0["iterations"] == 0


def test_highs_cross_check():
    """Third-party cross-check (SciPy HiGHS, not the reference) on a small constructed LP."""
    scipy = pytest.importorskip("scipy")
    from scipy.optimize import linprog
    from scipy.sparse import csr_matrix

    lp = gen.constructed_lp(150, 400, 8, seed=21)
    A = csr_matrix((lp.val, lp.col_idx, lp.row_off), shape=(lp.m, lp.n))
    r = linprog(lp.c, A_eq=A, b_eq=lp.con_lo, bounds=list(zip(lp.var_lo, lp.var_up)),
                method="highs")
    assert r.status == 0
    assert rel(r.fun, lp.optimal_objective) <= 1e-9
    res, _, _, _ = O.solve(lp, tol=1e-8)
    assert rel(res["primal_obj"], r.fun) <= 1e-7


def test_infeasibility_detection(golden_dir):
    """With detection on, both infeasible cases end PrimalInfeasible at one of the two checks that
    test it (iterations 200 and 400); with it off they run to the iteration limit, and a feasible
    LP follows the same iterations either way."""
    from tests.helpers import infeasible_cases, oracle_view
    for name, lp in infeasible_cases(golden_dir):
        res, _, _, _ = O.solve(lp, tol=1e-6, iteration_limit=3000, detect_infeasibility=True)
        assert res["status"] == 2 and res["iterations"] in (200, 400), (name, res)
        res, _, _, _ = O.solve(lp, tol=1e-6, iteration_limit=3000)
        assert res["status"] == 4, name
    afiro = oracle_view(lpm.ReadMps(golden_dir / "afiro_original.mps"))
    a, _, _, _ = O.solve(afiro, tol=1e-6, detect_infeasibility=True)
    b, _, _, _ = O.solve(afiro, tol=1e-6)
    assert a["status"] == b["status"] == 1 and a["iterations"] == b["iterations"]


def test_warm_start_from_a_nearby_point_converges_faster():
    """Starting from a perturbation of the constructed optimum (cuOptSetInitialPrimalSolution /
    cuOptSetInitialDualSolution) reaches 1e-6 in fewer iterations than the cold start."""
    lp = gen.constructed_lp(200, 500, 8, seed=11)
    rng = np.random.default_rng(3)
    x0 = lp.x_star + 1e-3 * rng.standard_normal(lp.n)
    y0 = lp.y_star + 1e-3 * rng.standard_normal(lp.m)
    cold, _, _, _ = O.solve(lp, tol=1e-6)
    warm, _, _, _ = O.solve(lp, tol=1e-6, initial_primal=x0, initial_dual=y0)
    assert cold["status"] == warm["status"] == 1
    assert warm["iterations"] < cold["iterations"]


def test_given_step_size_and_primal_weight():
    """A step size and primal weight passed in (as the strong-branching batch passes them)
    replace the power iteration and the initial weight: passing the values the solver computes
    itself changes nothing, and no power iteration runs."""
    lp = gen.constructed_lp(200, 500, 8, seed=11)
    cold, xc, yc, _ = O.solve(lp, tol=1e-12, iteration_limit=300)
    step, weight = O.initial_step_and_weight(lp)
    given, xg, yg, _ = O.solve(lp, tol=1e-12, iteration_limit=300, initial_step_size=step,
                               initial_primal_weight=weight)
    assert given["power_iterations"] == 0 < cold["power_iterations"]
    assert given["step_size"] == cold["step_size"]
    assert np.array_equal(xg, xc) and np.array_equal(yg, yc)
    other, _, _, _ = O.solve(lp, tol=1e-12, iteration_limit=300, initial_step_size=0.5 * step,
                             initial_primal_weight=2.0)
    assert other["step_size"] == 0.5 * step


def test_strong_branching_restatement():
    """batch_pdlp_solve on the oracle: every branch starts from the LP's own solution; branches
    that keep the LP's optimum feasible finish within a few checks."""
    lp = gen.constructed_lp(200, 500, 8, seed=11)
    rng = np.random.default_rng(5)
    frac = rng.choice(lp.n, 3, replace=False)
    root = lp.x_star[frac] + 0.5
    out = O.strong_branching(lp, frac, root, tol=1e-6)
    assert len(out) == 6
    for i, (res, x, _, _) in enumerate(out):
        j = frac[i % 3]
        assert res["status"] == 1 and res["power_iterations"] == 0
        if i < 3:
            assert x[j] <= np.floor(root[i]) + 1e-6
        else:
            assert x[j] >= np.ceil(root[i - 3]) - 1e-6


def _identity_lp():
    """pdlp_test.cu:640-733: A = I (3 x 3), 0 <= Ax <= 0, c = 0, free variables."""
    from types import SimpleNamespace
    z = np.zeros(3)
    return SimpleNamespace(row_off=np.arange(4), col_idx=np.arange(3), val=np.ones(3), c=z,
                           con_lo=z, con_up=z, var_lo=np.full(3, -np.inf),
                           var_up=np.full(3, np.inf), obj_offset=0.0, maximize=False, m=3, n=3)


def test_per_constraint_residual_on_the_reference_point():
    """pdlp_test.cu:640-733: at x = (0.02, 0.03, 0.1) the per-constraint primal residual is
    exactly 0.1 (and passes an absolute tolerance of 0.1) while the l2 residual is 0.106."""
    x0 = np.array([0.02, 0.03, 0.1])
    pcr, _, _, _ = O.solve(_identity_lp(), tol=0.1, iteration_limit=0, initial_primal=x0,
                           per_constraint_residual=True)
    l2, _, _, _ = O.solve(_identity_lp(), tol=0.1, iteration_limit=0, initial_primal=x0)
    assert pcr["l2_primal"] == 0.1
    assert l2["l2_primal"] == np.sqrt(0.02 ** 2 + 0.03 ** 2 + 0.1 ** 2) > 0.1


def test_per_constraint_residual_solve():
    """Under the per-constraint criterion the reported residuals are the per-constraint maxima of
    the returned point (checked here in numpy).  The dual form subtracts rel * c_j with the sign of
    c_j, as the reference does, so with c_j < -1 it stays above the tolerance: this LP runs to its
    iteration limit."""
    lp = gen.constructed_lp(200, 500, 8, seed=11)
    tol = 1e-3
    res, x, y, rc = O.solve(lp, tol=tol, iteration_limit=1000, time_limit=30,
                            per_constraint_residual=True)
    assert res["status"] == 4
    A = np.zeros((lp.m, lp.n))
    rows = np.repeat(np.arange(lp.m), np.diff(lp.row_off))
    A[rows, lp.col_idx] = lp.val
    ax = A @ x
    rp = ax - np.clip(ax, lp.con_lo, lp.con_up)
    cb = np.maximum(np.where(np.isfinite(lp.con_up), np.abs(lp.con_up), 0),
                    np.where(np.isfinite(lp.con_lo), np.abs(lp.con_lo), 0))
    rd = (lp.c - A.T @ y) - rc
    assert abs(res["l2_primal"] - max(0.0, np.max(rp - tol * cb))) <= 1e-12
    assert abs(res["l2_dual"] - max(0.0, np.max(rd - tol * lp.c))) <= 1e-12
    assert res["l2_dual"] > tol < tol * np.max(-lp.c)


def test_skewed_generator_with_explicit_slacks():
    """The skewed LP as specified: one slack column per '<=' row, every row an equality; the
    constructed optimum stays exact and the objective is unchanged."""
    a = gen.skewed_lp(2000, 6000, seed=7, cap=500)
    b = gen.skewed_lp(2000, 6000, seed=7, cap=500, explicit_slacks=True)
    k = int(np.sum(~np.isfinite(a.con_lo)))
    assert b.n == a.n + k and b.nnz == a.nnz + k
    assert np.array_equal(b.con_lo, b.con_up)
    e = gen.kkt_relative_error(b, b.x_star, b.y_star)
    assert e["rel_primal"] <= 1e-12 and e["rel_dual"] <= 1e-12 and e["rel_gap"] <= 1e-12
    assert b.optimal_objective == a.optimal_objective
    res, _, _, _ = O.solve(b, tol=1e-4, iteration_limit=20000, time_limit=60)
    assert res["status"] == 1


def test_tiny_lp_of_the_reference_python_tests():
    """test_lp_solver.py:46-80: x <= 1 twice, min x over x >= 0.  Optimal with x = 0, zero
    residuals, objectives and gap (the reference runs it in Stable2 because its Stable3 loops on
    it; the Stable3 restatement ends Optimal at the first check after iteration 1)."""
    from types import SimpleNamespace
    inf = np.inf
    lp = SimpleNamespace(row_off=np.array([0, 1, 2]), col_idx=np.array([0, 0]),
                         val=np.array([1.0, 1.0]), c=np.array([1.0]),
                         con_lo=np.array([-inf, -inf]), con_up=np.array([1.0, 1.0]),
                         var_lo=np.array([0.0]), var_up=np.array([inf]), obj_offset=0.0,
                         maximize=False)
    res, x, y, _ = O.solve(lp, tol=1e-2, iteration_limit=10000, time_limit=10)
    assert res["status"] == 1
    assert x[0] == 0.0 and res["primal_obj"] == 0.0 and res["dual_obj"] == 0.0
    assert res["l2_primal"] == 0.0 and res["l2_dual"] == 0.0 and res["gap"] == 0.0


@pytest.mark.parametrize("tol", [1e-4, 1e-6, 1e-8])
def test_reference_ranged_problem(golden, tol):
    """c_api_tests.cpp:105-112: Optimal with objective 32 within 1e-3."""
    g = golden["ranged_problem_objective"]
    res, _, _, _ = O.solve(oracle_view(reference_ranged_lp()), tol=tol)
    assert res["status"] == 1
    assert abs(res["primal_obj"] - g["value"]) <= g["abs_tol"]


def test_reference_maximize_dual_variables(golden):
    """c_api_tests.cpp:149-165: for a maximisation, the objective equals sum_i y_i rhs_i within
    1e-2 (the PDLP tolerance there) at the default tolerance, which pins the sign of the duals."""
    g = golden["maximize_dual_objective_match"]
    res, x, y, _ = O.solve(oracle_view(reference_maximize_dual_lp()), tol=1e-4)
    assert res["status"] == 1
    assert abs(res["primal_obj"] - y @ MAXIMIZE_DUAL_RHS) <= g["abs_tol"]
    assert (y >= 0).all()


@pytest.mark.parametrize("tol", [1e-6, 1e-8])
def test_chess_set(golden, tol):
    """dual_simplex/unit_tests/solve.cpp:86-88: objective 1333.33 (1e-2), x = (0 (1e-6), 66.6667
    (1e-3))."""
    g = golden["chess_set_dual_simplex"]
    res, x, _, _ = O.solve(oracle_view(chess_set_lp()), tol=tol)
    assert res["status"] == 1
    assert abs(res["primal_obj"] - g["objective"]) <= 1e-2
    assert abs(x[0] - g["x"][0]) <= 1e-6 and abs(x[1] - g["x"][1]) <= 1e-3


def test_trivial_two_row_lp():
    """python/cuopt/cuopt/tests/linear_programming/test_lp_solver.py:46-79 (run there in Stable2):
    Optimal at 1e-2 with x = 0, objectives 0 and gap 0."""
    res, x, y, _ = O.solve(oracle_view(trivial_two_row_lp()), tol=1e-2)
    assert res["status"] == 1
    assert x[0] == pytest.approx(0.0)
    assert res["primal_obj"] == pytest.approx(0.0) and res["dual_obj"] == pytest.approx(0.0)
    assert res["gap"] == pytest.approx(0.0)


@pytest.mark.parametrize("j,lo,up", [(5, 4.0, 5.0), (1, -7.0, 13.0)])
def test_afiro_with_the_reference_batch_tests_bounds(golden_dir, j, lo, up):
    """The climbers of pdlp_test.cu:1138-1287 (afiro with variable 5 in [4, 5], or variable 1 in
    [-7, 13]) solve Optimal on the oracle, at HiGHS's optimum (1e-7 relative at 1e-8 tolerance)."""
    pytest.importorskip("scipy")
    from tests.helpers import highs_objective, with_variable_bounds
    q = with_variable_bounds(oracle_view(lpm.ReadMps(golden_dir / "afiro_original.mps")), j, lo, up)
    res, _, _, _ = O.solve(q, tol=1e-8)
    assert res["status"] == 1
    assert rel(res["primal_obj"], highs_objective(q)) <= 1e-7


def _bound_variants(view, g):
    from tests.helpers import with_variable_bounds
    j = g["variable"]
    return [view if lo is None else with_variable_bounds(view, j, lo, g["upper"]) for lo in g["lower"]]


def _violation(q, x):
    from scipy.sparse import csr_matrix
    ax = csr_matrix((q.val, q.col_idx, q.row_off), shape=(q.m, q.n)) @ x
    return max(np.max(np.maximum(0.0, ax - q.con_up)), np.max(np.maximum(0.0, q.con_lo - ax)),
               np.max(np.maximum(0.0, q.var_lo - x)), np.max(np.maximum(0.0, x - q.var_up)))


def test_many_different_bounds(golden, golden_dir):
    """pdlp_test.cu:1720-1804: the 13 bound variants of good-mps-some-var-bounds solve Optimal with
    constraint violations under 1e-8, at HiGHS's optimum (1e-9 relative)."""
    pytest.importorskip("scipy")
    from tests.helpers import highs_objective
    g = golden["many_different_bounds"]
    view = oracle_view(lpm.ReadMps(golden_dir / "good-mps-some-var-bounds.mps"))
    for q in _bound_variants(view, g):
        res, x, _, _ = O.solve(q)
        assert res["status"] == 1
        assert _violation(q, x) <= g["constraint_tol"]
        assert rel(res["primal_obj"], highs_objective(q)) <= 1e-9


def test_some_climber_hits_the_iteration_limit(golden, golden_dir):
    """pdlp_test.cu:1806-1885: at 500 iterations the variant with variable 0 down to -2533 hits the
    limit, the unchanged LP is Optimal."""
    g = golden["some_climber_hit_iteration_limit"]
    view = oracle_view(lpm.ReadMps(golden_dir / "good-mps-some-var-bounds.mps"))
    want = {"IterationLimit": 4, "Optimal": 1}
    for q, status in zip(_bound_variants(view, g), g["statuses"]):
        res, _, _, _ = O.solve(q, iteration_limit=g["iteration_limit"])
        assert res["status"] == want[status]


def test_good_mps_1(golden, golden_dir):
    """test_lp_solver.py:82-89: good-mps-1 is Optimal at tolerance 1e-2."""
    g = golden["good_mps_1_optimal"]
    res, _, _, _ = O.solve(oracle_view(lpm.ReadMps(golden_dir / "good-mps-1.mps")), tol=g["tol"])
    assert res["status"] == 1


def test_afiro_at_the_minimal_absolute_tolerance(golden, golden_dir):
    """pdlp_test.cu:76-100: absolute tolerances at their minimum 1e-12 and relative ones 0 still end
    Optimal, at afiro's objective (1 %)."""
    v = oracle_view(lpm.ReadMps(golden_dir / "afiro_original.mps"))
    res, _, _, _ = O.solve(v, abs_tol=1e-12, rel_tol=0.0, time_limit=120)
    assert res["status"] == 1
    assert rel(res["primal_obj"], golden["afiro_objective"]["value"]) <= 0.01
    assert res["l2_primal"] <= 1e-12 and res["l2_dual"] <= 1e-12


def test_afiro_from_an_all_ones_primal(golden, golden_dir):
    """pdlp_test.cu:102-122: started from x = 1, afiro ends Optimal at its objective (1 %)."""
    v = oracle_view(lpm.ReadMps(golden_dir / "afiro_original.mps"))
    res, _, _, _ = O.solve(v, initial_primal=np.ones(v.n))
    assert res["status"] == 1
    assert rel(res["primal_obj"], golden["afiro_objective"]["value"]) <= 0.01


def test_afiro_iteration_limit_returns_the_current_iterate(golden_dir):
    """pdlp_test.cu:124-147: 10 iterations with tolerance 0 end IterationLimit with the current
    (non-zero) primal iterate."""
    v = oracle_view(lpm.ReadMps(golden_dir / "afiro_original.mps"))
    res, x, _, _ = O.solve(v, tol=0.0, iteration_limit=10)
    assert res["status"] == 4 and res["iterations"] == 10
    assert np.any(x != 0.0)


def test_objective_error_at_1e6_kkt_is_not_bounded_by_1e6():
    """Instance 284 of the 512-LP batch (481 x 1202, optimum 46.62, |b| = 278): at 1e-6 relative
    KKT the oracle's objective is 6.8e-6 (relative) from the constructed optimum, because the
    residuals are measured against |b| and |c| while the objective is much smaller; at 1e-8 it is
    within 1e-6.  This is why objective bounds are tested on solves to 1e-8."""
    from tests.helpers import OBJ_RTOL, REFINED_TOL, rel
    lp = gen.batch_instance(284)
    res6, _, _, _ = O.solve(lp, tol=1e-6)
    res8, _, _, _ = O.solve(lp, tol=REFINED_TOL)
    assert res6["status"] == res8["status"] == 1
    assert max(res6["rel_primal"], res6["rel_dual"], res6["rel_gap"]) <= 1e-6
    assert rel(res6["primal_obj"], lp.optimal_objective) > 5e-6
    assert rel(res8["primal_obj"], lp.optimal_objective) <= OBJ_RTOL


@pytest.mark.parametrize("i", [0, 257, 284, 458, 511])
def test_oracle_fixture_entries_reproduce(i):
    """Spot checks of tests/golden/oracle_results.json against the oracle run now (the fixture is
    what the GPU tests and the bench compare with)."""
    from tests.helpers import oracle_results
    fx = oracle_results()["batch"][i]
    lp = gen.batch_instance(i)
    assert (lp.m, lp.n) == (fx["m"], fx["n"])
    assert abs(lp.optimal_objective - fx["optimal_objective"]) <= 1e-12 * max(1.0, abs(fx["optimal_objective"]))
    for tol in (1e-6, 1e-8):
        res, _, _, _ = O.solve(lp, tol=tol)
        want = fx[f"{tol:g}"]
        assert res["status"] == want["status"]
        assert res["iterations"] == want["iterations"]
        assert abs(res["primal_obj"] - want["primal_objective"]) <= 1e-12 * max(1.0, abs(want["primal_objective"]))


_ref_missing = pytest.mark.skipif(
    not __import__("oracle.ref_simplex", fromlist=["available"]).available(),
    reason="oracle/_ref/ref_dual_simplex not built (make -C oracle ref REF=<reference root>)")


@_ref_missing
def test_reference_dual_simplex_chess_set(golden):
    """The reference's own CPU dual simplex, compiled from its sources, reproduces the known answer
    of its unit test (cpp/tests/dual_simplex/unit_tests/solve.cpp:86-88): 1333.33 at (0, 66.6667)."""
    from oracle import ref_simplex as R
    g = golden["chess_set_dual_simplex"]
    v = oracle_view(chess_set_lp())
    res, x = R.solve(v, maximize=bool(v.maximize))
    assert res["status"] == "OPTIMAL"
    assert abs(res["objective"] - g["objective"]) <= g["tol"] * abs(g["objective"])
    assert np.allclose(x, g["x"], atol=1e-4)


@_ref_missing
def test_reference_dual_simplex_agrees_with_the_oracle_on_a_small_lp():
    """On a 60 x 150 constructed LP the reference dual simplex and the FP64 PDLP oracle (1e-9)
    reach the constructed optimum."""
    from oracle import ref_simplex as R
    lp = gen.constructed_lp(60, 150, 6, seed=3)
    res, x = R.solve(lp)
    o, _, _, _ = O.solve(lp, tol=1e-9)
    assert res["status"] == "OPTIMAL" and o["status"] == 1
    assert abs(res["objective"] - lp.optimal_objective) <= 1e-6 * abs(lp.optimal_objective)
    assert abs(o["primal_obj"] - lp.optimal_objective) <= 1e-6 * abs(lp.optimal_objective)
