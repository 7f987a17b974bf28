"""GPU parity tests of the PDLP path through the C-ABI (libcuopt_b200.so).

Reference for every expectation: the CPU oracle (oracle/pdlp_oracle.cpp, an FP64 restatement of the
reference's Stable3 PDLP), the optimum known by construction of the synthetic LPs, and the golden
values of the reference's own tests (tests/golden/golden.json).

Floating-point tolerances (FP64 path): iterates after the same number of iterations agree with the
oracle to 1e-9 relative (summation order differs), objectives to 1e-9 relative, and solved
problems reach the relative KKT targets asked for.  Objectives are held to OBJ_RTOL = 1e-6
relative of the constructed optimum and of the FP64 oracle on solves to 1e-8 relative KKT (FP64, or
mixed precision refined in FP64): 1e-6 KKT alone does not bound the objective error by 1e-6.
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
def small_lp():
    return gen.constructed_lp(200, 500, 8, seed=11)


@pytest.mark.parametrize("k", [0, 10, 50, 200, 400, 1000])
def test_iterates_match_oracle(small_lp, k):
    """Same returned iterate as the oracle after k iterations (iteration limit)."""
    dm = datamodel_from_lp(small_lp)
    sol = lpm.Solve(dm, settings(tol=1e-12, iteration_limit=k))
    res, x, y, rc = O.solve(small_lp, tol=1e-12, iteration_limit=k)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.IterationLimit
    assert res["status"] == 4
    assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
    sx, sy = sol.get_primal_solution(), sol.get_dual_solution()
    scale_x = 1.0 + np.max(np.abs(x))
    scale_y = 1.0 + np.max(np.abs(y))
    assert np.max(np.abs(sx - x)) <= ITERATE_RTOL * scale_x
    assert np.max(np.abs(sy - y)) <= ITERATE_RTOL * scale_y
    assert np.max(np.abs(sol.get_reduced_cost() - rc)) <= ITERATE_RTOL * (1 + np.max(np.abs(rc)))
    assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-9
    assert rel(sol.get_dual_objective(), res["dual_obj"]) <= 1e-9


def test_solve_matches_oracle_and_optimum(small_lp):
    """At 1e-6: the oracle's status, iteration count and objective (1e-9 relative) and relative KKT
    <= 1e-6; at 1e-8: the constructed optimum and the oracle's objective within OBJ_RTOL."""
    dm = datamodel_from_lp(small_lp)
    sol = lpm.Solve(dm, settings(tol=1e-6))
    res, x, y, _ = O.solve(small_lp, tol=1e-6)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert res["status"] == 1
    assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
    assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-9
    assert relative_kkt(sol) <= 1e-6
    kkt = gen.kkt_relative_error(small_lp, sol.get_primal_solution(), sol.get_dual_solution())
    assert kkt["rel_primal"] <= 1e-6 and kkt["rel_gap"] <= 1e-6
    tight = lpm.Solve(dm, settings(tol=REFINED_TOL))
    res8, _, _, _ = O.solve(small_lp, tol=REFINED_TOL)
    assert rel(tight.get_primal_objective(), small_lp.optimal_objective) <= OBJ_RTOL
    assert rel(tight.get_primal_objective(), res8["primal_obj"]) <= 1e-9


def test_config0_full_size():
    """The 2000 x 5000 LP (8 nnz / column): Optimal at 1e-6 with the oracle's status, iteration
    count and objective (1e-9); at 1e-8, FP64 and mixed precision refined in FP64 both give the
    constructed optimum and the oracle's objective within OBJ_RTOL."""
    lp = gen.constructed_lp(2000, 5000, 8, seed=0)
    dm = datamodel_from_lp(lp)
    sol = lpm.Solve(dm, settings(tol=1e-6))
    res, _, _, _ = O.solve(lp, tol=1e-6)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal == res["status"]
    assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
    assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-9
    kkt = gen.kkt_relative_error(lp, sol.get_primal_solution(), sol.get_dual_solution())
    assert max(kkt["rel_primal"], kkt["rel_gap"]) <= 1e-6
    res8, _, _, _ = O.solve(lp, tol=REFINED_TOL)
    for s in (settings(tol=REFINED_TOL), refined_settings()):
        tight = lpm.Solve(dm, s)
        assert tight.get_termination_status() == lpm.LPTerminationStatus.Optimal
        assert relative_kkt(tight) <= REFINED_TOL
        assert rel(tight.get_primal_objective(), lp.optimal_objective) <= OBJ_RTOL
        assert rel(tight.get_primal_objective(), res8["primal_obj"]) <= OBJ_RTOL


def test_afiro_objective(golden, golden_dir):
    g = golden["afiro_objective"]
    dm = lpm.ReadMps(golden_dir / "afiro_original.mps")
    sol = lpm.Solve(dm, settings(tol=1e-4))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert rel(sol.get_primal_objective(), g["value"]) <= g["rel_tol"]
    res, _, _, _ = O.solve(oracle_view(dm), tol=1e-4)
    assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
    assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-9
    tight = lpm.Solve(dm, settings(tol=1e-8))
    assert abs(tight.get_primal_objective() - g["value"]) <= 1e-4


@pytest.mark.parametrize("name,key", [("max_offset.mps", "max_offset_objective"),
                                      ("good-max.mps", "good_max_objective")])
def test_maximize_fixtures(golden, golden_dir, name, key):
    g = golden[key]
    dm = lpm.ReadMps(golden_dir / name)
    sol = lpm.Solve(dm, settings(tol=1e-8))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert abs(sol.get_primal_objective() - g["value"]) <= g["abs_tol"]


def test_no_constraints(golden, golden_dir):
    dm = lpm.ReadMps(golden_dir / "lp-model-no-constraints.mps")
    sol = lpm.Solve(dm, settings(method=lpm.SolverMethod.Concurrent))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert abs(sol.get_primal_objective() - golden["no_constraints_objective"]["value"]) <= 1e-4
    assert not sol.get_solved_by_pdlp()
    pd = lpm.Solve(lpm.ReadMps(golden_dir / "empty_matrix.mps"), settings())
    assert int(pd.get_termination_status()) == golden["empty_matrix_pdlp_status"]["value"]


def test_time_limit_zero(small_lp):
    sol = lpm.Solve(datamodel_from_lp(small_lp), settings(tol=1e-8, time_limit=0.0))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.TimeLimit


def test_inequality_and_free_rows_match_oracle():
    lp = gen.skewed_lp(300, 900, seed=5, cap=200)
    dm = datamodel_from_lp(lp)
    for k in (10, 200):
        sol = lpm.Solve(dm, settings(tol=1e-12, iteration_limit=k))
        res, x, y, _ = O.solve(lp, tol=1e-12, iteration_limit=k)
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        np.testing.assert_allclose(sol.get_primal_solution(), x, rtol=1e-8,
                                   atol=1e-8 * (1 + np.max(np.abs(x))))
        np.testing.assert_allclose(sol.get_dual_solution(), y, rtol=1e-8,
                                   atol=1e-8 * (1 + np.max(np.abs(y))))


def test_maximize_offset_matches_oracle(small_lp):
    dm = datamodel_from_lp(small_lp, maximize=True, offset=3.5)
    dm.set_objective_coefficients(-small_lp.c)
    sol = lpm.Solve(dm, settings(tol=REFINED_TOL))
    res, x, y, _ = O.solve(oracle_view(dm), tol=REFINED_TOL)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert rel(sol.get_primal_objective(), res["primal_obj"]) <= 1e-8
    assert rel(sol.get_primal_objective(), -small_lp.optimal_objective + 3.5) <= OBJ_RTOL
    np.testing.assert_allclose(sol.get_dual_solution(), y, atol=1e-7 * (1 + np.abs(y).max()))


def test_mixed_precision_reaches_tolerance(small_lp):
    """Mixed precision at 1e-6: Optimal with relative KKT <= 1e-6 on the returned FP64 point
    (reported and recomputed on the host); refined in FP64 to 1e-8: the constructed optimum and the
    oracle's 1e-8 objective within OBJ_RTOL."""
    dm = datamodel_from_lp(small_lp)
    sol = lpm.Solve(dm, settings(tol=1e-6, precision=1))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert relative_kkt(sol) <= 1e-6
    kkt = gen.kkt_relative_error(small_lp, sol.get_primal_solution(), sol.get_dual_solution())
    assert kkt["rel_primal"] <= 1e-6 and kkt["rel_gap"] <= 1e-6
    ref = lpm.Solve(dm, refined_settings())
    res8, _, _, _ = O.solve(small_lp, tol=REFINED_TOL)
    assert ref.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert relative_kkt(ref) <= REFINED_TOL
    assert rel(ref.get_primal_objective(), small_lp.optimal_objective) <= OBJ_RTOL
    assert rel(ref.get_primal_objective(), res8["primal_obj"]) <= OBJ_RTOL


def test_mixed_precision_refinement_reaches_1e8():
    """Mixed precision to 1e-6, then FP64 iterative refinement to 1e-8 on the original LP."""
    lp = gen.constructed_lp(2000, 5000, 8, seed=0)
    s = settings(tol=1e-6, precision=1)
    s.set_parameter(lpm.CUOPT_PDLP_REFINEMENT_PASSES, 8)
    s.set_parameter(lpm.CUOPT_PDLP_REFINEMENT_TOLERANCE, 1e-8)
    sol = lpm.Solve(datamodel_from_lp(lp), s)
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    st = sol.stats
    assert st["refinement_passes"] >= 1
    assert max(st["l2_relative_primal_residual"], st["l2_relative_dual_residual"],
               st["relative_gap"]) <= 1e-8
    kkt = gen.kkt_relative_error(lp, sol.get_primal_solution(), sol.get_dual_solution())
    assert kkt["rel_primal"] <= 1e-8 and kkt["rel_gap"] <= 1e-8
    assert rel(sol.get_primal_objective(), lp.optimal_objective) <= 1e-8


def _transposed_lp(lp, seed):
    """An LP whose matrix is lp's transpose, so that long rows become long columns (A^T sweeps)."""
    import scipy.sparse as sp
    rng = np.random.default_rng(seed)
    a = sp.csr_matrix((lp.val, lp.col_idx, lp.row_off), shape=(lp.m, lp.n)).T.tocsr()
    a.sort_indices()
    m, n = a.shape
    x0 = rng.uniform(-1.0, 1.0, n)
    ax = a @ x0
    eq = rng.random(m) < 0.4
    lo = np.where(eq, ax, ax - rng.uniform(0.0, 1.0, m))
    up = np.where(eq, ax, np.where(rng.random(m) < 0.5, np.inf, ax + rng.uniform(0.0, 1.0, m)))
    vlo = np.where(rng.random(n) < 0.1, -np.inf, -2.0)
    vup = np.where(np.isinf(vlo), np.inf, 2.0)
    return gen.LP(m, n, a.indptr.astype(np.int32), a.indices.astype(np.int32), a.data.copy(),
                  rng.standard_normal(n), lo, up, vlo, vup, x0, np.zeros(m), np.zeros(n), "transposed")


@pytest.mark.parametrize("transpose", [False, True])
def test_long_rows_and_columns_match_oracle(transpose):
    """Rows (or, transposed, columns) of up to ~1800 elements take the long-row path of the sweeps
    (one warp per row); the iterates still match the oracle after 10, 200 and 400 iterations."""
    lp = gen.skewed_lp(400, 3000, seed=7, cap=3000)
    if transpose:
        lp = _transposed_lp(lp, seed=8)
    lens = np.diff(lp.row_off) if not transpose else np.bincount(lp.col_idx, minlength=lp.n)
    assert lens.max() > 4 * 256
    dm = datamodel_from_lp(lp)
    for k in (10, 200, 400):
        sol = lpm.Solve(dm, settings(tol=1e-12, iteration_limit=k))
        res, x, y, _ = O.solve(lp, tol=1e-12, iteration_limit=k)
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        np.testing.assert_allclose(sol.get_primal_solution(), x, rtol=1e-8,
                                   atol=1e-8 * (1 + np.max(np.abs(x))))
        np.testing.assert_allclose(sol.get_dual_solution(), y, rtol=1e-8,
                                   atol=1e-8 * (1 + np.max(np.abs(y))))


def test_repeat_solves_bitwise_identical():
    """Two solves of the same LP give bit-identical iterates (every row sum and every reduction is
    combined in a fixed order)."""
    lp = gen.skewed_lp(400, 3000, seed=7, cap=3000)
    dm = datamodel_from_lp(lp)
    a = lpm.Solve(dm, settings(tol=1e-12, iteration_limit=300))
    b = lpm.Solve(dm, settings(tol=1e-12, iteration_limit=300))
    assert np.array_equal(a.get_primal_solution(), b.get_primal_solution())
    assert np.array_equal(a.get_dual_solution(), b.get_dual_solution())


def test_infeasibility_detection_matches_oracle(golden_dir):
    """Infeasible LPs end PrimalInfeasible at the same check as in the oracle."""
    from tests.helpers import infeasible_cases
    for name, lp in infeasible_cases(golden_dir):
        s = settings(tol=1e-6, iteration_limit=3000)
        s.set_parameter(lpm.CUOPT_INFEASIBILITY_DETECTION, True)
        sol = lpm.Solve(datamodel_from_lp(lp), s)
        res, _, _, _ = O.solve(lp, tol=1e-6, iteration_limit=3000, detect_infeasibility=True)
        assert int(sol.get_termination_status()) == res["status"] == 2, name
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"], name


def test_warm_start_matches_oracle(small_lp):
    """An initial primal / dual solution gives the oracle's iterates, and a good one converges in
    fewer iterations than the cold start."""
    rng = np.random.default_rng(3)
    x0 = small_lp.x_star + 1e-3 * rng.standard_normal(small_lp.n)
    y0 = small_lp.y_star + 1e-3 * rng.standard_normal(small_lp.m)
    dm = datamodel_from_lp(small_lp)
    dm.set_initial_primal_solution(x0)
    dm.set_initial_dual_solution(y0)
    for k in (10, 200):
        sol = lpm.Solve(dm, settings(tol=1e-12, iteration_limit=k))
        res, x, y, _ = O.solve(small_lp, tol=1e-12, iteration_limit=k, initial_primal=x0,
                               initial_dual=y0)
        assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
        assert np.max(np.abs(sol.get_primal_solution() - x)) <= ITERATE_RTOL * (1 + np.abs(x).max())
        assert np.max(np.abs(sol.get_dual_solution() - y)) <= ITERATE_RTOL * (1 + np.abs(y).max())
    warm = lpm.Solve(dm, settings(tol=1e-6))
    cold = lpm.Solve(datamodel_from_lp(small_lp), settings(tol=1e-6))
    assert warm.get_termination_status() == cold.get_termination_status() == 1
    assert warm.get_lp_stats()["nb_iterations"] < cold.get_lp_stats()["nb_iterations"]


@pytest.mark.parametrize("cfg", [(200, 500, 8, 11), (2000, 5000, 8, 0)])
def test_mixed_step_size_from_lanczos_matches_power_iteration(cfg):
    """Mixed precision takes sigma_max(A) from a Golub-Kahan-Lanczos bidiagonalisation; the step
    size agrees with the FP64 power iteration's to 1e-5 relative (the power iteration stops at a
    1e-4 residual, the FP32 matrix differs from the FP64 one in the 8th digit)."""
    m, n, k, seed = cfg
    dm = datamodel_from_lp(gen.constructed_lp(m, n, k, seed=seed))
    a = lpm.Solve(dm, settings(tol=1e-12, iteration_limit=0, precision=1))
    b = lpm.Solve(dm, settings(tol=1e-12, iteration_limit=0))
    assert rel(a.stats["step_size"], b.stats["step_size"]) <= 1e-5
    assert a.stats["power_iterations"] < b.stats["power_iterations"]


def _pcr_settings(tol, iteration_limit=None, on=True):
    s = settings(tol=tol, iteration_limit=iteration_limit)
    s.set_parameter(lpm.CUOPT_PER_CONSTRAINT_RESIDUAL, bool(on))
    return s


def test_per_constraint_residual_on_the_reference_point():
    """pdlp_test.cu:640-733: A = I (3 x 3), 0 <= Ax <= 0, c = 0; at x = (0.02, 0.03, 0.1) the
    per-constraint primal residual is exactly 0.1 while the l2 one is 0.106."""
    from types import SimpleNamespace
    z = np.zeros(3)
    lp = SimpleNamespace(row_off=np.arange(4), col_idx=np.arange(3), val=np.ones(3), c=z,
                         con_lo=z, con_up=z, var_lo=np.full(3, -np.inf), var_up=np.full(3, np.inf))
    dm = datamodel_from_lp(lp)
    dm.set_initial_primal_solution(np.array([0.02, 0.03, 0.1]))
    pcr = lpm.Solve(dm, _pcr_settings(0.1, iteration_limit=0))
    l2 = lpm.Solve(dm, _pcr_settings(0.1, iteration_limit=0, on=False))
    assert pcr.get_lp_stats()["primal_residual"] == 0.1
    assert l2.get_lp_stats()["primal_residual"] == np.sqrt(0.02 ** 2 + 0.03 ** 2 + 0.1 ** 2)


@pytest.mark.parametrize("scale_c", [1.0, 0.05])
def test_per_constraint_residual_matches_oracle(small_lp, scale_c):
    """The per-constraint criterion (CUOPT_PER_CONSTRAINT_RESIDUAL) stops at the oracle's
    iteration with the oracle's status and reported maxima.  With c as generated its dual form
    cannot be met (it subtracts rel * c_j with c_j's sign, as the reference does); with c scaled
    to |c_j| < 1 the solve ends Optimal."""
    from dataclasses import replace
    lp = replace(small_lp, c=small_lp.c * scale_c)
    tol = 1e-4
    sol = lpm.Solve(datamodel_from_lp(lp), _pcr_settings(tol, iteration_limit=3000))
    res, x, _, _ = O.solve(lp, tol=tol, iteration_limit=3000, per_constraint_residual=True)
    assert int(sol.get_termination_status()) == res["status"] == (4 if scale_c == 1.0 else 1)
    assert sol.get_lp_stats()["nb_iterations"] == res["iterations"]
    st = sol.get_lp_stats()
    assert abs(st["primal_residual"] - res["l2_primal"]) <= 1e-9 * (1e-3 + res["l2_primal"])
    assert abs(st["dual_residual"] - res["l2_dual"]) <= 1e-9 * (1e-3 + res["l2_dual"])
    assert np.max(np.abs(sol.get_primal_solution() - x)) <= ITERATE_RTOL * (1 + np.abs(x).max())


def test_per_constraint_residual_in_batches(small_lp):
    """cuOptBatchSolve solves the problems one at a time under the per-constraint criterion (the
    reference's batch is independent solves); climber batches reject it, as the reference's batch
    mode does (convergence_information.cu:393-395)."""
    from dataclasses import replace
    lp = replace(small_lp, c=small_lp.c * 0.05)
    s = _pcr_settings(1e-4, iteration_limit=3000)
    sols, _ = lpm.BatchSolve([datamodel_from_lp(lp), datamodel_from_lp(lp)], s)
    single = lpm.Solve(datamodel_from_lp(lp), s)
    for sol in sols:
        assert sol.get_termination_status() == single.get_termination_status()
        assert np.array_equal(sol.get_primal_solution(), single.get_primal_solution())
    climbers, _ = lpm.SolveClimbers(datamodel_from_lp(lp), [0], [lp.var_lo[0]], [lp.var_up[0]], s)
    assert climbers[0].get_error_status() == 4  # CUOPT_VALIDATION_ERROR


def test_mixed_precision_stall_continues_in_fp64():
    """Instance 458 of the 512-LP batch (2539 x 6347): its FP32 iterates stall with the relative gap near 1e-4 (after which
    the primal weight drifts), so a mixed solve continues in FP64 from its own state and ends
    Optimal at 1e-6 with the constructed optimum (refinement_passes = 1), as the FP64 solve does.
    In a mixed batch the stalled instance is solved again in FP64; the others stay mixed."""
    lp = gen.batch_instance(458)
    dm = datamodel_from_lp(lp)
    mixed = lpm.Solve(dm, settings(tol=1e-6, precision=1, time_limit=60))
    fp64 = lpm.Solve(dm, settings(tol=1e-6, precision=0, time_limit=60))
    assert mixed.get_termination_status() == fp64.get_termination_status() == \
        lpm.LPTerminationStatus.Optimal
    assert mixed.stats["refinement_passes"] == 1
    assert relative_kkt(mixed) <= 1e-6 and relative_kkt(fp64) <= 1e-6
    other = gen.batch_instance(0)
    sols, _ = lpm.BatchSolve([dm, datamodel_from_lp(other)],
                             settings(tol=1e-6, precision=1, time_limit=60))
    assert [int(s.get_termination_status()) for s in sols] == [1, 1]
    assert [s.stats["refinement_passes"] for s in sols] == [1, 0]
    assert max(relative_kkt(s) for s in sols) <= 1e-6
    # Refined to 1e-8, alone and in a batch: the constructed optima within OBJ_RTOL.
    ref = lpm.Solve(dm, refined_settings(time_limit=60))
    assert rel(ref.get_primal_objective(), lp.optimal_objective) <= OBJ_RTOL
    sols, _ = lpm.BatchSolve([dm, datamodel_from_lp(other)], refined_settings(time_limit=60))
    assert [s.stats["refinement_passes"] for s in sols] == [1, 1]
    assert max(relative_kkt(s) for s in sols) <= REFINED_TOL
    assert rel(sols[0].get_primal_objective(), lp.optimal_objective) <= OBJ_RTOL
    assert rel(sols[1].get_primal_objective(), other.optimal_objective) <= OBJ_RTOL


def test_problem_from_pinned_or_device_arrays_solves_identically(small_lp):
    """cuOptCreateRangedProblem from pinned host arrays (or device arrays) keeps a device copy made
    while the library copies the arrays, and cuOptSolve reads it instead of uploading: the result
    is bitwise that of the same problem created from pageable arrays."""
    import ctypes as C
    torch = pytest.importorskip("torch")
    from cuopt_b200._lib import lib
    L = lib()
    lp = small_lp
    arrays = [(lp.c, np.float64), (lp.row_off, np.int32), (lp.col_idx, np.int32),
              (lp.val, np.float64), (lp.con_lo, np.float64), (lp.con_up, np.float64),
              (lp.var_lo, np.float64), (lp.var_up, np.float64)]
    s = settings(tol=1e-8)._create()

    def solve(kind):
        if kind == "pageable":
            bufs = [np.ascontiguousarray(a, dtype=dt) for a, dt in arrays]
            ptrs = [C.c_void_p(b.ctypes.data) for b in bufs]
        else:
            bufs = [torch.as_tensor(np.ascontiguousarray(a, dtype=dt)) for a, dt in arrays]
            bufs = [b.pin_memory() if kind == "pinned" else b.cuda() for b in bufs]
            ptrs = [C.c_void_p(b.data_ptr()) for b in bufs]
        h, sol = C.c_void_p(), C.c_void_p()
        assert L.cuOptCreateRangedProblem(lp.m, lp.n, 1, 0.0, *ptrs, b"C" * lp.n, C.byref(h)) == 0
        del bufs  # the library holds its own copies
        assert L.cuOptSolve(h, s, C.byref(sol)) == 0
        x, y = np.zeros(lp.n), np.zeros(lp.m)
        L.cuOptGetPrimalSolution(sol, C.c_void_p(x.ctypes.data))
        L.cuOptGetDualSolution(sol, C.c_void_p(y.ctypes.data))
        status = C.c_int32()
        L.cuOptGetTerminationStatus(sol, C.byref(status))
        L.cuOptDestroySolution(C.byref(sol))
        L.cuOptDestroyProblem(C.byref(h))
        return status.value, x, y

    try:
        ref = solve("pageable")
        assert ref[0] == 1
        for kind in ("pinned", "device"):
            got = solve(kind)
            assert got[0] == ref[0]
            assert np.array_equal(got[1], ref[1]) and np.array_equal(got[2], ref[2])
    finally:
        L.cuOptDestroySolverSettings(C.byref(s))


def test_c_caller_solves(golden, golden_dir, tmp_path):
    """The plain C caller (tests/c_api/solve_lp.c) solves afiro from its MPS file and a ranged
    maximisation built from arrays: both Optimal, afiro at its golden objective, the ranged LP at
    its optimum 11."""
    import subprocess
    from tests.test_c_abi import _build_c_caller
    exe = _build_c_caller(tmp_path)
    res = subprocess.run([str(exe), str(golden_dir / "afiro_original.mps")], capture_output=True,
                         text=True, timeout=120)
    assert res.returncode == 0, res.stderr
    lines = {l.split()[0]: l.split()[1:] for l in res.stdout.splitlines()}
    assert int(lines["mps"][0]) == 1 and int(lines["ranged"][0]) == 1
    g = golden["afiro_objective"]
    assert rel(float(lines["mps"][1]), g["value"]) <= g["rel_tol"]
    assert abs(float(lines["ranged"][1]) - 11.0) <= 1e-5


def test_concurrent_solves_on_host_threads_match_sequential():
    """Solves of different problems may run on different host threads at once (the reference's
    threading contract: each problem on its own stream, cuopt_c_internal.hpp:20-29); each result is
    bitwise the sequential one."""
    from concurrent.futures import ThreadPoolExecutor
    lps = [gen.constructed_lp(300 + 100 * i, 800 + 200 * i, 8, seed=90 + i) for i in range(4)]
    s = settings(tol=1e-6)

    def run(lp):
        sol = lpm.Solve(datamodel_from_lp(lp), s)
        return (int(sol.get_termination_status()), sol.get_lp_stats()["nb_iterations"],
                sol.get_primal_solution(), sol.get_dual_solution())

    seq = [run(lp) for lp in lps]
    with ThreadPoolExecutor(max_workers=4) as ex:
        par = list(ex.map(run, lps))
    for a, b in zip(seq, par):
        assert a[0] == b[0] == 1 and a[1] == b[1]
        assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])


def test_c1_small_matches_oracle_fixture():
    """The 750k x 1.5M constructed LP (12M non-zeros, the 1M x 2M workload's generator): FP64 at
    1e-6 ends with the oracle's status, iteration count and objective (1e-9 relative;
    tests/golden/oracle_results.json); mixed precision at 1e-6 reaches relative KKT <= 1e-6; FP64
    at 1e-8 and mixed precision refined in FP64 to 1e-8 give the constructed optimum and the
    oracle's 1e-8 objective within OBJ_RTOL."""
    fx = oracle_results()["single"]["c1_small"]
    lp = gen.constructed_lp(fx["m"], fx["n"], 8, seed=fx["seed"])
    assert rel(lp.optimal_objective, fx["optimal_objective"]) <= 1e-12
    dm = datamodel_from_lp(lp)
    fp64 = lpm.Solve(dm, settings(tol=1e-6, time_limit=120))
    want = fx["1e-06"]
    assert int(fp64.get_termination_status()) == want["status"] == 1
    assert fp64.get_lp_stats()["nb_iterations"] == want["iterations"]
    assert rel(fp64.get_primal_objective(), want["primal_objective"]) <= 1e-9
    mixed = lpm.Solve(dm, settings(tol=1e-6, precision=1, time_limit=120))
    assert mixed.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert relative_kkt(mixed) <= 1e-6
    want8 = fx["1e-08"]
    for s in (settings(tol=REFINED_TOL, time_limit=120), refined_settings(time_limit=120)):
        sol = lpm.Solve(dm, s)
        assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
        assert relative_kkt(sol) <= REFINED_TOL
        assert rel(sol.get_primal_objective(), lp.optimal_objective) <= OBJ_RTOL
        assert rel(sol.get_primal_objective(), want8["primal_objective"]) <= OBJ_RTOL


@pytest.mark.parametrize("shape", [(2000, 5000, 8, 0), (60_000, 150_000, 8, 5)])
def test_tiled_sweeps_follow_sliced_sweeps(shape):
    """Mixed precision with the tiled sweeps forced on (pdlp_tiled_sweeps = 1: panels of the
    gathered vector in shared memory, FP32 row sums) against the sliced-ELL sweeps (0): after 150
    iterations (before the first restart decision) the iterates agree to 1e-4 relative to their
    scale (the two sum in different orders and precisions, so they drift apart at FP32 rounding),
    and both solves end Optimal at 1e-6 with relative KKT <= 1e-6; the autotuned default (-1) ends
    Optimal too."""
    m, n, k, seed = shape
    lp = gen.constructed_lp(m, n, k, seed=seed)
    dm = datamodel_from_lp(lp)
    runs = {}
    for tiled in (0, 1):
        s = settings(tol=1e-12, iteration_limit=150, precision=1)
        s.set_parameter(lpm.CUOPT_PDLP_TILED_SWEEPS, tiled)
        runs[tiled] = lpm.Solve(dm, s)
    a, b = runs[0], runs[1]
    assert a.get_lp_stats()["nb_iterations"] == b.get_lp_stats()["nb_iterations"] == 150
    for u, v in ((a.get_primal_solution(), b.get_primal_solution()),
                 (a.get_dual_solution(), b.get_dual_solution())):
        assert np.max(np.abs(u - v)) <= 1e-4 * (1.0 + np.max(np.abs(u)))
    for tiled in (0, 1, -1):
        s = settings(tol=1e-6, precision=1, time_limit=60)
        s.set_parameter(lpm.CUOPT_PDLP_TILED_SWEEPS, tiled)
        sol = lpm.Solve(dm, s)
        assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
        assert relative_kkt(sol) <= 1e-6
