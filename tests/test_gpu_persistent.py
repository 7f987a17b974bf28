"""GPU tests of the forms of the plain PDHG iterations (pdlp_persistent_iterations): CUDA-graph
replays, the persistent cooperative kernel and the cluster-resident kernel (small LPs).

Every form computes each row exactly as the graph-replayed sweeps do, so the expectation is exact:
solves with each form forced and chosen by timing return bit-identical iterates, iteration counts
and statuses, for single LPs (FP64 and mixed precision) and for block-diagonal batches.  The grid barrier between the sweeps is the only
wait in the kernel; its bounded wait is checked on its own (cuOptProbeGridBarrier): a barrier that
nothing can complete must end at its deadline with status 1, and the context must stay usable.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cuopt_b200 import _lib
from cuopt_b200 import generators as gen
from cuopt_b200 import linear_programming as lpm
from tests.helpers import datamodel_from_lp, settings

pytestmark = pytest.mark.gpu

GRAPHS, PERSISTENT, CLUSTER, AUTO = 0, 1, 2, -1


def _settings(form, **kw):
    s = settings(**kw)
    s.set_parameter(lpm.CUOPT_PDLP_PERSISTENT_ITERATIONS, form)
    return s


def _same(a, b):
    assert a.get_termination_status() == b.get_termination_status()
    assert a.stats["number_of_steps_taken"] == b.stats["number_of_steps_taken"]
    assert np.array_equal(a.get_primal_solution(), b.get_primal_solution())
    assert np.array_equal(a.get_dual_solution(), b.get_dual_solution())
    assert np.array_equal(a.get_reduced_cost(), b.get_reduced_cost())


@pytest.fixture(scope="module")
def lp_c0():
    """The 2,000 x 5,000 constructed LP (8 non-zeros per column)."""
    return gen.constructed_lp(2000, 5000, 8, seed=0)


@pytest.mark.parametrize("precision", [0, 1])
def test_persistent_matches_graphs(lp_c0, precision):
    """Every form of the plain iterations gives the same solve.  In FP64 the graphs-only setting
    (0) also runs the multi-kernel power iteration, the others the cluster power iteration of
    small LPs, so the comparison covers that the two give the same step size bit for bit."""
    dm = datamodel_from_lp(lp_c0)
    g = lpm.Solve(dm, _settings(GRAPHS, tol=1e-6, precision=precision))
    p = lpm.Solve(dm, _settings(PERSISTENT, tol=1e-6, precision=precision))
    c = lpm.Solve(dm, _settings(CLUSTER, tol=1e-6, precision=precision))
    a = lpm.Solve(dm, _settings(AUTO, tol=1e-6, precision=precision))
    assert g.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert g.stats["step_size"] == c.stats["step_size"]
    if precision == 0:
        assert g.stats["power_iterations"] == c.stats["power_iterations"] > 0
    _same(g, p)
    _same(g, c)
    _same(g, a)
    assert g.stats["plain_iteration_form"] == GRAPHS
    assert p.stats["plain_iteration_form"] == PERSISTENT
    assert c.stats["plain_iteration_form"] == CLUSTER
    assert p.stats["persistent_blocks"] > 0
    # The timed choice: every form timed, the fastest kept.
    us = [a.stats["plain_iteration_us_graphs"], a.stats["plain_iteration_us_persistent"],
          a.stats["plain_iteration_us_cluster"]]
    assert all(u > 0 for u in us)
    assert a.stats["plain_iteration_form"] == int(np.argmin(us))


def test_persistent_matches_graphs_at_iteration_limits(lp_c0):
    """Runs cut by an iteration limit inside a persistent launch's range end on the same iterate."""
    dm = datamodel_from_lp(lp_c0)
    for k in (7, 33, 250):
        g = lpm.Solve(dm, _settings(GRAPHS, tol=1e-12, iteration_limit=k))
        p = lpm.Solve(dm, _settings(PERSISTENT, tol=1e-12, iteration_limit=k))
        c = lpm.Solve(dm, _settings(CLUSTER, tol=1e-12, iteration_limit=k))
        assert g.get_termination_status() == lpm.LPTerminationStatus.IterationLimit
        _same(g, p)
        _same(g, c)


@pytest.mark.parametrize("precision", [0, 1])
def test_sweep_block_shapes_give_the_same_iterates(lp_c0, precision):
    """4, 8 and 16 warps per block and the timed choice (pdlp_sweep_warps_per_block) only group
    the same warps differently: bit-identical solves."""
    dm = datamodel_from_lp(lp_c0)
    sols = {}
    for w in (0, 4, 8, 16):
        s = _settings(GRAPHS, tol=1e-6, precision=precision)
        s.set_parameter(lpm.CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK, w)
        sols[w] = lpm.Solve(dm, s)
    for w in (4, 8, 16):
        assert sols[w].stats["sweep_warps_per_block_primal"] == w
        assert sols[w].stats["sweep_warps_per_block_dual"] == w
        _same(sols[8], sols[w])
    _same(sols[8], sols[0])
    assert sols[0].stats["sweep_warps_per_block_primal"] in (4, 8, 16)
    assert all(t > 0 for t in sols[0].stats["sweep_block_shape_ms"])
    lp = gen.skewed_lp(400, 3000, seed=7, cap=3000)  # long rows (warp per row) as well
    a, b = (lpm.Solve(datamodel_from_lp(lp), _settings(GRAPHS, tol=1e-6)) for _ in range(2))
    s = _settings(GRAPHS, tol=1e-6)
    s.set_parameter(lpm.CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK, 16)
    _same(a, lpm.Solve(datamodel_from_lp(lp), s))


def test_batch_sweep_block_shapes_give_the_same_iterates():
    lps = [gen.constructed_lp(m, int(2.5 * m), k, seed=90 + i)
           for i, (m, k) in enumerate([(300, 6), (1100, 10), (2500, 8)])]
    dms = [datamodel_from_lp(lp) for lp in lps]
    ref = None
    for w in (0, 4, 16):
        s = _settings(GRAPHS, tol=1e-6, precision=1)
        s.set_parameter(lpm.CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK, w)
        sols = lpm.BatchSolve(dms, s)[0]
        if ref is None:
            ref = sols
        else:
            for a, b in zip(ref, sols):
                _same(a, b)


def test_persistent_long_rows():
    """Long rows (warp per row) and sliced rows in the same persistent sweeps."""
    lp = gen.skewed_lp(400, 3000, seed=7, cap=3000)
    dm = datamodel_from_lp(lp)
    g = lpm.Solve(dm, _settings(GRAPHS, tol=1e-6))
    p = lpm.Solve(dm, _settings(PERSISTENT, tol=1e-6))
    c = lpm.Solve(dm, _settings(CLUSTER, tol=1e-6))
    _same(g, p)
    _same(g, c)
    assert c.stats["plain_iteration_form"] == CLUSTER


def test_cluster_kernels_without_the_matrix_copy():
    """4000 x 10000 in FP64: the power iteration's vectors fit in a cluster block's shared memory
    but its share of the matrices does not (the kernel reads them from global memory), and the
    plain iterations' vectors fit: both cluster kernels give the multi-kernel solve bit for bit."""
    lp = gen.constructed_lp(4000, 10000, 8, seed=17)
    dm = datamodel_from_lp(lp)
    g = lpm.Solve(dm, _settings(GRAPHS, tol=1e-6))
    c = lpm.Solve(dm, _settings(CLUSTER, tol=1e-6))
    assert g.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert c.stats["plain_iteration_form"] == CLUSTER
    assert g.stats["step_size"] == c.stats["step_size"]
    _same(g, c)


def test_cluster_form_falls_back_on_large_lps():
    """The cluster form needs both gathered vectors in one block's shared memory: for
    20 000 + 50 000 FP64 entries (560 KB) a solve that asks for it runs the graphs."""
    lp = gen.constructed_lp(20000, 50000, 8, seed=5)
    s = lpm.Solve(datamodel_from_lp(lp), _settings(CLUSTER, tol=1e-4, iteration_limit=50))
    assert s.stats["plain_iteration_form"] == GRAPHS


@pytest.mark.parametrize("precision", [0, 1])
def test_batch_persistent_matches_graphs(precision):
    lps = [gen.constructed_lp(m, int(2.5 * m), k, seed=70 + i)
           for i, (m, k) in enumerate([(200, 6), (1300, 12), (450, 8), (3000, 9), (800, 7)])]
    dms = [datamodel_from_lp(lp) for lp in lps]
    g = lpm.BatchSolve(dms, _settings(GRAPHS, tol=1e-6, precision=precision))[0]
    p = lpm.BatchSolve(dms, _settings(PERSISTENT, tol=1e-6, precision=precision))[0]
    a = lpm.BatchSolve(dms, _settings(AUTO, tol=1e-6, precision=precision))[0]
    for sg, sp, sa in zip(g, p, a):
        assert sg.get_termination_status() == lpm.LPTerminationStatus.Optimal
        _same(sg, sp)
        _same(sg, sa)
    assert all(s.stats["plain_iteration_form"] == PERSISTENT for s in p)
    assert all(s.stats["plain_iteration_form"] == GRAPHS for s in g)


def test_batch_timing_decisions_are_remembered():
    """A second solve of the same batch reuses the first one's timed decisions (sweep block shapes,
    form of the plain iterations per set of active instances) and reports the same timings; the
    iterates do not depend on them."""
    lps = [gen.constructed_lp(m, int(2.5 * m), k, seed=110 + i)
           for i, (m, k) in enumerate([(300, 6), (1700, 9), (900, 11)])]
    dms = [datamodel_from_lp(lp) for lp in lps]
    s = _settings(AUTO, tol=1e-6, precision=1)
    first = lpm.BatchSolve(dms, s)[0]
    again = lpm.BatchSolve(dms, s)[0]
    for a, b in zip(first, again):
        assert a.get_termination_status() == lpm.LPTerminationStatus.Optimal
        _same(a, b)
    for key in ("plain_iteration_form", "plain_iteration_us_graphs",
                "plain_iteration_us_persistent", "sweep_warps_per_block_primal",
                "sweep_warps_per_block_dual", "sweep_block_shape_ms"):
        assert first[0].stats[key] == again[0].stats[key], key
    assert first[0].stats["plain_iteration_us_graphs"] > 0
    assert all(t > 0 for t in first[0].stats["sweep_block_shape_ms"])


def _probe(blocks, rounds, unreachable, budget_ms):
    lib = _lib.lib()
    st, ms = _lib.cuopt_int_t(), C.c_double()
    rc = lib.cuOptProbeGridBarrier(blocks, rounds, unreachable, budget_ms, None, C.byref(st),
                                   C.byref(ms))
    return rc, st.value, ms.value


def test_grid_barrier_completes_and_costs():
    for blocks in (20, 148, 296):
        rc, st, ms = _probe(blocks, 2000, 0, 5000.0)
        assert rc == 0 and st == 0
        assert ms / 2000 < 0.05  # well under 50 us per barrier


def test_grid_barrier_deadline_ends_the_wait():
    """A barrier that cannot complete ends at its 50 ms deadline with status 1; the context stays
    usable (a solve afterwards succeeds)."""
    rc, st, ms = _probe(148, 1, 1, 50.0)
    assert rc == 0
    assert st == 1
    assert 45.0 <= ms < 2000.0
    rc, st, ms = _probe(148, 10, 0, 1000.0)
    assert rc == 0 and st == 0
    lp = gen.constructed_lp(200, 500, 8, seed=11)
    sol = lpm.Solve(datamodel_from_lp(lp), _settings(PERSISTENT, tol=1e-6))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal


def test_grid_barrier_rejects_oversized_grids():
    rc, _, _ = _probe(1_000_000, 1, 0, 10.0)
    assert rc == 1  # CUOPT_INVALID_ARGUMENT: more blocks than can be co-resident, nothing launched
