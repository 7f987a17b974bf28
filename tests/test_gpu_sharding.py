"""GPU test of the batch split across ranks: the ranks' subsets, each solved by its own
cuOptBatchSolve call (here one after another on one GPU, as the ranks of `ShardedBatchSolve` would
on theirs), give the unsplit batch's solutions.

Every instance of a batch follows its own single-LP trajectory, so moving it into a smaller batch
changes only the summation order of its reductions.  Tolerance: after the same number of
iterations, iterates agree to 2e-9 relative to the vector's magnitude (the batch test bounds each
batch's iterates to 1e-9 of the oracle's; two batches are within twice that).
"""
from __future__ import annotations

import numpy as np
import pytest

from cuopt_b200 import generators as gen
from cuopt_b200 import linear_programming as lpm
from cuopt_b200.sharding import ShardedBatchSolve, solve_shard
from tests.helpers import datamodel_from_lp, settings

pytestmark = pytest.mark.gpu

SPLIT_RTOL = 2e-9


@pytest.fixture(scope="module")
def models():
    lps = [gen.constructed_lp(m, int(2.5 * m), k, seed=50 + i)
           for i, (m, k) in enumerate([(200, 6), (1300, 12), (450, 8), (3000, 9)])]
    lps.append(gen.skewed_lp(400, 3000, seed=7, cap=3000))
    return [datamodel_from_lp(lp) for lp in lps]


def _close(a, b):
    return np.max(np.abs(a - b), initial=0.0) <= SPLIT_RTOL * (1 + np.abs(b).max(initial=0.0))


@pytest.mark.parametrize("world", [2, 3])
def test_shards_give_the_unsplit_batch_solutions(models, world):
    s = settings(tol=1e-12, iteration_limit=200)
    full, _ = lpm.BatchSolve(models, s)
    got = [None] * len(models)
    for rank in range(world):
        idx, sols, _ = solve_shard(models, rank, world, s)
        for i, sol in zip(idx, sols):
            got[i] = sol
    for a, b in zip(got, full):
        assert a is not None
        assert a.get_termination_status() == b.get_termination_status() == \
            lpm.LPTerminationStatus.IterationLimit
        assert a.get_lp_stats()["nb_iterations"] == b.get_lp_stats()["nb_iterations"]
        assert _close(a.get_primal_solution(), b.get_primal_solution())
        assert _close(a.get_dual_solution(), b.get_dual_solution())
        assert _close(a.get_reduced_cost(), b.get_reduced_cost())


def test_without_a_process_group_it_is_the_batch(models):
    s = settings(tol=1e-12, iteration_limit=100)
    a, _ = ShardedBatchSolve(models, s)
    b, _ = lpm.BatchSolve(models, s)
    for sa, sb in zip(a, b):
        assert np.array_equal(sa.get_primal_solution(), sb.get_primal_solution())
        assert np.array_equal(sa.get_dual_solution(), sb.get_dual_solution())
