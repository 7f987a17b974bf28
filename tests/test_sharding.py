"""CPU tests of the batch split across ranks (cuopt_b200.sharding): the work-balanced partition,
and ShardedBatchSolve's collection over two gloo ranks on 127.0.0.1.

The solve itself needs a GPU, so the gloo ranks replace `BatchSolve` by a stand-in that records
which rank solved which instance; the split, the collection in input order, the max over ranks of
the batch time and the error path are what these tests check.  The GPU test of the split (the
shards' solutions match the unsplit batch's) is in test_gpu_sharding.py.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest

from cuopt_b200 import generators as gen
from cuopt_b200 import linear_programming as lpm
from cuopt_b200.sharding import instance_work, partition_instances
from tests.helpers import datamodel_from_lp

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


@pytest.mark.parametrize("parts", [1, 2, 3, 8])
def test_partition_covers_every_instance_once_and_balances(parts):
    rng = np.random.default_rng(parts)
    work = rng.integers(1_000, 100_000, size=517)
    shards = partition_instances(work, parts)
    assert len(shards) == parts
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(len(work)))
    for s in shards:
        assert s == sorted(s)
    loads = [int(work[s].sum()) for s in shards]
    assert max(loads) <= work.sum() / parts + work.max()
    assert partition_instances(work, parts) == shards          # a pure function of the sizes


def test_partition_edge_cases():
    assert partition_instances([], 3) == [[], [], []]
    assert partition_instances([5, 5], 4) == [[0], [1], [], []]
    # Heaviest first onto the least-loaded part, ties to the lower part and lower index.
    assert partition_instances([1, 9, 4, 4, 2], 2) == [[0, 1], [2, 3, 4]]
    assert partition_instances([3, 3, 3, 3], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition_instances([1], 0)
    with pytest.raises(ValueError):
        partition_instances([-1], 1)


def test_instance_work_counts_nonzeros_and_vectors():
    lp = gen.constructed_lp(200, 500, 6, seed=1)
    dm = datamodel_from_lp(lp)
    assert instance_work(dm) == lp.nnz + lp.m + lp.n


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _models(count, shift=0):
    out = []
    for i in range(count):
        m = 20 + 7 * ((i * 5 + shift) % 9)
        lp = gen.constructed_lp(m, 2 * m, 3, seed=100 + i)
        out.append(datamodel_from_lp(lp))
    return out


def _rank(rank, world, port, mode, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    import torch.distributed as dist

    from cuopt_b200 import sharding
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        def fake_batch(dms, settings=None):
            if mode == "error" and rank == 1:
                raise lpm.CuOptError(5, "cuOptBatchSolve")
            sols = [lpm.Solution(dm.c.copy(), np.zeros(dm.n_constraints), np.zeros(dm.n_variables),
                                 1, 0, "", {"number_of_steps_taken": rank}) for dm in dms]
            return sols, 0.5 * (rank + 1)

        lpm.BatchSolve = fake_batch
        dms = _models(7, shift=rank if mode == "mismatch" else 0)
        try:
            sols, t = sharding.ShardedBatchSolve(dms, None, collect=(mode != "local"))
            res = ("ok", [None if s is None else (s.primal_solution.tolist(),
                                                 s.stats["number_of_steps_taken"]) for s in sols],
                   t, [dm.c.tolist() for dm in dms])
        except Exception as e:
            res = ("raised", type(e).__name__, str(e))
        out.put((rank, res))
    finally:
        dist.destroy_process_group()


def _run(mode, world=2):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return got


def test_two_ranks_collect_every_solution_in_input_order():
    got = _run("collect")
    work = [instance_work(dm) for dm in _models(7)]
    shards = partition_instances(work, 2)
    owner = {i: r for r, s in enumerate(shards) for i in s}
    assert shards[0] and shards[1]
    for rank in (0, 1):
        status, sols, t, cs = got[rank]
        assert status == "ok"
        assert t == 1.0                                        # the slower rank's batch time
        for i, (x, solved_on) in enumerate(sols):
            assert x == cs[i]                                  # instance i's own solution
            assert solved_on == owner[i]                       # solved once, by its owner
    assert got[0][1] == got[1][1]


def test_without_collect_each_rank_keeps_its_own_solutions():
    got = _run("local")
    shards = partition_instances([instance_work(dm) for dm in _models(7)], 2)
    for rank in (0, 1):
        status, sols, t, _ = got[rank]
        assert status == "ok" and t == 1.0
        assert [i for i, s in enumerate(sols) if s is not None] == shards[rank]
        assert all(s[1] == rank for s in sols if s is not None)


def test_an_error_on_one_rank_is_raised_on_every_rank():
    got = _run("error")
    for rank in (0, 1):
        status, name, msg = got[rank]
        assert status == "raised" and name == "RuntimeError"
        assert "rank 1" in msg and "cuOptBatchSolve" in msg


def test_different_lists_on_the_ranks_are_rejected_everywhere():
    got = _run("mismatch")
    for rank in (0, 1):
        status, name, msg = got[rank]
        assert status == "raised" and name == "ValueError"


def test_without_a_process_group_it_is_batch_solve(monkeypatch):
    from cuopt_b200 import sharding
    calls = []
    monkeypatch.setattr(lpm, "BatchSolve", lambda dms, s=None: calls.append(len(dms)) or ([], 0.0))
    sharding.ShardedBatchSolve(_models(3))
    assert calls == [3]
