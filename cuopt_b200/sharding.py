"""Batches of independent LPs split across GPUs, one process per GPU.

The instances of a batch (the reference's `BatchSolve`, python/cuopt/cuopt/linear_programming/
solver/solver.py:109-160, and `cuOptBatchSolve`) are independent: nothing in one instance's PDHG
iterations reads another's.  So a batch shards across ranks with no exchange inside the solve:
rank r solves its own subset with one `cuOptBatchSolve` call on its own GPU, and the solutions are
collected on the host afterwards.

Subsets are balanced by work.  A PDHG iteration of one instance reads its non-zeros and its
vectors, so an instance's work per iteration is taken as nnz + m + n; subsets are filled greedily,
heaviest instance first, each onto the least-loaded rank (ties to the lower rank).  The split is a
pure function of the instances' sizes, so every rank computes the same one without communicating.
Iteration counts differ from instance to instance and are not known beforehand, so the balance is
of work per iteration, not of time.
"""
from __future__ import annotations

import hashlib

import numpy as np

from . import linear_programming as lpm

__all__ = ["instance_work", "partition_instances", "solve_shard", "ShardedBatchSolve"]


def instance_work(data_model) -> int:
    """Work of one PDHG iteration of the instance, in elements read: nnz + m + n."""
    return (len(data_model.get_constraint_matrix_values()) + data_model.n_constraints
            + data_model.n_variables)


def partition_instances(work, parts: int) -> list[list[int]]:
    """Splits instances with the given work into `parts` index lists, each in ascending order.

    Greedy longest-processing-time: the heaviest instance first (ties by index), each onto the
    part with the least work so far (ties to the lower part).  No part's work exceeds the mean by
    more than the heaviest single instance.  Parts beyond the instance count are empty.
    """
    parts = int(parts)
    if parts < 1:
        raise ValueError(f"parts must be >= 1 (got {parts})")
    w = np.asarray(work, dtype=np.int64).reshape(-1)
    if (w < 0).any():
        raise ValueError("instance work must be non-negative")
    order = sorted(range(len(w)), key=lambda i: (-int(w[i]), i))
    load = [0] * parts
    out: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        p = min(range(parts), key=lambda r: (load[r], r))
        out[p].append(i)
        load[p] += int(w[i])
    return [sorted(s) for s in out]


def _fingerprint(work) -> str:
    return hashlib.sha256(np.asarray(work, dtype=np.int64).tobytes()).hexdigest()


def solve_shard(data_model_list, rank: int, world_size: int,
                solver_settings: lpm.SolverSettings | None = None):
    """Solves rank `rank`'s subset of the batch on the current GPU with one cuOptBatchSolve call.

    Returns (indices, solutions, seconds): the subset's positions in `data_model_list` (ascending),
    their solutions in that order and the batch call's time (0.0 for an empty subset, which makes
    no call).
    """
    if not 0 <= rank < world_size:
        raise ValueError(f"rank {rank} outside a world of {world_size}")
    shards = partition_instances([instance_work(dm) for dm in data_model_list], world_size)
    mine = shards[rank]
    if not mine:
        return mine, [], 0.0
    sols, seconds = lpm.BatchSolve([data_model_list[i] for i in mine], solver_settings)
    return mine, sols, seconds


def ShardedBatchSolve(data_model_list, solver_settings: lpm.SolverSettings | None = None,
                      group=None, collect: bool = True):
    """`BatchSolve` over all ranks of a torch.distributed process group, one GPU per rank.

    Every rank passes the same list of LPs (checked: the call fails on every rank when the ranks'
    instance sizes differ) and solves its work-balanced subset (`partition_instances`) on its own
    device.  Returns (solutions, seconds) like `BatchSolve`: the solutions in input order and the
    longest of the ranks' batch times.  With `collect` the solutions of all ranks are gathered on
    every rank (host objects, after the solves); without it the entries solved on other ranks are
    None.  An error on any rank is raised on every rank after the exchange, so no rank is left
    waiting in a collective.  Without an initialised process group this is `BatchSolve`.

    The solve runs on the calling thread's current CUDA device; with an NCCL group, set it to the
    rank's own GPU first (`torch.cuda.set_device`), which the object collectives also need.
    """
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return lpm.BatchSolve(data_model_list, solver_settings)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    work = [instance_work(dm) for dm in data_model_list]
    prints = [None] * world
    dist.all_gather_object(prints, _fingerprint(work), group=group)
    if len(set(prints)) != 1:
        raise ValueError("ShardedBatchSolve: the ranks were given different lists of LPs")

    error = None
    try:
        mine, sols, seconds = solve_shard(data_model_list, rank, world, solver_settings)
    except Exception as e:  # reported to every rank below
        mine, sols, seconds = [], [], 0.0
        error = f"{type(e).__name__}: {e}"
    local = (mine, sols if collect else [], seconds, error)
    gathered = [None] * world
    dist.all_gather_object(gathered, local, group=group)
    failed = [(r, g[3]) for r, g in enumerate(gathered) if g[3] is not None]
    if failed:
        raise RuntimeError("ShardedBatchSolve failed on " +
                           "; ".join(f"rank {r}: {msg}" for r, msg in failed))

    out = [None] * len(data_model_list)
    for idx, s in ([(g[0], g[1]) for g in gathered] if collect else [(mine, sols)]):
        for i, sol in zip(idx, s):
            out[i] = sol
    return out, max(g[2] for g in gathered)
