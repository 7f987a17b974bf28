"""CPU tests of bench.py's replica path (N > 1): two gloo ranks on 127.0.0.1.

Each rank times its own copy of the workload (replicas only: no data-path collective); the job's
time is the max over ranks and the aggregate value counts every rank's units.  The reference arm
runs on rank 0 only.
"""
from __future__ import annotations

import os
import socket

import pytest

torch = pytest.importorskip("torch")
mp = pytest.importorskip("torch.multiprocessing")


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench
    r = bench.Replicas(world, rank, None, "gloo", timeout_s=60.0)
    r.barrier()
    t = r.max(10.0 * (rank + 1))          # per-rank times 10 and 20
    r.barrier()
    out.put((rank, t))
    r.close()


def test_two_replicas_take_the_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got == {0: 20.0, 1: 20.0}
    # The bench's whole-job value: world x units / the slowest rank's time.
    world, ms = 2, got[0]
    assert world * 1000.0 / ms == 100.0


def test_single_replica_needs_no_process_group():
    import bench
    r = bench.Replicas(1, 0, None, "gloo")
    r.barrier()
    assert r.max(3.5) == 3.5
    r.close()


def test_reference_arm_runs_on_rank_zero_only(monkeypatch):
    import bench
    monkeypatch.setenv("RANK", "1")
    called = []
    monkeypatch.setattr(bench, "make_lp", lambda *a: called.append(a))
    assert bench.run_reference(None) is None
    assert not called


def test_reference_arm_prints_one_contract_line():
    """`bench.py --impl reference` prints one JSON line with the contract's keys, on the small
    2000 x 5000 workload (whole FP64 oracle solves on the host, the Optimal status and the
    objective error against the constructed optimum recorded)."""
    import json
    import subprocess
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    res = subprocess.run([sys.executable, str(root / "bench.py"), "--impl", "reference",
                          "--config", "c0", "--steps", "2", "--warmup", "1",
                          "--reference-seconds", "60"], capture_output=True, text=True, timeout=300,
                         cwd=root, env={**os.environ, "RANK": "0", "WORLD_SIZE": "1"})
    assert res.returncode == 0, res.stderr
    lines = [l for l in res.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
              "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
              "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0 and d["higher_is_better"] is True
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert "2000x5000" in d["config"]["workload"]
    assert 1 <= d["steps"] <= 2 and d["steps_requested"] == 2 and d["dtype"] == "f64"
    assert d["status"] == 1 and d["objective_rel_error"] < 1e-4
