"""GPU test of cuOptComputeKKTErrorsNoAlloc, the KKT evaluation that allocates no device memory.

It must report, for the point cuOptSolveDevice returns, the residuals, objectives and gap that
cuOptSolveDevice itself reports in its statistics, on two calls in a row (its static scratch is
cleared on every call); flag malformed column indices and row offsets with NaN outputs and a
count, and clear that count on the next call; and leave the device's free memory unchanged.
Tolerances: residual norms and relative errors within 1e-7 relative (summation order and the
atomic A^T y accumulation differ), objectives within 1e-10 relative, the gap within
1e-10 x (1 + |primal| + |dual|).

The file name keeps it last in collection order, after the tests that use the allocating paths.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cuopt_b200 import generators as gen
from cuopt_b200._lib import PDLPStatistics, lib

pytestmark = pytest.mark.gpu

MAX_COLS = 1 << 19
RES_RTOL = 1e-7
OBJ_RTOL = 1e-10


def _settings(L, tol, iteration_limit=None):
    h = C.c_void_p()
    assert L.cuOptCreateSolverSettings(C.byref(h)) == 0
    for name in ("absolute_primal_tolerance", "relative_primal_tolerance", "absolute_dual_tolerance",
                 "relative_dual_tolerance", "absolute_gap_tolerance", "relative_gap_tolerance"):
        assert L.cuOptSetFloatParameter(h, name.encode(), tol) == 0
    assert L.cuOptSetParameter(h, b"log_to_console", b"false") == 0
    if iteration_limit is not None:
        assert L.cuOptSetIntegerParameter(h, b"iteration_limit", iteration_limit) == 0
    return h


def _device(lp, torch, c=None):
    dev = torch.device("cuda", 0)
    t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), device=dev, dtype=dt)
    return {"c": t(lp.c if c is None else c, torch.float64), "off": t(lp.row_off, torch.int32),
            "idx": t(lp.col_idx, torch.int32), "val": t(lp.val, torch.float64),
            "lo": t(lp.con_lo, torch.float64), "up": t(lp.con_up, torch.float64),
            "vlo": t(lp.var_lo, torch.float64), "vup": t(lp.var_up, torch.float64),
            "x": torch.empty(lp.n, device=dev, dtype=torch.float64),
            "y": torch.empty(lp.m, device=dev, dtype=torch.float64),
            "rc": torch.empty(lp.n, device=dev, dtype=torch.float64)}


def _p(t):
    return C.c_void_p(t.data_ptr())


def _solve(L, torch, d, lp, sense, offset, settings):
    st, status = PDLPStatistics(), C.c_int32()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.cuOptSolveDevice(lp.m, lp.n, sense, offset, _p(d["c"]), _p(d["off"]), _p(d["idx"]),
                            _p(d["val"]), _p(d["lo"]), _p(d["up"]), _p(d["vlo"]), _p(d["vup"]),
                            settings, stream, _p(d["x"]), _p(d["y"]), _p(d["rc"]), C.byref(st),
                            C.byref(status))
    assert rc == 0
    torch.cuda.synchronize()
    return st, status.value


def _no_alloc(L, torch, d, lp, sense, offset, n=None, out=None, idx=None, off=None):
    if out is None:
        out = torch.full((9,), -1.0, device="cuda", dtype=torch.float64)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.cuOptComputeKKTErrorsNoAlloc(lp.m, lp.n if n is None else n, sense, offset, _p(d["c"]),
                                        _p(d["off"] if off is None else off),
                                        _p(d["idx"] if idx is None else idx), _p(d["val"]),
                                        _p(d["lo"]), _p(d["up"]), _p(d["x"]), _p(d["y"]),
                                        _p(d["rc"]), stream, _p(out))
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def _check(st, out):
    assert out[8] == 0.0
    for got, want in ((out[0], st.l2_primal_residual), (out[1], st.l2_dual_residual),
                      (out[5], st.l2_relative_primal_residual),
                      (out[6], st.l2_relative_dual_residual), (out[7], st.relative_gap)):
        assert abs(got - want) <= RES_RTOL * abs(want) + 1e-14, (got, want)
    for got, want in ((out[2], st.primal_objective), (out[3], st.dual_objective)):
        assert abs(got - want) <= OBJ_RTOL * max(1.0, abs(want)), (got, want)
    scale = 1.0 + abs(st.primal_objective) + abs(st.dual_objective)
    assert abs(out[4] - st.gap) <= 1e-10 * scale


@pytest.mark.parametrize("sense,offset,iteration_limit", [(1, 0.0, None), (1, 0.0, 300),
                                                          (-1, 2.5, None)])
def test_no_alloc_matches_solver_statistics(sense, offset, iteration_limit):
    torch = pytest.importorskip("torch")
    L = lib()
    lp = gen.constructed_lp(2000, 5000, 8, seed=0)
    d = _device(lp, torch, c=lp.c if sense == 1 else -lp.c)
    s = _settings(L, 1e-6, iteration_limit)
    try:
        st, status = _solve(L, torch, d, lp, sense, offset, s)
    finally:
        L.cuOptDestroySolverSettings(C.byref(s))
    assert status == (1 if iteration_limit is None else 4)
    rc1, out1 = _no_alloc(L, torch, d, lp, sense, offset)
    rc2, out2 = _no_alloc(L, torch, d, lp, sense, offset)
    assert rc1 == 0 and rc2 == 0
    _check(st, out1)
    _check(st, out2)


def test_no_alloc_rejects_too_many_variables():
    torch = pytest.importorskip("torch")
    L = lib()
    lp = gen.constructed_lp(200, 500, 8, seed=1)
    d = _device(lp, torch)
    rc, out = _no_alloc(L, torch, d, lp, 1, 0.0, n=MAX_COLS + 1)
    assert rc == 1  # CUOPT_INVALID_ARGUMENT, before any device work
    assert np.all(out == -1.0)


def _solved_c0(L, torch):
    lp = gen.constructed_lp(2000, 5000, 8, seed=0)
    d = _device(lp, torch)
    s = _settings(L, 1e-6)
    try:
        st, status = _solve(L, torch, d, lp, 1, 0.0, s)
    finally:
        L.cuOptDestroySolverSettings(C.byref(s))
    assert status == 1
    return lp, d, st


def test_no_alloc_flags_bad_column_then_clears():
    """A column index equal to n is counted and skipped (NaN outputs); the next call with the
    original indices starts from a cleared count and gives the solver's statistics again."""
    torch = pytest.importorskip("torch")
    L = lib()
    lp, d, st = _solved_c0(L, torch)
    bad_idx = d["idx"].clone()
    bad_idx[123] = lp.n
    rc, out = _no_alloc(L, torch, d, lp, 1, 0.0, idx=bad_idx)
    assert rc == 0
    assert out[8] == 1.0
    assert np.all(np.isnan(out[:8]))
    rc, out = _no_alloc(L, torch, d, lp, 1, 0.0)
    assert rc == 0
    _check(st, out)


def test_no_alloc_flags_decreasing_row_offsets():
    """Row 5 given an end offset below its start is counted and skipped; every access stays inside
    the arrays (the neighbouring rows only grow or shrink within them)."""
    torch = pytest.importorskip("torch")
    L = lib()
    lp, d, st = _solved_c0(L, torch)
    off = d["off"].clone()
    assert int(off[5]) > 0
    off[6] = off[5] - 1
    rc, out = _no_alloc(L, torch, d, lp, 1, 0.0, off=off)
    assert rc == 0
    assert out[8] == 1.0
    assert np.all(np.isnan(out[:8]))
    rc, out = _no_alloc(L, torch, d, lp, 1, 0.0)
    assert rc == 0
    _check(st, out)


def test_no_alloc_leaves_free_memory_unchanged():
    """After a first call (which loads the library's device code and its static scratch), further
    calls take no device memory: the device's free bytes are the same before and after them."""
    torch = pytest.importorskip("torch")
    L = lib()
    lp, d, st = _solved_c0(L, torch)
    out = torch.full((9,), -1.0, device="cuda", dtype=torch.float64)
    rc, _ = _no_alloc(L, torch, d, lp, 1, 0.0, out=out)
    assert rc == 0
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        rc, res = _no_alloc(L, torch, d, lp, 1, 0.0, out=out)
        assert rc == 0
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    _check(st, res)
