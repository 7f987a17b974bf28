"""The C-ABI library on the CPU: it loads, exports every declared entry point, and its host logic
(problem objects, parameter registry, validation, MPS input/output) behaves like the reference's
cpp/src/pdlp/cuopt_c.cpp.  No GPU compute is called here."""
from __future__ import annotations

import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from cuopt_b200._lib import LIB_PATH, SIGNATURES, lib
from cuopt_b200 import linear_programming as lpm

ROOT = Path(__file__).resolve().parents[1]
HEADERS = [ROOT / "include" / "cuopt" / "linear_programming" / "cuopt_c.h", ROOT / "include" / "cuopt_b200.h"]


def declared_functions():
    names = set()
    for h in HEADERS:
        text = h.read_text()
        names |= set(re.findall(r"\b(cuOpt[A-Za-z0-9]+)\s*\(", text))
    return names


def exported_symbols():
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", str(LIB_PATH)], capture_output=True, text=True)
    return {ln.split()[-1] for ln in out.stdout.splitlines() if ln.strip()}


def test_library_exports_every_declared_symbol():
    declared = declared_functions()
    assert len(declared) >= 50
    missing = declared - exported_symbols()
    assert not missing, missing
    assert set(SIGNATURES) <= declared


def test_sizes_and_version():
    L = lib()
    assert L.cuOptGetFloatSize() == 8
    assert L.cuOptGetIntSize() == 4
    a, b, c = C.c_int32(), C.c_int32(), C.c_int32()
    assert L.cuOptGetVersion(C.byref(a), C.byref(b), C.byref(c)) == 0
    assert (a.value, b.value) == (26, 4)
    assert L.cuOptGetVersion(None, C.byref(b), C.byref(c)) == 1


def _settings():
    L = lib()
    h = C.c_void_p()
    assert L.cuOptCreateSolverSettings(C.byref(h)) == 0
    return h


def test_parameter_registry_matches_reference():
    """Names, defaults and ranges of solver_settings.cu:55-135; unknown names are rejected
    (c_api_tests.cpp:93)."""
    L = lib()
    h = _settings()
    v = C.c_double()
    assert L.cuOptGetFloatParameter(h, b"absolute_primal_tolerance", C.byref(v)) == 0
    assert v.value == 1e-4
    assert L.cuOptSetFloatParameter(h, b"absolute_primal_tolerance", 0.5) == 1  # above 1e-1
    assert L.cuOptSetParameter(h, b"bad_parameter_name", b"1") == 1
    i = C.c_int32()
    assert L.cuOptGetIntegerParameter(h, b"pdlp_solver_mode", C.byref(i)) == 0 and i.value == 4
    assert L.cuOptGetIntegerParameter(h, b"method", C.byref(i)) == 0 and i.value == 0
    assert L.cuOptGetIntegerParameter(h, b"presolve", C.byref(i)) == 0 and i.value == -1
    assert L.cuOptSetIntegerParameter(h, b"method", 4) == 1
    assert L.cuOptSetIntegerParameter(h, b"log_to_console", 0) == 0  # int -> bool fallback
    assert L.cuOptGetIntegerParameter(h, b"log_to_console", C.byref(i)) == 0 and i.value == 0
    assert L.cuOptSetParameter(h, b"time_limit", b"12.5") == 0
    buf = C.create_string_buffer(64)
    assert L.cuOptGetParameter(h, b"time_limit", 64, buf) == 0 and float(buf.value) == 12.5
    assert L.cuOptSetParameter(h, b"crossover", b"maybe") == 1
    assert L.cuOptSetParameter(h, b"pdlp_precision", b"1") == 0
    L.cuOptDestroySolverSettings(C.byref(h))
    assert h.value is None


def _problem(m=2, n=3, ranged=False, types=b"CCC"):
    L = lib()
    c = np.array([1.0, 2.0, 3.0])
    off = np.array([0, 2, 3], np.int32)
    idx = np.array([0, 2, 1], np.int32)
    val = np.array([1.0, -1.0, 2.0])
    lo = np.array([0.0, 0.0, 0.0])
    up = np.array([4.0, np.inf, 1.0])
    h = C.c_void_p()
    p = lambda a: C.c_void_p(a.ctypes.data)
    if ranged:
        cl, cu = np.array([-np.inf, 1.0]), np.array([3.0, 1.0])
        rc = L.cuOptCreateRangedProblem(m, n, -1, 2.5, p(c), p(off), p(idx), p(val), p(cl), p(cu),
                                        p(lo), p(up), types, C.byref(h))
    else:
        rhs = np.array([3.0, 1.0])
        rc = L.cuOptCreateProblem(m, n, 1, 0.0, p(c), p(off), p(idx), p(val), b"LE", p(rhs), p(lo),
                                  p(up), types, C.byref(h))
    return rc, h


def test_create_problem_and_getters():
    L = lib()
    rc, h = _problem()
    assert rc == 0
    m, n, nnz, s = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
    L.cuOptGetNumConstraints(h, C.byref(m))
    L.cuOptGetNumVariables(h, C.byref(n))
    L.cuOptGetNumNonZeros(h, C.byref(nnz))
    L.cuOptGetObjectiveSense(h, C.byref(s))
    assert (m.value, n.value, nnz.value, s.value) == (2, 3, 3, 1)
    sense = C.create_string_buffer(2)
    L.cuOptGetConstraintSense(h, sense)
    assert sense.raw == b"LE"
    vals, idx, off = np.zeros(3), np.zeros(3, np.int32), np.zeros(3, np.int32)
    L.cuOptGetConstraintMatrix(h, C.c_void_p(off.ctypes.data), C.c_void_p(idx.ctypes.data),
                               C.c_void_p(vals.ctypes.data))
    assert off.tolist() == [0, 2, 3] and idx.tolist() == [0, 2, 1] and vals.tolist() == [1, -1, 2]
    ismip = C.c_int32()
    L.cuOptIsMIP(h, C.byref(ismip))
    assert ismip.value == 0
    L.cuOptDestroyProblem(C.byref(h))
    assert h.value is None


def test_ranged_problem_bounds_roundtrip():
    L = lib()
    rc, h = _problem(ranged=True)
    assert rc == 0
    lo, up = np.zeros(2), np.zeros(2)
    L.cuOptGetConstraintLowerBounds(h, C.c_void_p(lo.ctypes.data))
    L.cuOptGetConstraintUpperBounds(h, C.c_void_p(up.ctypes.data))
    assert lo[0] == -np.inf and lo[1] == 1.0 and up.tolist() == [3.0, 1.0]
    off = C.c_double()
    L.cuOptGetObjectiveOffset(h, C.byref(off))
    assert off.value == 2.5
    L.cuOptDestroyProblem(C.byref(h))


def test_null_arguments_rejected():
    L = lib()
    assert L.cuOptCreateSolverSettings(None) == 1
    h = C.c_void_p()
    assert L.cuOptSolve(None, None, C.byref(h)) == 1
    assert L.cuOptGetTerminationStatus(None, None) == 1


def test_validation_and_mip_rejection_without_gpu():
    """Validation happens before any device work: crossing bounds -> Infeasible status, integer
    variables -> validation error (this library is LP only)."""
    L = lib()
    rc, h = _problem(types=b"CIC")
    s = _settings()
    sol = C.c_void_p()
    assert L.cuOptSolve(h, s, C.byref(sol)) == 4
    err = C.c_int32()
    L.cuOptGetErrorStatus(sol, C.byref(err))
    assert err.value == 4
    L.cuOptDestroySolution(C.byref(sol))
    L.cuOptDestroyProblem(C.byref(h))
    # crossing variable bounds
    p = lambda a: C.c_void_p(a.ctypes.data)
    c, off, idx, val = np.ones(1), np.array([0, 1], np.int32), np.zeros(1, np.int32), np.ones(1)
    rhs, lo, up = np.ones(1), np.array([2.0]), np.array([1.0])
    h2 = C.c_void_p()
    assert L.cuOptCreateProblem(1, 1, 1, 0.0, p(c), p(off), p(idx), p(val), b"E", p(rhs), p(lo),
                                p(up), b"C", C.byref(h2)) == 0
    assert L.cuOptSolve(h2, s, C.byref(sol)) == 0
    st = C.c_int32()
    L.cuOptGetTerminationStatus(sol, C.byref(st))
    assert st.value == 2  # CUOPT_TERIMINATION_STATUS_INFEASIBLE
    L.cuOptDestroySolution(C.byref(sol))
    L.cuOptDestroyProblem(C.byref(h2))
    L.cuOptDestroySolverSettings(C.byref(s))


def test_no_constraints_closed_form_without_gpu(golden, golden_dir):
    sol = lpm.Solve(lpm.ReadMps(golden_dir / "lp-model-no-constraints.mps"),
                    _py_settings(method=lpm.SolverMethod.Concurrent))
    assert sol.get_termination_status() == lpm.LPTerminationStatus.Optimal
    assert abs(sol.get_primal_objective() - golden["no_constraints_objective"]["value"]) <= 1e-12
    pd = lpm.Solve(lpm.ReadMps(golden_dir / "empty_matrix.mps"), _py_settings())
    assert int(pd.get_termination_status()) == golden["empty_matrix_pdlp_status"]["value"]


def _py_settings(method=lpm.SolverMethod.PDLP):
    s = lpm.SolverSettings()
    s.set_parameter(lpm.CUOPT_METHOD, int(method))
    s.set_parameter(lpm.CUOPT_LOG_TO_CONSOLE, False)
    return s


def test_mps_read_write_roundtrip(golden_dir, tmp_path):
    L = lib()
    h = C.c_void_p()
    assert L.cuOptReadProblem(str(golden_dir / "afiro_original.mps").encode(), C.byref(h)) == 0
    out = tmp_path / "afiro_rt.mps"
    assert L.cuOptWriteProblem(h, str(out).encode(), 0) == 0
    assert L.cuOptWriteProblem(h, str(out).encode(), 7) == 1
    a = lpm.ReadMps(golden_dir / "afiro_original.mps")
    b = lpm.ReadMps(out)
    assert a.n_constraints == b.n_constraints == 27 and a.n_variables == b.n_variables == 32
    np.testing.assert_array_equal(a.c, b.c)
    np.testing.assert_array_equal(a.A_offsets, b.A_offsets)
    np.testing.assert_array_equal(a.A_values, b.A_values)
    np.testing.assert_array_equal(a.constraint_lower_bounds, b.constraint_lower_bounds)
    np.testing.assert_array_equal(a.constraint_upper_bounds, b.constraint_upper_bounds)
    L.cuOptDestroyProblem(C.byref(h))
    assert L.cuOptReadProblem(b"/nonexistent/file.mps", C.byref(h)) == 2  # CUOPT_MPS_FILE_ERROR


def test_mps_ranges_and_bounds(golden_dir):
    dm = lpm.ReadMps(golden_dir / "good-mps-fixed-ranges.mps")
    assert dm.n_constraints > 0
    assert np.all(dm.constraint_lower_bounds <= dm.constraint_upper_bounds)
    dm2 = lpm.ReadMps(golden_dir / "lp-model-no-constraints.mps")
    assert dm2.variable_lower_bounds[0] == -np.inf and dm2.variable_upper_bounds[0] == 1.0
    assert dm2.maximize


def test_product_path_fails_loudly_without_library(tmp_path, monkeypatch):
    import cuopt_b200._lib as L
    monkeypatch.setattr(L, "_lib", None)
    monkeypatch.setattr(L, "LIB_PATH", tmp_path / "missing.so")
    with pytest.raises(ImportError):
        L.lib()


def _build_c_caller(tmp_path):
    """Compiles tests/c_api/solve_lp.c, a plain C caller of cuopt_c.h, against this library."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    root = Path(__file__).resolve().parents[1]
    exe = tmp_path / "solve_lp"
    cmd = [cc, "-std=c11", "-Wall", "-Werror", "-I", str(root / "include"),
           str(root / "tests" / "c_api" / "solve_lp.c"), "-o", str(exe),
           "-L", str(LIB_PATH.parent), "-lcuopt_b200", f"-Wl,-rpath,{LIB_PATH.parent}", "-lm"]
    res = subprocess.run(cmd, capture_output=True, text=True)
    assert res.returncode == 0, res.stderr
    return exe


def test_c_caller_compiles_and_links(tmp_path):
    """A C program written against cuopt_c.h builds and links against libcuopt_b200.so as it
    would against the reference's libcuopt."""
    assert _build_c_caller(tmp_path).exists()


def test_large_problem_checks_without_gpu():
    """The pre-solve checks split large arrays over host threads: a decreasing row offset near the
    end of 600 000 rows is a validation error, and a crossing bound near the end of 600 000
    variables (or of the ranged rows) ends Infeasible, all before any device work."""
    L = lib()
    s = _settings()
    p = lambda a: C.c_void_p(a.ctypes.data)
    m = n = 600_000

    def solve(off, vlo, vup, clo, cup):
        idx, val = np.arange(n, dtype=np.int32), np.ones(n)
        h, sol = C.c_void_p(), C.c_void_p()
        assert L.cuOptCreateRangedProblem(m, n, 1, 0.0, p(np.ones(n)), p(off), p(idx), p(val),
                                          p(clo), p(cup), p(vlo), p(vup), b"C" * n,
                                          C.byref(h)) == 0
        rc = L.cuOptSolve(h, s, C.byref(sol))
        st = C.c_int32()
        L.cuOptGetTerminationStatus(sol, C.byref(st))
        L.cuOptDestroySolution(C.byref(sol))
        L.cuOptDestroyProblem(C.byref(h))
        return rc, st.value

    off = np.arange(m + 1, dtype=np.int32)
    vlo, vup, clo, cup = np.zeros(n), np.ones(n), np.zeros(m), np.ones(m)
    bad_off = off.copy()
    bad_off[m - 3] = bad_off[m - 2] + 1  # offsets decrease at row m - 3
    assert solve(bad_off, vlo, vup, clo, cup)[0] == 4  # CUOPT_VALIDATION_ERROR
    bad_vup = vup.copy()
    bad_vup[n - 5] = -1.0
    assert solve(off, vlo, bad_vup, clo, cup) == (0, 2)  # Infeasible
    bad_cup = cup.copy()
    bad_cup[m - 7] = -1.0
    assert solve(off, vlo, vup, clo, bad_cup) == (0, 2)
    L.cuOptDestroySolverSettings(C.byref(s))


def test_without_a_gpu_every_solve_reports_a_cuda_error():
    """No CPU fallback: without a device, the single, batch, climber and strong-branching solves
    end with RuntimeError and a CUDA error message, and return no solution values."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cuopt_b200 import generators as gen
    from tests.helpers import datamodel_from_lp
    lp = gen.constructed_lp(50, 120, 4, seed=1)
    dm = datamodel_from_lp(lp)
    s = _py_settings()
    sols = [lpm.Solve(dm, s)]
    sols += lpm.BatchSolve([dm, dm], s)[0]
    sols += lpm.SolveClimbers(dm, [0, 1], [0.0, 0.0], [1.0, 1.0], s)[0]
    sols += lpm.BatchPDLPStrongBranching(dm, [2], [0.5] + [0.0] * (lp.n - 1), s)[0]
    assert len(sols) == 7
    for sol in sols:
        assert sol is not None
        assert sol.get_error_status() == lpm.ErrorStatus.RuntimeError
        assert "CUDA" in sol.get_error_message()
        assert sol.get_termination_status() == lpm.LPTerminationStatus.NoTermination
        assert not np.any(sol.get_primal_solution())


def test_large_problem_roundtrips_through_the_getters():
    """Arrays of several MiB (the library's huge-page blocks and threaded copies) come back from
    the getters exactly as given, also after freed blocks have been reused by a second problem."""
    L = lib()
    p = lambda a: C.c_void_p(a.ctypes.data)
    rng = np.random.default_rng(11)
    m, n, per_row = 400_000, 700_000, 3
    nnz = m * per_row
    for rep in range(2):
        off = np.arange(0, nnz + 1, per_row, dtype=np.int32)
        idx = rng.integers(0, n, nnz).astype(np.int32)
        val = rng.standard_normal(nnz)
        c, vlo, vup = rng.standard_normal(n), -rng.random(n), rng.random(n) + 1.0
        clo, cup = -rng.random(m) - rep, rng.random(m)
        h = C.c_void_p()
        assert L.cuOptCreateRangedProblem(m, n, -1, 0.5 * rep, p(c), p(off), p(idx), p(val),
                                          p(clo), p(cup), p(vlo), p(vup), b"C" * n,
                                          C.byref(h)) == 0
        got_off, got_idx = np.empty(m + 1, np.int32), np.empty(nnz, np.int32)
        got_val, got_c = np.empty(nnz), np.empty(n)
        got = {k: np.empty(len(v)) for k, v in
               (("clo", clo), ("cup", cup), ("vlo", vlo), ("vup", vup))}
        assert L.cuOptGetConstraintMatrix(h, p(got_off), p(got_idx), p(got_val)) == 0
        assert L.cuOptGetObjectiveCoefficients(h, p(got_c)) == 0
        assert L.cuOptGetConstraintLowerBounds(h, p(got["clo"])) == 0
        assert L.cuOptGetConstraintUpperBounds(h, p(got["cup"])) == 0
        assert L.cuOptGetVariableLowerBounds(h, p(got["vlo"])) == 0
        assert L.cuOptGetVariableUpperBounds(h, p(got["vup"])) == 0
        assert np.array_equal(got_off, off) and np.array_equal(got_idx, idx)
        assert np.array_equal(got_val, val) and np.array_equal(got_c, c)
        for k, v in (("clo", clo), ("cup", cup), ("vlo", vlo), ("vup", vup)):
            assert np.array_equal(got[k], v), k
        L.cuOptDestroyProblem(C.byref(h))


def test_reference_invalid_bounds_lp_is_infeasible():
    """c_api_test.c:1043-1175 (test_invalid_bounds, LP case): 0.2 <= x <= 0.5 as rows, variable
    bounds [1, 0]: cuOptSolve succeeds with termination status Infeasible, before any device work."""
    L = lib()
    p = lambda a: C.c_void_p(a.ctypes.data)
    off, idx, val = np.array([0, 1, 2], np.int32), np.zeros(2, np.int32), np.ones(2)
    clo, cup = np.array([0.2, -np.inf]), np.array([np.inf, 0.5])
    vlo, vup, c = np.array([1.0]), np.array([0.0]), np.array([2.0])
    h, s, sol = C.c_void_p(), _settings(), C.c_void_p()
    assert L.cuOptCreateRangedProblem(2, 1, 1, 0.0, p(c), p(off), p(idx), p(val), p(clo), p(cup),
                                      p(vlo), p(vup), b"C", C.byref(h)) == 0
    assert L.cuOptSolve(h, s, C.byref(sol)) == 0
    st = C.c_int32()
    assert L.cuOptGetTerminationStatus(sol, C.byref(st)) == 0
    assert st.value == 2  # CUOPT_TERIMINATION_STATUS_INFEASIBLE
    L.cuOptDestroySolution(C.byref(sol))
    L.cuOptDestroyProblem(C.byref(h))
    L.cuOptDestroySolverSettings(C.byref(s))
