"""MPS input through cuOptReadProblem, against the reference's MPS parser tests
(cpp/libmps_parser/tests/mps_parser_test.cpp) read in free format, which is how the reference's
cuOptReadProblem parses (cpp/src/pdlp/cuopt_c.cpp:103-107).  CPU only: reading a problem and its
getters do no device work.  Values are compared exactly, as the reference's tests do."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from cuopt_b200._lib import lib

INF = float("inf")


def _path(golden_dir, name):
    p = golden_dir / "mps" / name
    return p if p.exists() else golden_dir / name


def _num(v):
    return {"inf": INF, "-inf": -INF}.get(v, v) if isinstance(v, str) else v


class _Problem:
    def __init__(self, path):
        self.L = lib()
        self.h = C.c_void_p()
        self.rc = self.L.cuOptReadProblem(str(path).encode(), C.byref(self.h))

    def __enter__(self):
        return self

    def __exit__(self, *a):
        if self.h:
            self.L.cuOptDestroyProblem(C.byref(self.h))

    def _int(self, fn):
        v = C.c_int32()
        assert fn(self.h, C.byref(v)) == 0
        return v.value

    def sizes(self):
        return (self._int(self.L.cuOptGetNumConstraints), self._int(self.L.cuOptGetNumVariables),
                self._int(self.L.cuOptGetNumNonZeros))

    def _vec(self, fn, n, dtype=np.float64):
        out = np.empty(n, dtype)
        assert fn(self.h, C.c_void_p(out.ctypes.data)) == 0
        return out

    def matrix(self):
        m, _, nnz = self.sizes()
        off, idx, val = np.empty(m + 1, np.int32), np.empty(nnz, np.int32), np.empty(nnz)
        assert self.L.cuOptGetConstraintMatrix(self.h, C.c_void_p(off.ctypes.data),
                                               C.c_void_p(idx.ctypes.data),
                                               C.c_void_p(val.ctypes.data)) == 0
        return off, idx, val

    def c(self):
        return self._vec(self.L.cuOptGetObjectiveCoefficients, self.sizes()[1])

    def rhs(self):
        return self._vec(self.L.cuOptGetConstraintRightHandSide, self.sizes()[0])

    def sense(self):
        buf = C.create_string_buffer(max(self.sizes()[0], 1))
        assert self.L.cuOptGetConstraintSense(self.h, buf) == 0
        return buf.raw[:self.sizes()[0]].decode()

    def bounds(self):
        n = self.sizes()[1]
        return (self._vec(self.L.cuOptGetVariableLowerBounds, n),
                self._vec(self.L.cuOptGetVariableUpperBounds, n))

    def row_bounds(self):
        m = self.sizes()[0]
        return (self._vec(self.L.cuOptGetConstraintLowerBounds, m),
                self._vec(self.L.cuOptGetConstraintUpperBounds, m))

    def offset(self):
        v = C.c_double()
        assert self.L.cuOptGetObjectiveOffset(self.h, C.byref(v)) == 0
        return v.value


def test_bad_files_are_rejected(golden, golden_dir):
    """mps_parser_test.cpp:46-57, 286-301, 532-550: every bad file is a parse error
    (CUOPT_MPS_PARSE_ERROR), with no problem handle."""
    for name in golden["mps_parser"]["rejected"]:
        with _Problem(_path(golden_dir, name)) as p:
            assert p.rc == 3, name
            assert not p.h, name


def test_missing_file_is_a_file_error(golden_dir):
    """c_api_tests.cpp:100 (test_missing_file): CUOPT_MPS_FILE_ERROR."""
    with _Problem(golden_dir / "mps" / "no-such-file.mps") as p:
        assert p.rc == 2


def test_good_1_and_its_variants(golden, golden_dir):
    g = golden["mps_parser"]["good-1"]
    for name in g["files"]:
        with _Problem(_path(golden_dir, name)) as p:
            assert p.rc == 0, name
            off, idx, val = p.matrix()
            assert off.tolist() == g["row_offsets"] and idx.tolist() == g["columns"], name
            assert val.tolist() == g["values"], name
            assert p.rhs().tolist() == g["rhs"] and p.c().tolist() == g["c"], name
            assert p.sense() == g["sense"], name


def test_comments_end_records(golden, golden_dir):
    """mps_parser_test.cpp:167-199: '*' and '$' comment lines, and a '$' field that ends a record
    (ROW2's entry of VAR2 and the later RHS values are comments)."""
    g = golden["mps_parser"]["comments"]
    with _Problem(_path(golden_dir, g["file"])) as p:
        assert p.rc == 0
        off, idx, val = p.matrix()
        assert off.tolist() == g["row_offsets"] and idx.tolist() == g["columns"]
        assert val.tolist() == g["values"]
        assert p.rhs().tolist() == g["rhs"] and p.c().tolist() == g["c"]


def test_objname_picks_the_objective_row(golden, golden_dir):
    """mps_parser_test.cpp:505-530: without OBJNAME the first N row is the objective; with it (on
    its line or the next) the named one, whose COLUMNS has no entries."""
    for name in golden["mps_parser"]["objname"]["files"]:
        with _Problem(_path(golden_dir, name)) as p:
            assert p.rc == 0, name
            assert p.c().tolist() == golden["mps_parser"]["objname"]["c"], name
            assert p.sizes() == (2, 2, 4), name


@pytest.mark.parametrize("name", ["lp_model_with_var_bounds.mps", "free-format-mps-1.mps",
                                  "good-mps-some-var-bounds.mps", "good-mps-fixed-var.mps",
                                  "good-mps-free-var.mps", "good-mps-lower-bound-inf-var.mps",
                                  "good-mps-upper-bound-inf-var.mps"])
def test_variable_bounds(golden, golden_dir, name):
    """mps_parser_test.cpp:303-405: LO / UP / FX / FR / MI bounds and the defaults [0, inf)."""
    g = golden["mps_parser"]["var_bounds"][name]
    with _Problem(_path(golden_dir, name)) as p:
        assert p.rc == 0
        lo, up = p.bounds()
        assert lo.tolist() == [_num(v) for v in g["lower"]]
        assert up.tolist() == [_num(v) for v in g["upper"]]
        if "c" in g:
            assert p.c().tolist() == g["c"] and p.rhs().tolist() == g["rhs"]


def test_objective_rhs_is_the_negated_offset(golden, golden_dir):
    """mps_parser_test.cpp:390-394: an RHS entry of the objective row sets the offset to minus
    that value."""
    g = golden["mps_parser"]["rhs_cost_offset"]
    with _Problem(_path(golden_dir, g["file"])) as p:
        assert p.rc == 0 and p.offset() == g["value"]


def test_ranges_fixed_and_free(golden, golden_dir):
    """mps_parser_test.cpp:407-503: RANGES on L, G and E rows give these row bounds (1e-12)."""
    g = golden["mps_parser"]["ranges"]
    for name in g["files"]:
        with _Problem(_path(golden_dir, name)) as p:
            assert p.rc == 0, name
            lo, up = p.row_bounds()
            np.testing.assert_allclose(lo, g["lower"], rtol=0, atol=1e-12)
            np.testing.assert_allclose(up, g["upper"], rtol=0, atol=1e-12)


@pytest.mark.parametrize("name", ["good-mip-mps-1.mps", "good-mip-mps-1-no-mark.mps",
                                  "good-mip-mps-no-bounds.mps", "good-mip-mps-partial-bounds.mps"])
def test_integer_markers_and_their_default_bounds(golden, golden_dir, name):
    """mps_parser_test.cpp:567-748: columns between INTORG / INTEND markers are integer; UI bounds;
    integer columns with no bound at all get [0, 1]; OBJSENSE MAX on its own line."""
    g = golden["mps_parser"]["mip"]
    want = g[name]
    with _Problem(_path(golden_dir, name)) as p:
        assert p.rc == 0
        off, idx, val = p.matrix()
        assert off.tolist() == g["row_offsets"] and idx.tolist() == g["columns"]
        assert val.tolist() == g["values"]
        assert p.rhs().tolist() == g["rhs"] and p.c().tolist() == g["c"]
        assert p._int(p.L.cuOptGetObjectiveSense) == (-1 if g["maximize"] else 1)
        types = C.create_string_buffer(2)
        assert p.L.cuOptGetVariableTypes(p.h, types) == 0
        assert types.raw.decode() == want["types"]
        lo, up = p.bounds()
        assert lo.tolist() == [_num(v) for v in want["lower"]]
        assert up.tolist() == [_num(v) for v in want["upper"]]


def test_user_problem_file_is_written_before_the_solve(golden_dir, tmp_path):
    """solve.cu:1282-1284: with user_problem_file set, the solve first writes the problem as MPS
    (here the solve itself needs a GPU; the file is written before it starts)."""
    from cuopt_b200 import linear_programming as lpm
    out = tmp_path / "afiro_out.mps"
    s = lpm.SolverSettings()
    s.set_parameter("user_problem_file", str(out))
    lpm.Solve(lpm.ReadMps(golden_dir / "afiro_original.mps"), s)
    a, b = lpm.ReadMps(golden_dir / "afiro_original.mps"), lpm.ReadMps(out)
    for k in ("A_offsets", "A_indices", "A_values", "c", "constraint_lower_bounds",
              "constraint_upper_bounds", "variable_lower_bounds", "variable_upper_bounds"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_solution_file(golden_dir, tmp_path):
    """solver_solution.cu:428-448, solution_writer.cu:16-40: the status line, the objective and one
    'name value' line per column (the no-constraints LP, solved in closed form on the host)."""
    from cuopt_b200 import linear_programming as lpm
    out = tmp_path / "x.sol"
    s = lpm.SolverSettings()
    s.set_parameter(lpm.CUOPT_METHOD, int(lpm.SolverMethod.Concurrent))
    s.set_parameter("solution_file", str(out))
    with _Problem(golden_dir / "lp-model-no-constraints.mps") as p:  # keeps the column names
        assert p.rc == 0
        sh, sol = s._create(), C.c_void_p()
        try:
            assert p.L.cuOptSolve(p.h, sh, C.byref(sol)) == 0
            st = C.c_int32()
            p.L.cuOptGetTerminationStatus(sol, C.byref(st))
            assert st.value == 1
        finally:
            p.L.cuOptDestroySolution(C.byref(sol))
            p.L.cuOptDestroySolverSettings(C.byref(sh))
    lines = out.read_text().splitlines()
    assert lines[0] == "# Status: Optimal"
    assert float(lines[1].split(":")[1]) == 1.0
    assert lines[2].split()[0] == "x1" and float(lines[2].split()[1]) == 1.0
