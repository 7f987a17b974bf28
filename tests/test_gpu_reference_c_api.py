"""The reference's own C API test file (cpp/tests/linear_programming/c_api_tests/c_api_test.c),
compiled unmodified against this library's cuopt_c.h and linked with libcuopt_b200.so
(tests/c_api/ref_cases.mk), runs its LP cases with the expectations of the reference's gtest
harness (c_api_tests.cpp): sizes, afiro Optimal and at an iteration limit, bad parameter name,
missing file, the ranged problem at 32, invalid bounds, writing afiro, and the maximisation whose
objective equals its dual objective (methods served by PDLP)."""
from __future__ import annotations

import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
BINARY = ROOT / "tests" / "c_api" / "_ref" / "ref_c_api_cases"


@pytest.mark.skipif(not BINARY.exists(),
                    reason="tests/c_api/_ref/ref_c_api_cases not built (make -f tests/c_api/ref_cases.mk)")
def test_reference_c_api_lp_cases(tmp_path):
    r = subprocess.run([str(BINARY), str(ROOT / "tests" / "golden" / "afiro_original.mps"),
                        str(tmp_path / "afiro_written.mps")], capture_output=True, text=True,
                       timeout=600)
    cases = [line.split(" ", 3) for line in r.stdout.splitlines() if line.startswith("case ")]
    names = {c[1] for c in cases}
    assert {"int_size", "float_size", "afiro", "iteration_limit", "bad_parameter_name",
            "missing_file", "ranged_problem", "invalid_bounds_lp", "write_problem",
            "maximize_problem_dual_variables"} <= names
    failed = [c for c in cases if c[2] != "ok"]
    assert not failed, failed
    assert r.returncode == 0, r.stdout[-2000:]
