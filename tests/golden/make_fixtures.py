"""Regenerates the golden fixtures in this folder from the reference project (run where the
reference tree is available, with its root as the one argument; the fixtures are committed so
tests never read the reference).

Fixtures:
  *.mps           copies of the reference's small LP datasets (datasets/linear_programming/)
  mps/*.mps       the reference's MPS parser test datasets (same folder)
  golden.json     expected values taken from the reference's own tests, with their source lines.
"""
from __future__ import annotations

import json
import shutil
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
DATASETS = ["afiro_original.mps", "good-max.mps", "max_offset.mps", "lp-model-no-constraints.mps",
            "empty_matrix.mps", "lp_model_with_var_bounds.mps", "good-mps-fixed-ranges.mps",
            "good-mps-some-var-bounds.mps", "good-mps-1.mps"]

# The reference's MPS parser test datasets (cpp/libmps_parser/tests/mps_parser_test.cpp), copied
# into mps/: every bad file must be rejected, the good ones read to the values in golden.json.
MPS_PARSER_DATASETS = (
    [f"bad-mps-{i}.mps" for i in range(1, 16) if i != 8]
    + ["bad-mps-bound-1.mps", "bad-mps-bound-2.mps", "bad-mps-fixed-objname-after-rows.mps",
       "bad-mps-fixed-ranges-name.mps", "bad-mps-fixed-ranges-value.mps", "good-fixed-mps-2.mps",
       "good-mps-1-clrf.mps", "good-mps-1-comments.mps", "free-format-mps-1.mps",
       "good-mps-fixed-empty-name.mps", "good-mps-fixed-no-name.mps",
       "good-mps-fixed-two-objectives.mps", "good-mps-fixed-two-objectives-objname.mps",
       "good-mps-fixed-two-objectives-objname-next-line.mps", "good-mps-fixed-var.mps",
       "good-mps-free-var.mps", "good-mps-lower-bound-inf-var.mps",
       "good-mps-upper-bound-inf-var.mps", "good-mps-rhs-cost.mps", "good-mps-free-ranges.mps"])

MPS_PARSER_MIP_DATASETS = ["good-mip-mps-1.mps", "good-mip-mps-1-no-mark.mps",
                           "good-mip-mps-no-bounds.mps", "good-mip-mps-partial-bounds.mps"]

GOLDEN = {
    "afiro_objective": {
        "value": -464.7531, "rel_tol": 0.01,
        "source": "python/cuopt/cuopt/tests/linear_programming/test_lp_solver.py:109; "
                  "cpp/tests/linear_programming/pdlp_test.cu:48-74 (1% tolerance)"},
    "afiro_methodical1_initial_step_size": {
        "value": 1.4893, "abs_tol": 1e-4,
        "source": "cpp/tests/linear_programming/pdlp_test.cu:243-286"},
    "afiro_methodical1_initial_primal_weight": {
        "value": 0.0141652, "abs_tol": 1e-4,
        "source": "cpp/tests/linear_programming/pdlp_test.cu:243-286"},
    "good_max_objective": {
        "value": 17.0, "abs_tol": 1e-4,
        "source": "cpp/tests/linear_programming/pdlp_test.cu:993-1011"},
    "max_offset_objective": {
        "value": 0.0, "abs_tol": 1e-4,
        "source": "cpp/tests/linear_programming/pdlp_test.cu:1013-1031"},
    "no_constraints_objective": {
        "value": 1.0, "abs_tol": 1e-4,
        "source": "cpp/tests/linear_programming/pdlp_test.cu:1033-1053 (method Concurrent)"},
    "empty_matrix_pdlp_status": {
        "value": 6, "source": "cpp/tests/linear_programming/pdlp_test.cu:952-968 (NumericalError)"},
    "ranged_problem_objective": {
        "value": 32.0, "abs_tol": 1e-3,
        "source": "cpp/tests/linear_programming/c_api_tests/c_api_tests.cpp:105-112, "
                  "c_api_test.c:927-1041"},
    "maximize_dual_objective_match": {
        "abs_tol": 1e-2,
        "source": "cpp/tests/linear_programming/c_api_tests/c_api_tests.cpp:149-165, "
                  "c_api_test.c:1461-1614"},
    "many_different_bounds": {
        "variable": 0, "upper": 10.0,
        "lower": [-133.0, None, -133.0, None, -183.0, -233.0, None, -1033.0, -1033.0, -1283.0,
                  -2533.0, None, None],
        "constraint_tol": 1e-8,
        "note": "None keeps the variable's own bounds; every climber as its single solve, with "
                "constraint violations under constraint_tol",
        "source": "cpp/tests/linear_programming/pdlp_test.cu:1720-1804 (good-mps-some-var-bounds)"},
    "some_climber_hit_iteration_limit": {
        "variable": 0, "upper": 10.0, "lower": [-2533.0, None], "iteration_limit": 500,
        "statuses": ["IterationLimit", "Optimal"],
        "note": "the test's comment: one climber converges within the limit, the other hits it",
        "source": "cpp/tests/linear_programming/pdlp_test.cu:1806-1885"},
    "good_mps_1_optimal": {
        "tol": 1e-2, "status": "Optimal",
        "source": "python/cuopt/cuopt/tests/linear_programming/test_lp_solver.py:82-89"},
    "mps_parser": {
        "source": "cpp/libmps_parser/tests/mps_parser_test.cpp (free format, as cuOptReadProblem "
                  "reads: cpp/src/pdlp/cuopt_c.cpp:103-107)",
        "rejected": ["bad-mps-%d.mps" % i for i in range(1, 16) if i != 8]
        + ["bad-mps-bound-1.mps", "bad-mps-bound-2.mps", "bad-mps-fixed-objname-after-rows.mps",
           "bad-mps-fixed-ranges-name.mps", "bad-mps-fixed-ranges-value.mps",
           "good-fixed-mps-2.mps"],
        "good-1": {"files": ["good-mps-1.mps", "good-mps-1-clrf.mps", "free-format-mps-1.mps",
                             "good-mps-fixed-empty-name.mps", "good-mps-fixed-no-name.mps",
                             "good-mps-fixed-two-objectives.mps"],
                   "row_offsets": [0, 2, 4], "columns": [0, 1, 0, 1],
                   "values": [3.0, 4.0, 2.7, 10.1], "rhs": [5.4, 4.9], "c": [0.2, 0.1],
                   "sense": "LL", "lines": "59-93, 95-129, 249-263, 201-211, 505-512"},
        "comments": {"file": "good-mps-1-comments.mps", "row_offsets": [0, 2, 3],
                     "columns": [0, 1, 0], "values": [3.0, 4.0, 2.7], "rhs": [5.4, 4.9],
                     "c": [0.2, 0.1], "lines": "167-199"},
        "objname": {"files": ["good-mps-fixed-two-objectives-objname.mps",
                              "good-mps-fixed-two-objectives-objname-next-line.mps"],
                    "c": [0.0, 0.0], "lines": "514-530 (objective COST6679327, no entries)"},
        "var_bounds": {
            "lp_model_with_var_bounds.mps": {"lower": [0.0, 1.0], "upper": [1.0, 2.0],
                                             "c": [2.0, -1.0], "rhs": [3.0], "lines": "303-333"},
            "free-format-mps-1.mps": {"lower": [0.0, 0.0], "upper": ["inf", "inf"],
                                      "lines": "335-344"},
            "good-mps-some-var-bounds.mps": {"lower": [-1.0, 0.0], "upper": ["inf", 2.0],
                                             "lines": "346-355"},
            "good-mps-fixed-var.mps": {"lower": [2.0, 0.0], "upper": [2.0, "inf"],
                                       "lines": "357-366"},
            "good-mps-free-var.mps": {"lower": ["-inf", 0.0], "upper": ["inf", "inf"],
                                      "lines": "368-377"},
            "good-mps-lower-bound-inf-var.mps": {"lower": ["-inf", 0.0], "upper": ["inf", "inf"],
                                                 "lines": "379-388"},
            "good-mps-upper-bound-inf-var.mps": {"lower": [0.0, 0.0], "upper": ["inf", "inf"],
                                                 "lines": "396-405"}},
        "rhs_cost_offset": {"file": "good-mps-rhs-cost.mps", "value": -5.0, "lines": "390-394"},
        "mip": {
            "good-mip-mps-1.mps": {"types": "II", "lower": [0.0, 0.0], "upper": [10.0, 10.0],
                                   "lines": "567-617"},
            "good-mip-mps-1-no-mark.mps": {"types": "II", "lower": [0.0, 0.0],
                                           "upper": [10.0, 10.0], "lines": "619-656"},
            "good-mip-mps-no-bounds.mps": {"types": "IC", "lower": [0.0, 0.0],
                                           "upper": [1.0, "inf"], "lines": "658-702"},
            "good-mip-mps-partial-bounds.mps": {"types": "IC", "lower": [0.0, 0.0],
                                                "upper": [1.0, 10.0], "lines": "704-748"},
            "row_offsets": [0, 2, 4], "columns": [0, 1, 0, 1],
            "values": [8000.0, 4000.0, 15.0, 30.0], "rhs": [40000.0, 200.0], "c": [100.0, 150.0],
            "maximize": True},
        "ranges": {"files": ["good-mps-fixed-ranges.mps", "good-mps-free-ranges.mps"],
                   "lower": [1.2, 1.5, 7.9, 3.5, 3.9, 4.9], "upper": [5.4, 4.9, 9.5, 6.9, 3.9, 4.9],
                   "lines": "407-503"}},
    "chess_set_dual_simplex": {
        "objective": 1333.333333, "x": [0.0, 66.666667], "tol": 1e-5,
        "source": "cpp/tests/dual_simplex/unit_tests/solve.cpp:23-94"},
}


def main(ref_root: str) -> None:
    """ref_root: the root of the reference project's source tree (holds datasets/)."""
    src = Path(ref_root) / "datasets" / "linear_programming"
    for name in DATASETS:
        shutil.copyfile(src / name, HERE / name)
    (HERE / "mps").mkdir(exist_ok=True)
    for name in MPS_PARSER_DATASETS:
        shutil.copyfile(src / name, HERE / "mps" / name)
    for name in MPS_PARSER_MIP_DATASETS:
        shutil.copyfile(src.parent / "mixed_integer_programming" / name, HERE / "mps" / name)
    (HERE / "golden.json").write_text(json.dumps(GOLDEN, indent=2) + "\n")
    print("wrote", len(DATASETS), "datasets and golden.json to", HERE)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_fixtures.py <reference project root>")
    main(sys.argv[1])
