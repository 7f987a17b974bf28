/* A C caller of cuOpt's LP C API, built against include/cuopt/linear_programming/cuopt_c.h and
 * linked to libcuopt_b200.so without changes: it solves an MPS file given on the command line
 * and a two-variable ranged LP built from arrays, printing one line per solve:
 *   <label> <termination status> <objective>
 * Exit code 0 when every call returned CUOPT_SUCCESS. */
#include <math.h>
#include <stdio.h>

#include <cuopt/linear_programming/cuopt_c.h>

static int check(cuopt_int_t rc, const char* what)
{
  if (rc != CUOPT_SUCCESS) fprintf(stderr, "%s returned %d\n", what, (int)rc);
  return rc != CUOPT_SUCCESS;
}

static int solve_and_print(const char* label, cuOptOptimizationProblem problem)
{
  cuOptSolverSettings settings = NULL;
  cuOptSolution solution       = NULL;
  cuopt_int_t status           = -1;
  cuopt_float_t objective      = 0.0;
  int failed = check(cuOptCreateSolverSettings(&settings), "cuOptCreateSolverSettings");
  failed |= check(cuOptSetFloatParameter(settings, CUOPT_ABSOLUTE_PRIMAL_TOLERANCE, 1e-6), "tol");
  failed |= check(cuOptSetFloatParameter(settings, CUOPT_RELATIVE_PRIMAL_TOLERANCE, 1e-6), "tol");
  failed |= check(cuOptSetFloatParameter(settings, CUOPT_ABSOLUTE_DUAL_TOLERANCE, 1e-6), "tol");
  failed |= check(cuOptSetFloatParameter(settings, CUOPT_RELATIVE_DUAL_TOLERANCE, 1e-6), "tol");
  failed |= check(cuOptSetFloatParameter(settings, CUOPT_ABSOLUTE_GAP_TOLERANCE, 1e-6), "tol");
  failed |= check(cuOptSetFloatParameter(settings, CUOPT_RELATIVE_GAP_TOLERANCE, 1e-6), "tol");
  failed |= check(cuOptSetIntegerParameter(settings, CUOPT_METHOD, CUOPT_METHOD_PDLP), "method");
  failed |= check(cuOptSetParameter(settings, CUOPT_LOG_TO_CONSOLE, "false"), "log");
  failed |= check(cuOptSolve(problem, settings, &solution), "cuOptSolve");
  failed |= check(cuOptGetTerminationStatus(solution, &status), "cuOptGetTerminationStatus");
  failed |= check(cuOptGetObjectiveValue(solution, &objective), "cuOptGetObjectiveValue");
  printf("%s %d %.10g\n", label, (int)status, (double)objective);
  cuOptDestroySolution(&solution);
  cuOptDestroySolverSettings(&settings);
  return failed;
}

int main(int argc, char** argv)
{
  int failed = 0;
  if (argc > 1) {
    cuOptOptimizationProblem mps = NULL;
    failed |= check(cuOptReadProblem(argv[1], &mps), "cuOptReadProblem");
    if (mps) failed |= solve_and_print("mps", mps);
    cuOptDestroyProblem(&mps);
  }
  /* max 3 x0 + 2 x1  s.t.  x0 + x1 <= 4,  1 <= x0 + 3 x1 <= 6,  0 <= x0 <= 3,  x1 >= 0
   * optimum x = (3, 1), objective 11. */
  const cuopt_int_t row_offsets[]  = {0, 2, 4};
  const cuopt_int_t columns[]      = {0, 1, 0, 1};
  const cuopt_float_t values[]     = {1.0, 1.0, 1.0, 3.0};
  const cuopt_float_t c[]          = {3.0, 2.0};
  const cuopt_float_t row_lo[]     = {-CUOPT_INFINITY, 1.0};
  const cuopt_float_t row_up[]     = {4.0, 6.0};
  const cuopt_float_t var_lo[]     = {0.0, 0.0};
  const cuopt_float_t var_up[]     = {3.0, CUOPT_INFINITY};
  const char var_types[]           = {CUOPT_CONTINUOUS, CUOPT_CONTINUOUS};
  cuOptOptimizationProblem ranged  = NULL;
  failed |= check(cuOptCreateRangedProblem(2, 2, CUOPT_MAXIMIZE, 0.0, c, row_offsets, columns,
                                           values, row_lo, row_up, var_lo, var_up, var_types,
                                           &ranged),
                  "cuOptCreateRangedProblem");
  if (ranged) failed |= solve_and_print("ranged", ranged);
  cuOptDestroyProblem(&ranged);
  return failed;
}
