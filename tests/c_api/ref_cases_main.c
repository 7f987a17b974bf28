/* TEST INFRASTRUCTURE: runs LP cases of the reference's own C API test file
 * (cpp/tests/linear_programming/c_api_tests/c_api_test.c in the cuOpt project, compiled where it
 * lies by tests/c_api/ref_cases.mk) against this library, with the expectations of the reference's
 * gtest harness (cpp/tests/linear_programming/c_api_tests/c_api_tests.cpp, lines cited per case).
 * Prints one "case <name> ok|FAIL <detail>" line per case and exits non-zero if any case fails.
 * argv[1]: the afiro_original.mps dataset; argv[2]: a writable temporary .mps path. */
#include <cuopt/linear_programming/cuopt_c.h>

#include <math.h>
#include <stdio.h>

/* The reference test file's entry points (declared as its c_api_tests.h declares them). */
int test_int_size();
int test_float_size();
cuopt_int_t solve_mps_file(const char* filename, double time_limit, double iteration_limit,
                           cuopt_int_t* termination_status, cuopt_float_t* solve_time,
                           cuopt_int_t method);
cuopt_int_t test_missing_file();
cuopt_int_t test_bad_parameter_name();
cuopt_int_t test_ranged_problem(cuopt_int_t* termination_status_ptr, cuopt_float_t* objective_ptr);
cuopt_int_t test_invalid_bounds(cuopt_int_t test_mip);
cuopt_int_t test_write_problem(const char* input_filename, const char* output_filename);
cuopt_int_t test_maximize_problem_dual_variables(cuopt_int_t method,
                                                 cuopt_int_t* termination_status_ptr,
                                                 cuopt_float_t* objective_ptr,
                                                 cuopt_float_t* dual_variables,
                                                 cuopt_float_t* reduced_costs,
                                                 cuopt_float_t* dual_obj_ptr);

static int failures = 0;

static void report(const char* name, int ok, const char* detail)
{
  printf("case %s %s %s\n", name, ok ? "ok" : "FAIL", detail);
  failures += !ok;
}

int main(int argc, char** argv)
{
  char buf[256];
  if (argc < 3) {
    fprintf(stderr, "usage: ref_c_api_cases <afiro_original.mps> <tmp.mps>\n");
    return 2;
  }
  /* c_api_tests.cpp:21-23 */
  report("int_size", test_int_size() == 4, "");
  report("float_size", test_float_size() == 8, "");
  /* c_api_tests.cpp:25-33: afiro Optimal within 60 s (method PDLP: the library's method) */
  {
    cuopt_int_t st = -1;
    cuopt_float_t t = 0;
    const cuopt_int_t rc = solve_mps_file(argv[1], 60, CUOPT_INFINITY, &st, &t, CUOPT_METHOD_PDLP);
    snprintf(buf, sizeof buf, "rc=%d status=%d", rc, st);
    report("afiro", rc == CUOPT_SUCCESS && st == CUOPT_TERIMINATION_STATUS_OPTIMAL, buf);
  }
  /* c_api_tests.cpp:71-78: afiro at an iteration limit of 1 */
  {
    cuopt_int_t st = -1;
    cuopt_float_t t = 0;
    const cuopt_int_t rc = solve_mps_file(argv[1], 60, 1, &st, &t, CUOPT_METHOD_PDLP);
    snprintf(buf, sizeof buf, "rc=%d status=%d", rc, st);
    report("iteration_limit", rc == CUOPT_SUCCESS && st == CUOPT_TERIMINATION_STATUS_ITERATION_LIMIT,
           buf);
  }
  /* c_api_tests.cpp:93 and :101 */
  report("bad_parameter_name", test_bad_parameter_name() == CUOPT_INVALID_ARGUMENT, "");
  report("missing_file", test_missing_file() == CUOPT_MPS_FILE_ERROR, "");
  /* c_api_tests.cpp:105-112: Optimal, objective 32 within 1e-3 */
  {
    cuopt_int_t st = -1;
    cuopt_float_t obj = 0;
    const cuopt_int_t rc = test_ranged_problem(&st, &obj);
    snprintf(buf, sizeof buf, "rc=%d status=%d objective=%.9g", rc, st, obj);
    report("ranged_problem",
           rc == CUOPT_SUCCESS && st == CUOPT_TERIMINATION_STATUS_OPTIMAL && fabs(obj - 32.0) <= 1e-3,
           buf);
  }
  /* c_api_tests.cpp:114-120 (the LP half; integer variables are outside this library) */
  report("invalid_bounds_lp", test_invalid_bounds(0) == CUOPT_SUCCESS, "");
  /* c_api_tests.cpp:140-147 */
  report("write_problem", test_write_problem(argv[1], argv[2]) == CUOPT_SUCCESS, "");
  /* c_api_tests.cpp:149-165, for the methods the library solves by PDLP as the reference's PDLP
   * and concurrent cases do: Optimal, objective equal to the dual objective within 1e-2. */
  {
    const cuopt_int_t methods[2] = {CUOPT_METHOD_CONCURRENT, CUOPT_METHOD_PDLP};
    for (int q = 0; q < 2; ++q) {
      cuopt_int_t st = -1;
      cuopt_float_t obj = 0, dobj = 0, duals[3], rcs[4];
      const cuopt_int_t rc =
        test_maximize_problem_dual_variables(methods[q], &st, &obj, duals, rcs, &dobj);
      snprintf(buf, sizeof buf, "method=%d rc=%d status=%d objective=%.9g dual=%.9g", methods[q],
               rc, st, obj, dobj);
      report("maximize_problem_dual_variables",
             rc == CUOPT_SUCCESS && st == CUOPT_TERIMINATION_STATUS_OPTIMAL &&
               fabs(obj - dobj) <= 1e-2,
             buf);
    }
  }
  printf("failures %d\n", failures);
  return failures ? 1 : 0;
}
