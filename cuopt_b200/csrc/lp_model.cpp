// Problem / settings / solution objects behind the C interface, validation and solve dispatch.
#include "lp_model.hpp"

#include <cuopt/linear_programming/constants.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <exception>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <stdexcept>
#include <thread>

#include "common.cuh"
#include "host_io.hpp"
#include "pdlp_schedule.hpp"

namespace cuopt_b200 {

namespace {
constexpr double kInf = std::numeric_limits<double>::infinity();
}

void lp_problem::constraint_bounds(std::vector<double>& lo, std::vector<double>& up) const
{
  if (ranged) {
    lo.assign(con_lo.begin(), con_lo.end());
    up.assign(con_up.begin(), con_up.end());
    return;
  }
  lo.resize(m);
  up.resize(m);
  for (int i = 0; i < m; ++i) {  // transform_bounds_functor (problem_helpers.cuh:26-51)
    const char t = row_types[i];
    if (t == 'E') {
      lo[i] = rhs[i];
      up[i] = rhs[i];
    } else if (t == 'G') {
      lo[i] = rhs[i];
      up[i] = kInf;
    } else if (t == 'L') {
      lo[i] = -kInf;
      up[i] = rhs[i];
    } else {
      lo[i] = -kInf;
      up[i] = -kInf;
    }
  }
}

bool lp_problem::is_mip() const
{
  return std::any_of(var_types.begin(), var_types.end(), [](char t) { return t == 'I'; });
}

// ------------------------------------------------------------------------------------------
// Settings registry: same names, ranges and defaults as the reference
// (cpp/src/math_optimization/solver_settings.cu:55-135), plus this library's pdlp_* additions.

lp_settings::lp_settings()
{
  const double inf = kInf;
  fparams          = {
    {CUOPT_TIME_LIMIT, 0.0, inf, inf},
    {CUOPT_WORK_LIMIT, 0.0, inf, inf},
    {CUOPT_ABSOLUTE_DUAL_TOLERANCE, 0.0, 1e-1, 1e-4},
    {CUOPT_RELATIVE_DUAL_TOLERANCE, 0.0, 1e-1, 1e-4},
    {CUOPT_ABSOLUTE_PRIMAL_TOLERANCE, 0.0, 1e-1, 1e-4},
    {CUOPT_RELATIVE_PRIMAL_TOLERANCE, 0.0, 1e-1, 1e-4},
    {CUOPT_ABSOLUTE_GAP_TOLERANCE, 0.0, 1e-1, 1e-4},
    {CUOPT_RELATIVE_GAP_TOLERANCE, 0.0, 1e-1, 1e-4},
    {CUOPT_MIP_ABSOLUTE_TOLERANCE, 0.0, 1e-1, 1e-4},
    {CUOPT_MIP_RELATIVE_TOLERANCE, 0.0, 1e-1, 1e-4},
    {CUOPT_MIP_INTEGRALITY_TOLERANCE, 0.0, 1e-1, 1e-5},
    {CUOPT_MIP_ABSOLUTE_GAP, 0.0, inf, 1e-10},
    {CUOPT_MIP_RELATIVE_GAP, 0.0, 1e-1, 1e-4},
    {CUOPT_PRIMAL_INFEASIBLE_TOLERANCE, 0.0, 1e-1, 1e-10},
    {CUOPT_DUAL_INFEASIBLE_TOLERANCE, 0.0, 1e-1, 1e-10},
    {CUOPT_MIP_CUT_CHANGE_THRESHOLD, 0.0, inf, 1e-3},
    {CUOPT_MIP_CUT_MIN_ORTHOGONALITY, 0.0, 1.0, 0.5},
    {CUOPT_PDLP_REFINEMENT_TOLERANCE, 0.0, 1e-1, 1e-8},
  };
  iparams = {
    {CUOPT_ITERATION_LIMIT, 0, INT_MAX, INT_MAX},
    {CUOPT_PDLP_SOLVER_MODE, CUOPT_PDLP_SOLVER_MODE_STABLE1, CUOPT_PDLP_SOLVER_MODE_STABLE3,
     CUOPT_PDLP_SOLVER_MODE_STABLE3},
    {CUOPT_METHOD, CUOPT_METHOD_CONCURRENT, CUOPT_METHOD_BARRIER, CUOPT_METHOD_CONCURRENT},
    {CUOPT_NUM_CPU_THREADS, -1, INT_MAX, -1},
    {CUOPT_AUGMENTED, -1, 1, -1},
    {CUOPT_FOLDING, -1, 1, -1},
    {CUOPT_DUALIZE, -1, 1, -1},
    {CUOPT_ORDERING, -1, 1, -1},
    {CUOPT_BARRIER_DUAL_INITIAL_POINT, -1, 1, -1},
    {CUOPT_MIP_CUT_PASSES, -1, INT_MAX, 10},
    {CUOPT_MIP_MIXED_INTEGER_ROUNDING_CUTS, -1, 1, -1},
    {CUOPT_MIP_MIXED_INTEGER_GOMORY_CUTS, -1, 1, -1},
    {CUOPT_MIP_KNAPSACK_CUTS, -1, 1, -1},
    {CUOPT_MIP_STRONG_CHVATAL_GOMORY_CUTS, -1, 1, -1},
    {CUOPT_MIP_REDUCED_COST_STRENGTHENING, -1, INT_MAX, -1},
    {CUOPT_NUM_GPUS, 1, 2, 1},
    {CUOPT_MIP_BATCH_PDLP_STRONG_BRANCHING, 0, 1, 0},
    {CUOPT_PRESOLVE, CUOPT_PRESOLVE_DEFAULT, CUOPT_PRESOLVE_PSLP, CUOPT_PRESOLVE_DEFAULT},
    {CUOPT_MIP_DETERMINISM_MODE, CUOPT_MODE_OPPORTUNISTIC, CUOPT_MODE_DETERMINISTIC,
     CUOPT_MODE_OPPORTUNISTIC},
    {CUOPT_RANDOM_SEED, -1, INT_MAX, -1},
    {CUOPT_MIP_RELIABILITY_BRANCHING, -1, INT_MAX, -1},
    {CUOPT_PDLP_PRECISION, CUOPT_PDLP_PRECISION_FP64, CUOPT_PDLP_PRECISION_MIXED,
     CUOPT_PDLP_PRECISION_FP64},
    {CUOPT_PDLP_REFINEMENT_PASSES, 0, 64, 0},
    {CUOPT_PDLP_TILED_SWEEPS, CUOPT_PDLP_TILED_SWEEPS_AUTO, CUOPT_PDLP_TILED_SWEEPS_ON,
     CUOPT_PDLP_TILED_SWEEPS_AUTO},
    {CUOPT_PDLP_PERSISTENT_ITERATIONS, CUOPT_PDLP_PERSISTENT_ITERATIONS_AUTO,
     CUOPT_PDLP_PERSISTENT_ITERATIONS_CLUSTER, CUOPT_PDLP_PERSISTENT_ITERATIONS_AUTO},
    {CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK, 0, 16, 0},
  };
  bparams = {
    {CUOPT_INFEASIBILITY_DETECTION, false}, {CUOPT_STRICT_INFEASIBILITY, false},
    {CUOPT_PER_CONSTRAINT_RESIDUAL, false}, {CUOPT_SAVE_BEST_PRIMAL_SO_FAR, false},
    {CUOPT_FIRST_PRIMAL_FEASIBLE, false},   {CUOPT_MIP_SCALING, true},
    {CUOPT_MIP_HEURISTICS_ONLY, false},     {CUOPT_LOG_TO_CONSOLE, true},
    {CUOPT_CROSSOVER, false},               {CUOPT_ELIMINATE_DENSE_COLUMNS, true},
    {CUOPT_CUDSS_DETERMINISTIC, false},     {CUOPT_DUAL_POSTSOLVE, true},
  };
  sparams = {{CUOPT_LOG_FILE, ""}, {CUOPT_SOLUTION_FILE, ""}, {CUOPT_USER_PROBLEM_FILE, ""}};
}

namespace {
bool parse_int(const std::string& v, int32_t& out)
{
  try {
    out = std::stoi(v);
    return true;
  } catch (const std::exception&) {
    return false;
  }
}
bool parse_float(const std::string& v, double& out)
{
  try {
    out = std::stod(v);
    return true;
  } catch (const std::exception&) {
    return false;
  }
}
bool parse_bool(const std::string& v, bool& out)
{
  if (v == "true" || v == "True" || v == "TRUE" || v == "1" || v == "t" || v == "T") {
    out = true;
    return true;
  }
  if (v == "false" || v == "False" || v == "FALSE" || v == "0" || v == "f" || v == "F") {
    out = false;
    return true;
  }
  return false;
}
}  // namespace

// set_parameter_from_string (reference solver_settings.cu:137-204)
int lp_settings::set_from_string(const std::string& name, const std::string& value)
{
  for (auto& p : iparams)
    if (name == p.name) {
      int32_t v;
      if (!parse_int(value, v) || v < p.min || v > p.max) return CUOPT_INVALID_ARGUMENT;
      p.value = v;
      return CUOPT_SUCCESS;
    }
  for (auto& p : fparams)
    if (name == p.name) {
      double v;
      if (!parse_float(value, v) || v < p.min || v > p.max) return CUOPT_INVALID_ARGUMENT;
      p.value = v;
      return CUOPT_SUCCESS;
    }
  for (auto& p : bparams)
    if (name == p.name) {
      bool v;
      if (!parse_bool(value, v)) return CUOPT_INVALID_ARGUMENT;
      p.value = v;
      return CUOPT_SUCCESS;
    }
  for (auto& p : sparams)
    if (name == p.name) {
      p.value = value;
      return CUOPT_SUCCESS;
    }
  return CUOPT_INVALID_ARGUMENT;
}

int lp_settings::set_int(const std::string& name, int32_t v)
{
  for (auto& p : iparams)
    if (name == p.name) {
      if (v < p.min || v > p.max) return CUOPT_INVALID_ARGUMENT;
      p.value = v;
      return CUOPT_SUCCESS;
    }
  return CUOPT_INVALID_ARGUMENT;
}
int lp_settings::set_float(const std::string& name, double v)
{
  for (auto& p : fparams)
    if (name == p.name) {
      if (!(v >= p.min && v <= p.max)) return CUOPT_INVALID_ARGUMENT;
      p.value = v;
      return CUOPT_SUCCESS;
    }
  return CUOPT_INVALID_ARGUMENT;
}
int lp_settings::set_bool(const std::string& name, bool v)
{
  for (auto& p : bparams)
    if (name == p.name) {
      p.value = v;
      return CUOPT_SUCCESS;
    }
  return CUOPT_INVALID_ARGUMENT;
}
int lp_settings::get_int(const std::string& name, int32_t& v) const
{
  for (auto& p : iparams)
    if (name == p.name) {
      v = p.value;
      return CUOPT_SUCCESS;
    }
  return CUOPT_INVALID_ARGUMENT;
}
int lp_settings::get_float(const std::string& name, double& v) const
{
  for (auto& p : fparams)
    if (name == p.name) {
      v = p.value;
      return CUOPT_SUCCESS;
    }
  return CUOPT_INVALID_ARGUMENT;
}
int lp_settings::get_bool(const std::string& name, bool& v) const
{
  for (auto& p : bparams)
    if (name == p.name) {
      v = p.value;
      return CUOPT_SUCCESS;
    }
  return CUOPT_INVALID_ARGUMENT;
}
int lp_settings::get_as_string(const std::string& name, std::string& v) const
{
  for (auto& p : iparams)
    if (name == p.name) {
      v = std::to_string(p.value);
      return CUOPT_SUCCESS;
    }
  for (auto& p : fparams)
    if (name == p.name) {
      v = std::to_string(p.value);
      return CUOPT_SUCCESS;
    }
  for (auto& p : bparams)
    if (name == p.name) {
      v = p.value ? "true" : "false";
      return CUOPT_SUCCESS;
    }
  for (auto& p : sparams)
    if (name == p.name) {
      v = p.value;
      return CUOPT_SUCCESS;
    }
  return CUOPT_INVALID_ARGUMENT;
}
double lp_settings::f(const char* name) const
{
  double v = 0;
  get_float(name, v);
  return v;
}
int32_t lp_settings::i(const char* name) const
{
  int32_t v = 0;
  get_int(name, v);
  return v;
}
bool lp_settings::b(const char* name) const
{
  bool v = false;
  get_bool(name, v);
  return v;
}

// ------------------------------------------------------------------------------------------

// True when bad(i) holds for some i in [0, count), tested on up to 8 host threads for large counts.
template <class Pred>
static bool any_of_index(int64_t count, Pred bad)
{
  constexpr int64_t kPerThread = int64_t(1) << 18;
  const int nt = (int)std::min<int64_t>(std::max(1u, std::min(8u, std::thread::hardware_concurrency())),
                                        std::max<int64_t>(1, count / kPerThread));
  if (nt <= 1) {
    for (int64_t i = 0; i < count; ++i)
      if (bad(i)) return true;
    return false;
  }
  std::atomic<bool> found{false};
  auto part = [&](int t) {
    for (int64_t i = count * t / nt, e = count * (t + 1) / nt; i < e && !found.load(); ++i)
      if (bad(i)) found = true;
  };
  std::vector<std::thread> pool;
  int started = 0;
  try {
    for (; started < nt; ++started) pool.emplace_back(part, started);
  } catch (...) {  // no thread to spare: the rest is tested here
  }
  for (int t = started; t < nt; ++t) part(t);
  for (auto& th : pool) th.join();
  return found.load();
}

std::string validate_problem(const lp_problem& p)
{
  if (p.m < 0 || p.n < 0) return "Negative problem dimensions.";
  if ((int)p.row_off.size() != p.m + 1) return "A_offsets must have num_constraints + 1 entries.";
  if (p.row_off[0] != 0) return "A_offsets first value should be 0.";
  if (any_of_index(p.m, [&](int64_t i) { return p.row_off[i + 1] < p.row_off[i]; }))
    return "A_offsets values must in an increasing order.";
  const int64_t nnz = p.row_off[p.m];
  if ((int64_t)p.col_idx.size() != nnz || (int64_t)p.val.size() != nnz)
    return "A_index and A_values must have same sizes.";
  // Column indices are range-checked on the device while the matrix layout is built
  // (a violation is reported as CUOPT_VALIDATION_ERROR by cuOptSolve).
  if ((int)p.c.size() != p.n) return "c must be set before calling the solver.";
  if ((int)p.var_lo.size() != p.n || (int)p.var_up.size() != p.n)
    return "Sizes for vectors related to the variables are not the same.";
  if (p.ranged) {
    if ((int)p.con_lo.size() != p.m || (int)p.con_up.size() != p.m)
      return "Sizes for vectors related to the constraints are not the same.";
  } else {
    if ((int)p.row_types.size() != p.m || (int)p.rhs.size() != p.m)
      return "Sizes for vectors related to the constraints are not the same.";
    for (char t : p.row_types)
      if (t != 'E' && t != 'G' && t != 'L') return "row_types values must equal to 'E', 'G' or 'L'.";
  }
  return "";
}

namespace {

// Variables with no constraints: each coordinate minimises c_j x_j over [l_j, u_j] on its own.
// (The reference hands such problems to dual simplex under Concurrent, and returns
// NumericalError from PDLP, solve.cu:562-567.)
lp_solution solve_without_constraints(const lp_problem& p)
{
  lp_solution s;
  auto& r      = s.r;
  const double sg = p.maximize ? -1.0 : 1.0;
  r.x.assign(p.n, 0.0);
  r.rc.assign(p.n, 0.0);
  double obj   = 0.0;
  bool bounded = true;
  for (int j = 0; j < p.n; ++j) {
    const double cj = sg * p.c[j];
    double v;
    if (cj > 0)
      v = p.var_lo[j];
    else if (cj < 0)
      v = p.var_up[j];
    else
      v = std::min(std::max(0.0, p.var_lo[j]), p.var_up[j]);
    if (!std::isfinite(v)) bounded = false;
    r.x[j]  = v;
    r.rc[j] = p.c[j];
    obj += p.c[j] * (std::isfinite(v) ? v : 0.0);
  }
  r.status     = bounded ? CUOPT_TERIMINATION_STATUS_OPTIMAL : CUOPT_TERIMINATION_STATUS_UNBOUNDED;
  r.primal_obj = obj + p.obj_offset;
  r.dual_obj   = r.primal_obj;
  s.solved_by_pdlp = false;
  return s;
}

}  // namespace

std::string solver_mode_error(const lp_settings& st)
{
  // Only Stable3, the reference's default mode (solve.cu:167-209), is built; the others need the
  // adaptive step size (adaptive_step_size_strategy.cu:168-270) and the KKT / trust-region
  // restarts, which are not.  Asking for them is an error rather than a silent substitution.
  const int wpb = st.i(CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK);
  if (wpb != 0 && wpb != 4 && wpb != 8 && wpb != 16)
    return "pdlp_sweep_warps_per_block must be 0 (chosen by timing), 4, 8 or 16";
  const int mode = st.i(CUOPT_PDLP_SOLVER_MODE);
  if (mode == CUOPT_PDLP_SOLVER_MODE_STABLE3) return {};
  static const char* names[] = {"Stable1", "Stable2", "Methodical1", "Fast1"};
  return std::string("pdlp_solver_mode ") + (mode >= 0 && mode < 4 ? names[mode] : "?") +
         " is not available in this library (only Stable3, the default, is built)";
}

pdlp_params params_from_settings(const lp_settings& st)
{
  pdlp_params prm;
  prm.abs_primal        = st.f(CUOPT_ABSOLUTE_PRIMAL_TOLERANCE);
  prm.rel_primal        = st.f(CUOPT_RELATIVE_PRIMAL_TOLERANCE);
  prm.abs_dual          = st.f(CUOPT_ABSOLUTE_DUAL_TOLERANCE);
  prm.rel_dual          = st.f(CUOPT_RELATIVE_DUAL_TOLERANCE);
  prm.abs_gap           = st.f(CUOPT_ABSOLUTE_GAP_TOLERANCE);
  prm.rel_gap           = st.f(CUOPT_RELATIVE_GAP_TOLERANCE);
  prm.iteration_limit   = st.i(CUOPT_ITERATION_LIMIT);
  prm.time_limit        = st.f(CUOPT_TIME_LIMIT);
  prm.precision         = st.i(CUOPT_PDLP_PRECISION);
  prm.refinement_passes = st.i(CUOPT_PDLP_REFINEMENT_PASSES);
  prm.refinement_tol    = st.f(CUOPT_PDLP_REFINEMENT_TOLERANCE);
  prm.tiled_sweeps      = st.i(CUOPT_PDLP_TILED_SWEEPS);
  prm.persistent        = st.i(CUOPT_PDLP_PERSISTENT_ITERATIONS);
  prm.sweep_wpb         = st.i(CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK);
  prm.log_to_console    = st.b(CUOPT_LOG_TO_CONSOLE);
  prm.detect_infeasibility  = st.b(CUOPT_INFEASIBILITY_DETECTION);
  prm.per_constraint_residual = st.b(CUOPT_PER_CONSTRAINT_RESIDUAL);
  prm.primal_infeasible_tol = st.f(CUOPT_PRIMAL_INFEASIBLE_TOLERANCE);
  prm.dual_infeasible_tol   = st.f(CUOPT_DUAL_INFEASIBLE_TOLERANCE);
  return prm;
}

// Constraint bounds as PDLP takes them: a ranged problem's own arrays, otherwise built from the
// row types and right-hand sides.
struct row_bounds {
  const double* lo = nullptr;
  const double* up = nullptr;
  std::vector<double> lo_store, up_store;
};

// The checks and special cases that come before PDLP (reference solve.cu:1124-1342 and
// problem_checking.cu).  Returns true when the problem goes to PDLP with constraint bounds `rb`;
// otherwise `out` already holds the answer.
static bool prepare_for_pdlp(const lp_problem& p, const lp_settings& st, row_bounds& rb,
                             lp_solution& out)
{
  const auto t0 = std::chrono::steady_clock::now();
  if (p.quadratic) {
    out.error_code    = CUOPT_VALIDATION_ERROR;
    out.error_message = "Quadratic objectives are not supported by this library.";
    return false;
  }
  if (p.is_mip()) {
    out.error_code    = CUOPT_VALIDATION_ERROR;
    out.error_message = "Integer variables are not supported by this library (LP only).";
    return false;
  }
  std::string err = validate_problem(p);
  if (err.empty()) err = solver_mode_error(st);
  if (!err.empty()) {
    out.error_code    = CUOPT_VALIDATION_ERROR;
    out.error_message = err;
    return false;
  }
  trace("validate_problem");
  if (p.ranged) {
    rb.lo = p.con_lo.data();
    rb.up = p.con_up.data();
  } else {
    p.constraint_bounds(rb.lo_store, rb.up_store);
    rb.lo = rb.lo_store.data();
    rb.up = rb.up_store.data();
  }
  const double* lo = rb.lo;
  const double* up = rb.up;
  // has_crossing_bounds (reference problem_checking.cu:316-339)
  if (any_of_index(p.n, [&](int64_t j) { return !(p.var_up[j] >= p.var_lo[j]); }) ||
      (p.ranged && any_of_index(p.m, [&](int64_t i) { return !(up[i] >= lo[i]); }))) {
    out.r.status = CUOPT_TERIMINATION_STATUS_INFEASIBLE;
    return false;
  }
  const int method = st.i(CUOPT_METHOD);
  if (p.m == 0) {
    if (method == CUOPT_METHOD_PDLP) {
      out.r.status = CUOPT_TERIMINATION_STATUS_NUMERICAL_ERROR;
      return false;
    }
    out = solve_without_constraints(p);
    out.r.solve_time = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return false;
  }
  if (p.n == 0) {
    out.r.status = CUOPT_TERIMINATION_STATUS_NUMERICAL_ERROR;
    return false;
  }
  return true;
}

device_problem::~device_problem()
{
  if (!base) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess) {
    cudaFreeAsync(base, s);
    cudaStreamDestroy(s);
  }
  if (cur >= 0 && cur != device) cudaSetDevice(cur);
  cudaGetLastError();
}

static void set_error(lp_solution& out, int code, const char* what)
{
  out.error_code    = code;
  out.error_message = what;
}

lp_solution solve_problem(const lp_problem& p, const lp_settings& st)
{
  lp_solution out;
  trace("solve_problem: start");
  try {
    row_bounds rb;
    if (!prepare_for_pdlp(p, st, rb, out)) return out;
    pdlp_params prm = params_from_settings(st);
    if ((int)st.initial_primal.size() == p.n) prm.initial_primal = st.initial_primal;
    if ((int)st.initial_dual.size() == p.m) prm.initial_dual = st.initial_dual;
    lp_input in;
    in.dev        = p.dev.p.get();
    in.m          = p.m;
    in.n          = p.n;
    in.row_off    = p.row_off.data();
    in.col_idx    = p.col_idx.data();
    in.val        = p.val.data();
    in.c          = p.c.data();
    in.con_lo     = rb.lo;
    in.con_up     = rb.up;
    in.var_lo     = p.var_lo.data();
    in.var_up     = p.var_up.data();
    in.obj_offset = p.obj_offset;
    in.maximize   = p.maximize;
    trace("constraint bounds + checks");
    out.r         = pdlp_solve(in, prm);
    trace("pdlp_solve");
    if (st.b(CUOPT_CROSSOVER) && out.r.status == CUOPT_TERIMINATION_STATUS_OPTIMAL) {
      ensure_host(out.r);
      out.r.crossover = vertex_polish(p, out.r);
    }
    if (prm.log_to_console)
      std::printf("PDLP status %d  objective %+.10e  iterations %lld  time %.3fs\n", out.r.status,
                  out.r.primal_obj, (long long)out.r.iterations, out.r.solve_time);
  } catch (const std::bad_alloc& e) {
    out.error_code    = CUOPT_OUT_OF_MEMORY;
    out.error_message = "Memory allocation failed";
  } catch (const cuda_error& e) {
    out.error_code    = CUOPT_RUNTIME_ERROR;
    out.error_message = e.what();
  } catch (const std::invalid_argument& e) {
    out.error_code    = CUOPT_VALIDATION_ERROR;
    out.error_message = e.what();
  } catch (const std::exception& e) {
    out.error_code    = CUOPT_RUNTIME_ERROR;
    out.error_message = e.what();
  }
  return out;
}

// Starting point of one instance: its solution (user order; duals in the solver's sign
// convention), step size and primal weight.
struct batch_warm {
  host_array<double> x, y;
  double step = 0.0, weight = 1.0;
};

// One block-diagonal batch on the device (see pdlp_batch_solve_device); `warm`, when given, holds
// a starting point per instance of `ids`.
static void solve_batch_chunk(const std::vector<const lp_problem*>& ps,
                              const std::vector<size_t>& ids, const std::vector<row_bounds>& rb,
                              const pdlp_params& prm, bool crossover, std::vector<lp_solution>& out,
                              const std::vector<batch_warm>* warm = nullptr)
{
  const auto t_chunk = std::chrono::steady_clock::now();
  batch_device_input bi;
  bi.count = (int)ids.size();
  bi.row_start.assign(1, 0);
  bi.col_start.assign(1, 0);
  int64_t nnz = 0;
  for (size_t id : ids) {
    const lp_problem& p = *ps[id];
    bi.row_start.push_back(bi.row_start.back() + p.m);
    bi.col_start.push_back(bi.col_start.back() + p.n);
    nnz += p.row_off[p.m];
    bi.obj_offset.push_back(p.obj_offset);
    bi.maximize.push_back(p.maximize ? 1 : 0);
  }
  const int m = bi.row_start.back(), n = bi.col_start.back();
  const size_t nz = (size_t)std::max<int64_t>(nnz, 1);
  std::vector<int> e0(bi.count + 1, 0);
  for (int b = 0; b < bi.count; ++b) e0[b + 1] = e0[b] + ps[ids[b]]->row_off[ps[ids[b]]->m];
  cudaStream_t s;
  B200_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct stream_guard {
    cudaStream_t s;
    ~stream_guard() { cudaStreamDestroy(s); }
  } guard{s};
  alloc_scope scope(s);
  configure_pool_once();
  dbuf<int> doff(m + 1), didx(nz), dri(m), dci(n), drs(bi.count + 1), dcs(bi.count + 1),
    des(bi.count + 1);
  dbuf<double> dval(nz), dc(n), dlo(m), dup(m), dvl(n), dvu(n), x(n), y(m), rc(n), dx0, dy0;
  if (warm) {
    dx0.resize(n);
    dy0.resize(m);
  }
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  trace("batch: device allocation");
  {
    // Every instance's arrays go straight to their place in the batch arrays (consecutive
    // instances of one array travel as one copy); offsets, indices and instance ids are made
    // global on the device.
    staged_upload h2d(s);
    std::vector<host_piece> pieces(bi.count);
    auto gather = [&](auto* dst, auto&& piece_of) {
      for (int b = 0; b < bi.count; ++b) pieces[b] = piece_of(*ps[ids[b]], b);
      h2d.put_gather(dst, pieces);
    };
    gather(doff.data() + 1, [&](const lp_problem& p, int) {
      return host_piece{p.row_off.data() + 1, (size_t)p.m * sizeof(int)};
    });
    gather(didx.data(), [&](const lp_problem& p, int) {
      return host_piece{p.col_idx.data(), (size_t)p.row_off[p.m] * sizeof(int)};
    });
    gather(dval.data(), [&](const lp_problem& p, int) {
      return host_piece{p.val.data(), (size_t)p.row_off[p.m] * sizeof(double)};
    });
    gather(dc.data(), [&](const lp_problem& p, int) {
      return host_piece{p.c.data(), (size_t)p.n * sizeof(double)};
    });
    gather(dlo.data(), [&](const lp_problem& p, int b) {
      return host_piece{rb[ids[b]].lo, (size_t)p.m * sizeof(double)};
    });
    gather(dup.data(), [&](const lp_problem& p, int b) {
      return host_piece{rb[ids[b]].up, (size_t)p.m * sizeof(double)};
    });
    gather(dvl.data(), [&](const lp_problem& p, int) {
      return host_piece{p.var_lo.data(), (size_t)p.n * sizeof(double)};
    });
    gather(dvu.data(), [&](const lp_problem& p, int) {
      return host_piece{p.var_up.data(), (size_t)p.n * sizeof(double)};
    });
    if (warm) {
      gather(dx0.data(), [&](const lp_problem& p, int b) {
        return host_piece{(*warm)[b].x.data(), (size_t)p.n * sizeof(double)};
      });
      gather(dy0.data(), [&](const lp_problem& p, int b) {
        return host_piece{(*warm)[b].y.data(), (size_t)p.m * sizeof(double)};
      });
      bi.initial_primal = dx0.data();
      bi.initial_dual   = dy0.data();
      for (const batch_warm& w : *warm) {
        bi.initial_step.push_back(w.step);
        bi.initial_weight.push_back(w.weight);
      }
    }
    h2d.put(drs.data(), bi.row_start.data(), bi.count + 1);
    h2d.put(dcs.data(), bi.col_start.data(), bi.count + 1);
    h2d.put(des.data(), e0.data(), bi.count + 1);
    h2d.finish();
  }
  rebase_batch_arrays(bi.count, drs.data(), dcs.data(), des.data(), doff.data(), didx.data(),
                      dri.data(), dci.data(), s);
  bi.m        = m;
  bi.n        = n;
  bi.row_off  = doff.data();
  bi.col_idx  = didx.data();
  bi.val      = dval.data();
  bi.c        = dc.data();
  bi.con_lo   = dlo.data();
  bi.con_up   = dup.data();
  bi.var_lo   = dvl.data();
  bi.var_up   = dvu.data();
  bi.row_inst = dri.data();
  bi.col_inst = dci.data();
  trace("batch: upload");
  std::vector<pdlp_result> rs = pdlp_batch_solve_device(bi, prm, s, x.data(), y.data(), rc.data());
  host_array<double> hx(n), hy(m), hrc(n);
  staged_download(hx.data(), x.data(), n * sizeof(double), s);
  staged_download(hy.data(), y.data(), m * sizeof(double), s);
  staged_download(hrc.data(), rc.data(), n * sizeof(double), s);
  // Every instance's slices of the batch solution (independent copies, split over host threads).
  parallel_ranges(bi.count, [&](int b0, int b1) {
    for (int b = b0; b < b1; ++b) {
      lp_solution& o = out[ids[b]];
      o.r            = rs[b];
      o.r.x.assign(hx.begin() + bi.col_start[b], hx.begin() + bi.col_start[b + 1]);
      o.r.rc.assign(hrc.begin() + bi.col_start[b], hrc.begin() + bi.col_start[b + 1]);
      o.r.y.assign(hy.begin() + bi.row_start[b], hy.begin() + bi.row_start[b + 1]);
    }
  });
  // Instances whose FP32 iterates stalled continue, together, in FP64 from where they stopped:
  // their solutions, step sizes and primal weights start an FP64 batch.  With refinement asked
  // for (pdlp_refinement_passes > 0), the Optimal instances of a mixed batch continue with them,
  // and all of them to the refinement tolerance, as a single solve's FP64 continuation does.
  const bool refine = prm.precision == 1 && prm.refinement_passes > 0;
  std::vector<size_t> stalled;
  std::vector<batch_warm> restart;
  for (int b = 0; b < bi.count; ++b)
    if (rs[b].status == kStalled || (refine && rs[b].status == kOptimal)) {
      const lp_solution& o = out[ids[b]];
      batch_warm w;
      w.x.assign(o.r.x.begin(), o.r.x.end());
      w.y.assign(o.r.y.begin(), o.r.y.end());
      if (bi.maximize[b])  // returned duals are negated for maximisation
        for (double& v : w.y) v = -v;
      w.step   = rs[b].step_size;
      w.weight = rs[b].primal_weight;
      stalled.push_back(ids[b]);
      restart.push_back(std::move(w));
    }
  if (!stalled.empty()) {
    pdlp_params q = prm;
    q.precision   = 0;
    if (refine) {
      q.abs_primal = q.rel_primal = prm.refinement_tol;
      q.abs_dual = q.rel_dual = prm.refinement_tol;
      q.abs_gap = q.rel_gap = prm.refinement_tol;
    }
    q.time_limit  = std::max(
      0.0, prm.time_limit -
             std::chrono::duration<double>(std::chrono::steady_clock::now() - t_chunk).count());
    std::vector<int64_t> mixed_iters;
    for (int b = 0; b < bi.count; ++b)
      if (rs[b].status == kStalled || (refine && rs[b].status == kOptimal))
        mixed_iters.push_back(rs[b].iterations);
    solve_batch_chunk(ps, stalled, rb, q, false, out, &restart);
    for (size_t i = 0; i < stalled.size(); ++i) {
      out[stalled[i]].r.refinement_passes = 1;
      out[stalled[i]].r.iterations += mixed_iters[i];
    }
  }
  if (!crossover) return;
  // Crossover of the Optimal instances: all their active-set solves in one launch.
  std::vector<const lp_problem*> pp;
  std::vector<pdlp_result*> rr;
  for (int b = 0; b < bi.count; ++b) {
    lp_solution& o = out[ids[b]];
    if (o.r.status != CUOPT_TERIMINATION_STATUS_OPTIMAL) continue;
    pp.push_back(ps[ids[b]]);
    rr.push_back(&o.r);
  }
  const std::vector<bool> polished = vertex_polish_batch(pp, rr);
  for (size_t k = 0; k < rr.size(); ++k) rr[k]->crossover = polished[k];
}

std::vector<lp_solution> solve_batch(const std::vector<const lp_problem*>& ps, const lp_settings& st)
{
  std::vector<lp_solution> out(ps.size());
  // The block-diagonal batch evaluates l2 residuals only; the per-constraint criterion solves the
  // problems one at a time, as the reference's batch of independent solves does.
  if (st.b(CUOPT_PER_CONSTRAINT_RESIDUAL)) {
    for (size_t i = 0; i < ps.size(); ++i) out[i] = solve_problem(*ps[i], st);
    return out;
  }
  std::vector<row_bounds> rb(ps.size());
  std::vector<char> goes(ps.size(), 0);
  // Every problem is checked and prepared on its own (split over host threads).
  parallel_ranges((int)ps.size(), [&](int i0, int i1) {
    for (int i = i0; i < i1; ++i) {
      try {
        goes[i] = prepare_for_pdlp(*ps[i], st, rb[i], out[i]);
      } catch (const std::exception& e) {
        set_error(out[i], CUOPT_RUNTIME_ERROR, e.what());
      }
    }
  });
  std::vector<size_t> eligible;
  for (size_t i = 0; i < ps.size(); ++i)
    if (goes[i]) eligible.push_back(i);
  const pdlp_params prm = params_from_settings(st);
  // Chunks that fit the batch layout: at most 65535 instances and int32 totals.
  size_t pos = 0;
  while (pos < eligible.size()) {
    std::vector<size_t> chunk;
    int64_t m = 0, n = 0, nnz = 0;
    while (pos < eligible.size() && chunk.size() < 65535) {
      const lp_problem& p = *ps[eligible[pos]];
      if (!chunk.empty() && (m + p.m >= INT_MAX || n + p.n >= INT_MAX ||
                             nnz + p.row_off[p.m] >= INT_MAX))
        break;
      m += p.m;
      n += p.n;
      nnz += p.row_off[p.m];
      chunk.push_back(eligible[pos++]);
    }
    try {
      solve_batch_chunk(ps, chunk, rb, prm, st.b(CUOPT_CROSSOVER), out);
    } catch (const std::bad_alloc&) {
      for (size_t id : chunk) set_error(out[id], CUOPT_OUT_OF_MEMORY, "Memory allocation failed");
    } catch (const std::invalid_argument& e) {
      for (size_t id : chunk) set_error(out[id], CUOPT_VALIDATION_ERROR, e.what());
    } catch (const std::exception& e) {
      for (size_t id : chunk) set_error(out[id], CUOPT_RUNTIME_ERROR, e.what());
    }
  }
  return out;
}

std::vector<lp_solution> solve_climbers(const lp_problem& p, const lp_settings& st,
                                        const std::vector<int>& var, const std::vector<double>& lo,
                                        const std::vector<double>& up, const climber_start* start)
{
  const int count = (int)var.size();
  std::vector<lp_solution> out(count);
  if (st.b(CUOPT_PER_CONSTRAINT_RESIDUAL)) {  // as the reference (convergence_information.cu:393-395)
    for (auto& o : out)
      set_error(o, CUOPT_VALIDATION_ERROR, "Batch mode not supported for per_constraint_residual");
    return out;
  }
  for (int b = 0; b < count; ++b)
    if (var[b] < 0 || var[b] >= p.n) {
      for (auto& o : out) set_error(o, CUOPT_INVALID_ARGUMENT, "climber variable out of range");
      return out;
    }
  auto modified = [&](int b) {
    lp_problem q    = p;
    q.var_lo[var[b]] = lo[b];
    q.var_up[var[b]] = up[b];
    return q;
  };
  row_bounds rb;
  lp_solution base;
  bool reaches = false;
  try {
    reaches = prepare_for_pdlp(p, st, rb, base);
  } catch (const std::exception& e) {
    set_error(base, CUOPT_RUNTIME_ERROR, e.what());
  }
  if (!reaches || base.error_code != CUOPT_SUCCESS) {
    // The base LP does not go to PDLP (no constraints, validation error, ...): every climber is
    // answered like a single solve of its LP.
    for (int b = 0; b < count; ++b) out[b] = solve_problem(modified(b), st);
    return out;
  }
  try {
    const int m = p.m, n = p.n;
    const int64_t nnz = p.row_off[m];
    cudaStream_t s;
    B200_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct stream_guard {
      cudaStream_t s;
      ~stream_guard() { cudaStreamDestroy(s); }
    } guard{s};
    alloc_scope scope(s);
    configure_pool_once();
    const size_t nz = (size_t)std::max<int64_t>(nnz, 1);
    dbuf<int> doff(m + 1), didx(nz);
    dbuf<double> dval(nz), dc(n), dlo(m), dup(m), dvl(n), dvu(n);
    {
      staged_upload h2d(s);
      h2d.put(doff.data(), p.row_off.data(), m + 1);
      h2d.put(didx.data(), p.col_idx.data(), nnz);
      h2d.put(dval.data(), p.val.data(), nnz);
      h2d.put(dc.data(), p.c.data(), n);
      h2d.put(dlo.data(), rb.lo, m);
      h2d.put(dup.data(), rb.up, m);
      h2d.put(dvl.data(), p.var_lo.data(), n);
      h2d.put(dvu.data(), p.var_up.data(), n);
      h2d.finish();
    }
    lp_device_input in;
    in.m          = m;
    in.n          = n;
    in.row_off    = doff.data();
    in.col_idx    = didx.data();
    in.val        = dval.data();
    in.c          = dc.data();
    in.con_lo     = dlo.data();
    in.con_up     = dup.data();
    in.var_lo     = dvl.data();
    in.var_up     = dvu.data();
    in.obj_offset = p.obj_offset;
    in.maximize   = p.maximize;
    pdlp_params prm = params_from_settings(st);
    const std::vector<double>* x0 = start ? &start->x : &st.initial_primal;
    const std::vector<double>* y0 = start ? &start->y : &st.initial_dual;
    if (start) {
      prm.initial_step_size     = start->step_size;
      prm.initial_primal_weight = start->primal_weight;
    }
    dbuf<double> dx0, dy0;
    if ((int)x0->size() == n) {
      dx0.resize(n);
      dx0.upload(x0->data(), n, s);
      in.initial_primal = dx0.data();
    }
    if ((int)y0->size() == m) {
      dy0.resize(m);
      dy0.upload(y0->data(), m, s);
      in.initial_dual = dy0.data();
    }
    std::vector<double> hx((size_t)count * n), hy((size_t)count * m), hrc((size_t)count * n);
    std::vector<pdlp_result> rs =
      pdlp_climber_solve_device(in, prm, var, lo, up, s, hx.data(), hy.data(), hrc.data());
    for (int b = 0; b < count; ++b) {
      out[b].r = rs[b];
      if (rs[b].status == CUOPT_TERIMINATION_STATUS_INFEASIBLE && rs[b].iterations == 0)
        continue;  // crossing bounds: no solution vectors, as for a single solve
      out[b].r.x.assign(hx.begin() + (size_t)b * n, hx.begin() + (size_t)(b + 1) * n);
      out[b].r.rc.assign(hrc.begin() + (size_t)b * n, hrc.begin() + (size_t)(b + 1) * n);
      out[b].r.y.assign(hy.begin() + (size_t)b * m, hy.begin() + (size_t)(b + 1) * m);
    }
    if (st.b(CUOPT_CROSSOVER)) {  // all the Optimal climbers' active-set solves in one launch
      std::vector<lp_problem> mods;
      std::vector<int> which;
      for (int b = 0; b < count; ++b)
        if (out[b].r.status == CUOPT_TERIMINATION_STATUS_OPTIMAL && !out[b].r.x.empty()) {
          mods.push_back(modified(b));
          which.push_back(b);
        }
      std::vector<const lp_problem*> pp;
      std::vector<pdlp_result*> rr;
      for (size_t k = 0; k < which.size(); ++k) {
        pp.push_back(&mods[k]);
        rr.push_back(&out[which[k]].r);
      }
      const std::vector<bool> polished = vertex_polish_batch(pp, rr);
      for (size_t k = 0; k < which.size(); ++k) out[which[k]].r.crossover = polished[k];
    }
  } catch (const std::bad_alloc&) {
    for (auto& o : out) set_error(o, CUOPT_OUT_OF_MEMORY, "Memory allocation failed");
  } catch (const std::invalid_argument& e) {
    for (auto& o : out) set_error(o, CUOPT_VALIDATION_ERROR, e.what());
  } catch (const std::exception& e) {
    for (auto& o : out) set_error(o, CUOPT_RUNTIME_ERROR, e.what());
  }
  return out;
}

std::vector<lp_solution> solve_strong_branching(const lp_problem& p, const lp_settings& st,
                                                const std::vector<int>& frac,
                                                const std::vector<double>& root)
{
  const int count = (int)frac.size();
  std::vector<int> var(2 * (size_t)count);
  std::vector<double> lo(2 * (size_t)count), up(2 * (size_t)count);
  for (int i = 0; i < count; ++i) {
    const int j = frac[i];
    if (j < 0 || j >= p.n) {
      std::vector<lp_solution> out(2 * (size_t)count);
      for (auto& o : out) set_error(o, CUOPT_INVALID_ARGUMENT, "fractional variable out of range");
      return out;
    }
    var[i]         = j;
    lo[i]          = p.var_lo[j];
    up[i]          = std::floor(root[i]);
    var[count + i] = j;
    lo[count + i]  = std::ceil(root[i]);
    up[count + i]  = p.var_up[j];
  }
  // The settings run_batch_pdlp gives both solves (solve.cu:795-834).
  lp_settings sb = st;
  sb.set_int(CUOPT_METHOD, CUOPT_METHOD_PDLP);
  sb.set_int(CUOPT_PDLP_SOLVER_MODE, CUOPT_PDLP_SOLVER_MODE_STABLE3);
  sb.set_bool(CUOPT_INFEASIBILITY_DETECTION, false);
  sb.set_int(CUOPT_ITERATION_LIMIT, 100000);
  lp_settings base_settings = sb;
  base_settings.set_bool(CUOPT_CROSSOVER, false);
  lp_solution base = solve_problem(p, base_settings);
  ensure_host(base.r);
  climber_start start;
  if (base.error_code == CUOPT_SUCCESS && base.solved_by_pdlp && (int)base.r.x.size() == p.n &&
      (int)base.r.y.size() == p.m) {
    start.x.assign(base.r.x.begin(), base.r.x.end());
    start.y.assign(base.r.y.begin(), base.r.y.end());
    start.step_size     = base.r.step_size;
    start.primal_weight = base.r.primal_weight;
  }
  return solve_climbers(p, sb, var, lo, up, start.x.empty() ? nullptr : &start);
}

}  // namespace cuopt_b200
