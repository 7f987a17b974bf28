// Host-side objects behind the opaque C handles.
#pragma once

#include <cstdint>
#include <memory>
#include <utility>
#include <string>
#include <vector>

#include "pdlp_engine.hpp"

namespace cuopt_b200 {

// cuOptOptimizationProblem: the user's LP, copied at creation (reference optimization_problem_t,
// cpp/include/cuopt/linear_programming/optimization_problem.hpp:160-319).


struct lp_problem {
  int m = 0, n = 0;
  bool maximize     = false;
  double obj_offset = 0.0;
  host_array<double> c;
  host_array<int> row_off, col_idx;
  host_array<double> val;
  bool ranged = false;           // true: con_lo / con_up given; false: row_types + rhs
  std::vector<char> row_types;   // 'E' 'L' 'G'
  host_array<double> rhs;
  host_array<double> con_lo, con_up;
  host_array<double> var_lo, var_up;
  std::vector<char> var_types;   // 'C' 'I'
  bool quadratic = false;
  std::vector<std::string> row_names, col_names;
  std::string name, objective_name;
  // Device copy made at creation (see device_problem).  A copy of the problem (e.g. one with a
  // variable's bounds changed) does not share it.
  struct mirror_ref {
    std::shared_ptr<const device_problem> p;
    mirror_ref() = default;
    mirror_ref(const mirror_ref&) {}
    mirror_ref& operator=(const mirror_ref&)
    {
      p.reset();
      return *this;
    }
    mirror_ref(mirror_ref&&) noexcept            = default;
    mirror_ref& operator=(mirror_ref&&) noexcept = default;
  } dev;

  // Constraint bounds as PDLP sees them (reference problem_helpers.cuh:26-51).
  void constraint_bounds(std::vector<double>& lo, std::vector<double>& up) const;
  bool is_mip() const;
};

// Parameter registry mirroring the reference's solver_settings_t
// (cpp/src/math_optimization/solver_settings.cu:55-135): names, ranges and defaults.
struct lp_settings {
  lp_settings();
  // Each returns 0 on success, CUOPT_INVALID_ARGUMENT otherwise.
  int set_from_string(const std::string& name, const std::string& value);
  int set_int(const std::string& name, int32_t v);
  int set_float(const std::string& name, double v);
  int set_bool(const std::string& name, bool v);
  int get_int(const std::string& name, int32_t& v) const;
  int get_float(const std::string& name, double& v) const;
  int get_bool(const std::string& name, bool& v) const;
  int get_as_string(const std::string& name, std::string& v) const;

  struct fparam { const char* name; double min, max, value; };
  struct iparam { const char* name; int32_t min, max, value; };
  struct bparam { const char* name; bool value; };
  struct sparam { const char* name; std::string value; };
  std::vector<fparam> fparams;
  std::vector<iparam> iparams;
  std::vector<bparam> bparams;
  std::vector<sparam> sparams;

  double f(const char* name) const;
  int32_t i(const char* name) const;
  bool b(const char* name) const;

  std::vector<double> initial_primal, initial_dual;
};

// cuOptSolution
struct lp_solution {
  int error_code = 0;  // CUOPT_SUCCESS / CUOPT_VALIDATION_ERROR / ...
  std::string error_message;
  pdlp_result r;
  bool solved_by_pdlp = true;
};

// Validation of a problem before solving (reference pdlp/utilities/problem_checking.cu:20-300).
// Returns an empty string when valid, otherwise the reason.
std::string validate_problem(const lp_problem& p);

// Solver parameters from the settings registry.
pdlp_params params_from_settings(const lp_settings& s);
// Non-empty (a validation message) when the settings ask for a PDLP mode that is not built.
std::string solver_mode_error(const lp_settings& s);

// Full solve as done by cuOptSolve: validation, trivial cases, PDLP.
lp_solution solve_problem(const lp_problem& p, const lp_settings& s);

// Solves independent problems together: every problem that reaches PDLP joins one block-diagonal
// batch (per-instance Stable3 state); the others are answered as solve_problem would.
std::vector<lp_solution> solve_batch(const std::vector<const lp_problem*>& ps, const lp_settings& s);

// Starting point shared by the climbers of a batch: an initial solution in the user's order, and
// optionally the step size and primal weight to start from (NaN: computed / 1).
struct climber_start {
  std::vector<double> x, y;
  double step_size     = std::numeric_limits<double>::quiet_NaN();
  double primal_weight = std::numeric_limits<double>::quiet_NaN();
};

// Climber batch: the LP solved once per climber b with variable var[b] bounded by [lo[b], up[b]];
// all climbers share one matrix read per sweep (see climber_engine.cuh).  Without `start`, the
// settings' initial solution (if any) is every climber's starting point.
std::vector<lp_solution> solve_climbers(const lp_problem& p, const lp_settings& s,
                                        const std::vector<int>& var, const std::vector<double>& lo,
                                        const std::vector<double>& up,
                                        const climber_start* start = nullptr);

// Strong branching as the reference's batch_pdlp_solve / run_batch_pdlp do it
// (cpp/src/pdlp/solve.cu:743-919): the LP is solved once (Stable3, no infeasibility detection,
// iteration limit 100000), then the down branches (var[i] <= floor(root[i])) and the up branches
// (var[i] >= ceil(root[i])) run as one climber batch started from that solution, its step size and
// its primal weight, under the same limits.
std::vector<lp_solution> solve_strong_branching(const lp_problem& p, const lp_settings& s,
                                                const std::vector<int>& frac,
                                                const std::vector<double>& root);

// Reverse-mode sensitivities of an optimal solution (see adjoint.cu): gx (n) and optional gy (m)
// in; any of dc (n), dlo / dup (m, constraint bounds) and dval (nnz, CSR order) out.
void solution_adjoint(const lp_problem& p, const pdlp_result& sol, const double* gx,
                      const double* gy, double* dc, double* dlo, double* dup, double* dval);
// The same for many solutions at once: every active-set solve of the batch runs in one launch.
struct adjoint_job {
  const lp_problem* p;
  const pdlp_result* sol;
  const double* gx;
  const double* gy;
  double *dc, *dlo, *dup, *dval;
};
void solution_adjoint_batch(const std::vector<adjoint_job>& jobs);

// Crossover to a vertex on the solution's active set (see adjoint.cu): when the free variables
// and the constraints held at a bound form a square, non-singular system whose solution is primal
// and dual feasible, the solution is replaced by that exact vertex and true is returned; otherwise
// (a degenerate optimum) the solution is left unchanged.
bool vertex_polish(const lp_problem& p, pdlp_result& r);
// vertex_polish of many solutions, with all their active-set solves in one launch.
std::vector<bool> vertex_polish_batch(const std::vector<const lp_problem*>& ps,
                                      const std::vector<pdlp_result*>& rs);

// MPS input / output (reference cpp/libmps_parser).  read_mps returns 0 or CUOPT_MPS_* codes.
int read_mps(const std::string& path, lp_problem& out, std::string& err);
int write_mps(const lp_problem& p, const std::string& path);
// The reference's .sol output of a single solve (pdlp/solver_solution.cu:428-448,
// math_optimization/solution_writer.cu:16-40): "# Status: ..." (Optimal, Primal Feasible, or
// Infeasible for every other status) and, when feasible, "# Objective value: ..." and one
// "name value" line per named column.
int write_sol_file(const lp_problem& p, lp_solution& s, const std::string& path);

}  // namespace cuopt_b200
