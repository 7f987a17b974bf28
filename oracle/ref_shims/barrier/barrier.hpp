// Stand-in for the GPU barrier solver's declarations.  Only solve_linear_program_with_barrier
// reaches it; the dual simplex entry point never does, and this stub reports a numerical issue.
#pragma once
#include <dual_simplex/presolve.hpp>
#include <dual_simplex/simplex_solver_settings.hpp>
#include <dual_simplex/solution.hpp>
#include <dual_simplex/solve.hpp>

namespace cuopt::linear_programming::dual_simplex {
template <typename i_t, typename f_t>
struct barrier_solver_settings_t {};
template <typename i_t, typename f_t>
class barrier_solver_t {
 public:
  template <typename... A>
  explicit barrier_solver_t(A&&...)
  {
  }
  template <typename... A>
  lp_status_t solve(A&&...)
  {
    return lp_status_t::NUMERICAL_ISSUES;
  }
};
}  // namespace cuopt::linear_programming::dual_simplex
