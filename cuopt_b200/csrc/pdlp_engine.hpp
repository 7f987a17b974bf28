// PDLP engine interface used by the C API layer.
//
// Counterpart of the reference's solve_lp -> run_pdlp -> pdlp_solver_t::run_solver chain
// (cpp/src/pdlp/solve.cu:556-590, 1124-1342; cpp/src/pdlp/pdlp.cu:2013-2457).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <limits>
#include <memory>
#include <vector>

#include "host_array.hpp"

namespace cuopt_b200 {

// The LP as handed over by the C interface: user order, minimise or maximise,
// con_lo <= A x <= con_up, var_lo <= x <= var_up.
// Device copies of a problem's arrays in the user's order, made when the problem is created from
// pinned host memory or device memory (the reference keeps its problems on the device too); a
// host-path solve on the same device reads them instead of uploading.  Null members were not
// copied.  The arrays live in one allocation, released with the object.
struct device_problem {
  int device         = -1;
  void* base         = nullptr;
  const int* row_off = nullptr;
  const int* col_idx = nullptr;
  const double* val  = nullptr;
  const double* c = nullptr, *var_lo = nullptr, *var_up = nullptr;
  const double* con_lo = nullptr, *con_up = nullptr;
  device_problem() = default;
  device_problem(const device_problem&)            = delete;
  device_problem& operator=(const device_problem&) = delete;
  ~device_problem();
};

struct lp_input {
  const device_problem* dev = nullptr;  // optional device copy of the arrays below
  int m = 0, n = 0;
  const int* row_off    = nullptr;  // m + 1
  const int* col_idx    = nullptr;  // nnz
  const double* val     = nullptr;  // nnz
  const double* c       = nullptr;  // n
  const double* con_lo  = nullptr;  // m
  const double* con_up  = nullptr;  // m
  const double* var_lo  = nullptr;  // n
  const double* var_up  = nullptr;  // n
  double obj_offset     = 0.0;
  bool maximize         = false;
};

struct pdlp_params {
  double abs_primal = 1e-4, rel_primal = 1e-4;
  double abs_dual = 1e-4, rel_dual = 1e-4;
  double abs_gap = 1e-4, rel_gap = 1e-4;
  int64_t iteration_limit = 2147483647;
  double time_limit       = 1e300;
  int precision           = 0;  // 0 FP64, 1 mixed FP32/FP64
  int refinement_passes   = 0;
  int tiled_sweeps        = -1;  // mixed precision: -1 autotuned, 0 sliced ELL only, 1 tiled
  int persistent          = -1;  // plain iterations: -1 timed, 0 graphs, 1 persistent, 2 cluster
  int sweep_wpb           = 0;  // plain sweeps: warps per block (0: chosen by timing 4, 8, 16)
  double refinement_tol   = 1e-8;
  bool log_to_console     = false;
  // Infeasibility detection (CUOPT_INFEASIBILITY_DETECTION and its two tolerances).
  bool detect_infeasibility   = false;
  double primal_infeasible_tol = 1e-10;
  double dual_infeasible_tol   = 1e-10;
  // CUOPT_PER_CONSTRAINT_RESIDUAL: the primal / dual tests (and the reported residuals) use the
  // per-constraint maxima instead of the l2 norms.
  bool per_constraint_residual = false;
  std::vector<double> initial_primal;  // user order, optional
  std::vector<double> initial_dual;    // user order, optional
  // Given by the warm start of a strong-branching batch (the reference's run_batch_pdlp,
  // cpp/src/pdlp/solve.cu:743-882, and pdlp.cu:2027-2083): a finite step size replaces the power
  // iteration, a finite primal weight the initial 1 (and the best weight of the PID controller).
  double initial_step_size     = std::numeric_limits<double>::quiet_NaN();
  double initial_primal_weight = std::numeric_limits<double>::quiet_NaN();
};

// A solution's x, y and reduced costs left on the device by a host-path solve (user order, the
// signs the user sees), as the reference keeps its solutions: getters copy from it straight to the
// caller's buffer, and host code that needs the vectors downloads them first (ensure_host).
struct device_solution {
  int device    = -1;
  void* base    = nullptr;
  double* x     = nullptr;
  double* y     = nullptr;
  double* rc    = nullptr;
  int n = 0, m = 0;
  device_solution() = default;
  device_solution(const device_solution&)            = delete;
  device_solution& operator=(const device_solution&) = delete;
  ~device_solution();
};

struct pdlp_result {
  int status = 0;  // CUOPT_TERIMINATION_STATUS_*
  host_array<double> x, y, rc;  // user order (empty while they are only on the device, `dev`)
  std::shared_ptr<const device_solution> dev;
  int64_t iterations = 0;
  double primal_obj = 0, dual_obj = 0;
  double l2_primal = 0, l2_dual = 0, rel_primal = 0, rel_dual = 0, gap = 0, rel_gap = 0;
  double solve_time = 0, setup_time = 0, loop_time = 0;
  double step_size = 0, primal_weight = 0;
  int restarts = 0, power_iterations = 0, refinement_passes = 0;
  bool crossover = false;  // the solution was replaced by the vertex of its active set
  double kernel_launches = 0;
  // Form of the plain iterations: 0 CUDA graphs, 1 persistent kernel (its grid in blocks), 2
  // cluster-resident kernel, and
  // the median microseconds per iteration of the check-to-check cycles each form ran while the
  // choice was made (0 where it was not timed).
  int plain_form = 0, persistent_blocks = 0;
  double us_plain_graphs = 0, us_plain_persistent = 0, us_plain_cluster = 0;
  // Warps per block of the plain primal / dual sweeps and the ms per launch measured with 4, 8
  // and 16 warps per block (0 where not timed).
  int wpb_primal = 8, wpb_dual = 8;
  double wpb_ms[2][3] = {{0, 0, 0}, {0, 0, 0}};
};

struct sweep_profile {
  double ms_primal = 0, ms_dual = 0, bytes_primal = 0, bytes_dual = 0;
  // Per row-length class, for the primal sweep (classes[0], rows of A^T) and the dual sweep
  // (classes[1], rows of A): [0] rows in the long class (warp per row), [1] their non-zeros,
  // [2] ms of the long-row blocks launched alone, [3] rows in slices, [4] their non-zeros, [5]
  // stored slice elements (padding included), [6] ms of the slice blocks launched alone.
  double classes[2][7] = {};
};

// The same LP with every array in device memory (user order).
struct lp_device_input {
  int m = 0, n = 0;
  const int* row_off   = nullptr;
  const int* col_idx   = nullptr;
  const double* val    = nullptr;
  const double* c      = nullptr;
  const double* con_lo = nullptr;
  const double* con_up = nullptr;
  const double* var_lo = nullptr;
  const double* var_up = nullptr;
  double obj_offset    = 0.0;
  bool maximize        = false;
  const double* initial_primal = nullptr;  // optional, n (user order)
  const double* initial_dual   = nullptr;  // optional, m
};

// Runs PDLP (Stable3) on the GPU from host arrays (uploads them, returns x / y / rc on the host).
// Throws std::exception subclasses on CUDA or input errors.
// A block-diagonal batch of `count` independent LPs on the device: the CSR concatenates the
// instances' rows with global column indices; row_inst / col_inst give every user row / column
// its instance (device); row_start / col_start (host, count + 1) delimit the instances.
struct batch_device_input {
  int count = 0;
  int m = 0, n = 0;
  const int* row_off   = nullptr;
  const int* col_idx   = nullptr;
  const double* val    = nullptr;
  const double* c      = nullptr;
  const double* con_lo = nullptr;
  const double* con_up = nullptr;
  const double* var_lo = nullptr;
  const double* var_up = nullptr;
  const int* row_inst  = nullptr;
  const int* col_inst  = nullptr;
  std::vector<int> row_start, col_start;
  std::vector<double> obj_offset;
  std::vector<char> maximize;
  // Optional warm start (used to continue instances whose FP32 iterates stalled, in FP64):
  // initial primal / dual solutions in the batch's user order (device, n / m; duals in the
  // solver's sign convention), and per instance the step size and primal weight to start from.
  const double* initial_primal = nullptr;
  const double* initial_dual   = nullptr;
  std::vector<double> initial_step, initial_weight;
};

// Arrays of a batch uploaded instance by instance (instance b's rows from row_start[b], columns
// from col_start[b], non-zeros from nnz_start[b]; all three device arrays of count + 1 entries):
// makes the row offsets and column indices global and fills the instance of every row / column.
void rebase_batch_arrays(int count, const int* row_start, const int* col_start,
                         const int* nnz_start, int* row_off, int* col_idx, int* row_inst,
                         int* col_inst, cudaStream_t s);

pdlp_result pdlp_solve(const lp_input& in, const pdlp_params& p);

// Solves every instance of the batch with its own Stable3 state; x / y / reduced costs are written
// to device arrays of the batch's total sizes (user order, instances concatenated).
std::vector<pdlp_result> pdlp_batch_solve_device(const batch_device_input& in,
                                                 const pdlp_params& p, cudaStream_t stream,
                                                 double* x_out, double* y_out, double* rc_out);

// Runs PDLP on device-resident arrays.  x_out (n), y_out (m), rc_out (n) are device arrays in the
// user's order; the returned result carries statistics only (its x / y / rc stay empty).
pdlp_result pdlp_solve_device(const lp_device_input& in, const pdlp_params& p, cudaStream_t stream,
                              double* x_out, double* y_out, double* rc_out);

// Times `iterations` plain iterations sweep by sweep (see cuOptProfilePDHGSweeps).
// Climber batch (strong branching): the LP of `in` solved once per climber b with variable var[b]
// (user order) bounded by [lo[b], up[b]] instead; FP64.  x_out (B x n), y_out (B x m) and rc_out
// (B x n) are host arrays, climber-major, user order.
std::vector<pdlp_result> pdlp_climber_solve_device(const lp_device_input& in, const pdlp_params& p,
                                                   const std::vector<int>& var,
                                                   const std::vector<double>& lo,
                                                   const std::vector<double>& up,
                                                   cudaStream_t stream, double* x_out,
                                                   double* y_out, double* rc_out);

sweep_profile pdlp_profile_sweeps(const lp_device_input& in, const pdlp_params& p,
                                  cudaStream_t stream, int iterations);

// Fills r.x / r.y / r.rc from r.dev when the vectors are only on the device (then drops it).
void ensure_host(pdlp_result& r);

// Copies r's x (which 0), y (1) or reduced costs (2) to dst (host or device memory of any kind),
// from the device when the vectors are there.
void copy_solution_vector(const pdlp_result& r, int which, double* dst);

}  // namespace cuopt_b200
