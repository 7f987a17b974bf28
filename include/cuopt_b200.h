/*
 * cuopt_b200 extensions to the cuOpt LP C interface.
 *
 * These entry points sit beside the drop-in cuopt_c.h interface.  Each one names the reference
 * interface it replaces, or says that it has no counterpart in the reference.
 */
#ifndef CUOPT_B200_H
#define CUOPT_B200_H

#include <cuopt/linear_programming/cuopt_c.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Per-solve statistics, the counterpart of optimization_problem_solution_t::
 * additional_termination_information_t (cpp/include/cuopt/linear_programming/pdlp/
 * solver_solution.hpp:53-93) plus the fields this library adds (power iterations, restarts,
 * refinement passes, device time of the iteration loop). */
typedef struct {
  cuopt_int_t number_of_steps_taken;
  cuopt_int_t total_number_of_attempted_steps;
  cuopt_float_t l2_primal_residual;
  cuopt_float_t l2_relative_primal_residual;
  cuopt_float_t l2_dual_residual;
  cuopt_float_t l2_relative_dual_residual;
  cuopt_float_t primal_objective;
  cuopt_float_t dual_objective;
  cuopt_float_t gap;
  cuopt_float_t relative_gap;
  cuopt_float_t solve_time;
  cuopt_int_t solved_by_pdlp;
  /* additions */
  cuopt_int_t restarts;
  cuopt_int_t power_iterations;
  cuopt_int_t refinement_passes;
  cuopt_float_t step_size;
  cuopt_float_t primal_weight;
  cuopt_float_t setup_time;     /* seconds spent before the first PDHG iteration */
  cuopt_float_t loop_time;      /* seconds spent in the iteration loop */
  cuopt_float_t kernel_launches; /* kernels this library launched for the solve */
  cuopt_int_t crossover;         /* 1: the solution is the vertex of its active set ("crossover") */
  /* Form of the plain iterations between termination checks (pdlp_persistent_iterations): 0
   * CUDA-graph replays, 1 one persistent cooperative launch per run, 2 one thread-block cluster
   * per run with the gathered vectors in shared memory (small LPs), -1 still undecided when the
   * solve ended; the persistent grid in blocks; and the median microseconds per iteration of the
   * check-to-check cycles (major steps and launch boundaries included) that each form ran while
   * the choice was made (0 where it was not timed). */
  cuopt_int_t plain_iteration_form;
  cuopt_int_t persistent_blocks;
  cuopt_float_t plain_iteration_us_graphs;
  cuopt_float_t plain_iteration_us_persistent;
  cuopt_float_t plain_iteration_us_cluster;
  /* Warps per block of the plain primal and dual sweeps (pdlp_sweep_warps_per_block), and the
   * milliseconds per launch each shape took when they were chosen: primal with 4, 8, 16 warps,
   * then dual with 4, 8, 16 (0 where not timed). */
  cuopt_int_t sweep_warps_per_block_primal;
  cuopt_int_t sweep_warps_per_block_dual;
  cuopt_float_t sweep_block_shape_ms[6];
} cuOptPDLPStatistics;

cuopt_int_t cuOptGetPDLPStatistics(cuOptSolution solution, cuOptPDLPStatistics* stats);

/* Solve an LP whose arrays all live in device memory, writing the solution to device memory.
 * Counterpart of the reference's C++ entry solve_lp(optimization_problem_t&, settings)
 * (cpp/include/cuopt/linear_programming/solve.hpp:42-47), whose problem setters accept device
 * pointers; the reference C API has no device-resident variant.  Inputs are in the user's order
 * (CSR rows = constraints); `stream` is a cudaStream_t (NULL: the legacy default stream).  The
 * arrays are read, never modified or kept.  d_primal (n), d_dual (m), d_reduced_cost (n) receive the
 * solution; `stats` and `termination_status` may be NULL.  Returns CUOPT_SUCCESS or an error code
 * (CUOPT_VALIDATION_ERROR for inconsistent sizes or column indices out of range). */
cuopt_int_t cuOptSolveDevice(cuopt_int_t num_constraints,
                             cuopt_int_t num_variables,
                             cuopt_int_t objective_sense,
                             cuopt_float_t objective_offset,
                             const cuopt_float_t* d_objective_coefficients,
                             const cuopt_int_t* d_row_offsets,
                             const cuopt_int_t* d_column_indices,
                             const cuopt_float_t* d_values,
                             const cuopt_float_t* d_constraint_lower_bounds,
                             const cuopt_float_t* d_constraint_upper_bounds,
                             const cuopt_float_t* d_variable_lower_bounds,
                             const cuopt_float_t* d_variable_upper_bounds,
                             cuOptSolverSettings settings,
                             void* stream,
                             cuopt_float_t* d_primal,
                             cuopt_float_t* d_dual,
                             cuopt_float_t* d_reduced_cost,
                             cuOptPDLPStatistics* stats,
                             cuopt_int_t* termination_status);

/* Measurement hook (no counterpart in the reference): the same index stream as
 * cuOptProfileGatherRate, but every index receives an atomic add whose result is unused (a
 * fire-and-forget reduction into the vector), with 1, 2 and 4 chunks in flight.  Returns the best
 * rate in reductions per second: the rate a sweep that scatters its products instead of gathering
 * its operand would face. */
cuopt_int_t cuOptProfileScatterRate(cuopt_int_t vector_length,
                                    int64_t scatters,
                                    cuopt_int_t element_bytes,
                                    void* stream,
                                    cuopt_float_t* scatters_per_second,
                                    cuopt_int_t* chunks_in_flight);

/* Measurement and test hook (no counterpart in the reference): the grid barrier that the
 * persistent plain-iteration kernel (pdlp_persistent_iterations) places after every sweep, run
 * alone.  A cooperative launch of `blocks` blocks of 256 threads (at most the co-resident count)
 * passes `rounds` barriers.  With `unreachable` != 0 every barrier waits for one arrival more than
 * the grid has, so no barrier can complete: each wait ends at the launch's deadline (`budget_ms`
 * after its start, at most 10 s) and records status 1 (2 if its poll limit came first) instead of
 * hanging.  Returns the recorded status (0: every barrier completed) and the device time from the
 * first block's start to its end, in milliseconds. */
cuopt_int_t cuOptProbeGridBarrier(cuopt_int_t blocks,
                                  cuopt_int_t rounds,
                                  cuopt_int_t unreachable,
                                  cuopt_float_t budget_ms,
                                  void* stream,
                                  cuopt_int_t* status,
                                  cuopt_float_t* elapsed_ms);

/* Measurement hook (no counterpart in the reference): the cluster barrier that the cluster-resident
 * kernels (small LPs) place between their steps, run alone: one cluster of `blocks` (1 to 16)
 * blocks of `threads` threads passes `rounds` barriers.  Returns the device time from the first
 * block's start to its end, in milliseconds (CUOPT_INVALID_ARGUMENT where the device cannot run
 * such a cluster). */
cuopt_int_t cuOptProbeClusterBarrier(cuopt_int_t blocks,
                                     cuopt_int_t threads,
                                     cuopt_int_t rounds,
                                     void* stream,
                                     cuopt_float_t* elapsed_ms);

/* Measurement hook (no counterpart in the reference): the random-gather ceiling of the device.
 * Streams `gathers` random int32 indices into a vector of `vector_length` elements of
 * `element_bytes` (4 or 8) bytes, in the sliced-ELL sweeps' chunk shape (a warp reads 32 lanes x 4
 * indices with evict-first loads, then gathers the elements they name), with 1, 2, 4 and 8 chunks
 * in flight per thread.  Returns the best rate in gathers per second and the chunk count that gave
 * it.  On uniformly random sparsity this rate, not HBM bandwidth, bounds the fused sweeps. */
cuopt_int_t cuOptProfileGatherRate(cuopt_int_t vector_length,
                                   int64_t gathers,
                                   cuopt_int_t element_bytes,
                                   void* stream,
                                   cuopt_float_t* gathers_per_second,
                                   cuopt_int_t* chunks_in_flight);

/* Measurement hook (no counterpart in the reference): the plain sweeps of cuOptProfilePDHGSweeps
 * split by row-length class.  After the same preparation, the long-row blocks (one warp per row)
 * and the slice blocks (32-row slices) of each sweep are launched alone, `iterations` times each
 * after a warm-up, with 8 warps per block.  out (14 values): for the primal sweep (rows of A^T),
 * then the dual sweep (rows of A): rows in the long class, their non-zeros, ms per launch of the
 * long-row blocks, rows in slices, their non-zeros, stored slice elements (padding included), ms
 * per launch of the slice blocks. */
cuopt_int_t cuOptProfileSweepClasses(cuopt_int_t num_constraints,
                                     cuopt_int_t num_variables,
                                     const cuopt_float_t* d_objective_coefficients,
                                     const cuopt_int_t* d_row_offsets,
                                     const cuopt_int_t* d_column_indices,
                                     const cuopt_float_t* d_values,
                                     const cuopt_float_t* d_constraint_lower_bounds,
                                     const cuopt_float_t* d_constraint_upper_bounds,
                                     const cuopt_float_t* d_variable_lower_bounds,
                                     const cuopt_float_t* d_variable_upper_bounds,
                                     cuOptSolverSettings settings,
                                     void* stream,
                                     cuopt_int_t iterations,
                                     double* out);

/* Measurement hook (no counterpart in the reference): prepares the device-resident LP exactly as
 * cuOptSolveDevice does, then runs `iterations` plain PDHG iterations launching the two fused
 * sweeps separately between CUDA events on `stream`.  Returns the mean device time of one primal
 * sweep (A^T y fused with the primal projection / reflection / Halpern step) and of one dual sweep
 * (A x_bar fused with the dual step), in milliseconds, and the algorithmic bytes each sweep must
 * move (matrix values and indices, row offsets, one gather pass, the epilogue's vector reads and
 * writes). */
cuopt_int_t cuOptProfilePDHGSweeps(cuopt_int_t num_constraints,
                                   cuopt_int_t num_variables,
                                   const cuopt_float_t* d_objective_coefficients,
                                   const cuopt_int_t* d_row_offsets,
                                   const cuopt_int_t* d_column_indices,
                                   const cuopt_float_t* d_values,
                                   const cuopt_float_t* d_constraint_lower_bounds,
                                   const cuopt_float_t* d_constraint_upper_bounds,
                                   const cuopt_float_t* d_variable_lower_bounds,
                                   const cuopt_float_t* d_variable_upper_bounds,
                                   cuOptSolverSettings settings,
                                   void* stream,
                                   cuopt_int_t iterations,
                                   double* ms_primal_sweep,
                                   double* ms_dual_sweep,
                                   double* bytes_primal_sweep,
                                   double* bytes_dual_sweep);

/* Solve `count` independent LPs in one call.  The counterpart of the reference's
 * cuopt::cython::call_batch_solve (cpp/src/pdlp/utilities/cython_solve.cu:317-352, used by the
 * Python BatchSolve, python/cuopt/cuopt/linear_programming/solver/solver.py:109), which runs the
 * problems on up to four host threads.  Here the instances form one block-diagonal LP: every PDHG
 * sweep is one launch over all of them, each keeping its own scaling, step size, restarts and
 * termination (and its single-solve iterates); finished instances drop out of the sweeps.
 * solutions[i] receives the solution of
 * problems[i]; each must be released with cuOptDestroySolution.  Returns CUOPT_SUCCESS when every
 * instance ran (inspect each termination status), or the first error code. */
cuopt_int_t cuOptBatchSolve(const cuOptOptimizationProblem* problems,
                            cuopt_int_t count,
                            cuOptSolverSettings settings,
                            cuOptSolution* solutions);

/* Climber batch (strong branching): solves `count` copies of `problem` that differ only in the
 * bounds of one variable each: copy i has variable variable_indices[i] bounded by
 * [lower_bounds[i], upper_bounds[i]].  Counterpart of the reference's pdlp_solver_settings_t::
 * new_bounds with solve_lp in batch mode (cpp/src/pdlp/solve.cu:1124-1342, pdlp.cu:1447-1746).
 * All copies share one read of the matrix per PDHG sweep; each follows the iterates of a single
 * solve of its LP (FP64), starting from the settings' initial solution when one is set.  A copy
 * whose bounds cross is PrimalInfeasible without iterating.  solutions[i] receives copy i's
 * solution (release with cuOptDestroySolution).  Returns CUOPT_SUCCESS or the first error code. */
cuopt_int_t cuOptSolveClimbers(cuOptOptimizationProblem problem,
                               cuOptSolverSettings settings,
                               cuopt_int_t count,
                               const cuopt_int_t* variable_indices,
                               const cuopt_float_t* lower_bounds,
                               const cuopt_float_t* upper_bounds,
                               cuOptSolution* solutions);

/* Strong branching on `count` fractional variables (counterpart of the reference's
 * batch_pdlp_solve and run_batch_pdlp, cpp/src/pdlp/solve.cu:743-919): solutions[0 .. count) are
 * the down branches (fractional[i] bounded above by floor(root_solution[i])),
 * solutions[count .. 2 count) the up branches (bounded below by ceil(root_solution[i]));
 * `solutions` holds 2 * count handles.  As in the reference, the LP itself is solved first
 * (Stable3, no infeasibility detection, iteration limit 100000) and every branch starts from its
 * solution, step size and primal weight, under the same limits. */
cuopt_int_t cuOptBatchPDLPStrongBranching(cuOptOptimizationProblem problem,
                                          cuOptSolverSettings settings,
                                          cuopt_int_t count,
                                          const cuopt_int_t* fractional,
                                          const cuopt_float_t* root_solution,
                                          cuOptSolution* solutions);

/* Reverse-mode sensitivity of an optimal LP solution (no counterpart in the reference).
 * Given dL/dx (size n) and optionally dL/dy (size m, may be NULL) at the solution returned by
 * cuOptSolve, computes dL/dc (n), dL/dlower and dL/dupper of the constraint bounds (m each) and
 * dL/dA for every stored non-zero of the constraint matrix (nnz, CSR order of the problem), by
 * implicit differentiation of the KKT conditions on the solution's active set.  For a row whose
 * bounds are equal, the gradient with respect to its right-hand side is in dl_dlower.  At a
 * non-degenerate vertex these are the exact derivatives; otherwise those of the minimum-norm
 * response (in the equilibrated variables).  The active-set solves are matrix-free: LSQR on the
 * GPU, one thread block per system.  Any output pointer may be NULL.  Returns
 * CUOPT_INVALID_ARGUMENT if the solution is not Optimal. */
cuopt_int_t cuOptSolutionAdjoint(cuOptOptimizationProblem problem,
                                 cuOptSolution solution,
                                 const cuopt_float_t* dl_dx,
                                 const cuopt_float_t* dl_dy,
                                 cuopt_float_t* dl_dc,
                                 cuopt_float_t* dl_dlower,
                                 cuopt_float_t* dl_dupper,
                                 cuopt_float_t* dl_dvalues);

/* cuOptSolutionAdjoint for `count` (problem, solution) pairs at once (no counterpart in the
 * reference): every pointer argument is an array of `count` pointers with the meaning of the single
 * call's argument (dl_dx[i] required; dl_dy, the output arrays, or any of their entries may be
 * NULL).  All the active-set solves of the batch run in one launch, one thread block each.
 * Returns CUOPT_INVALID_ARGUMENT (and writes nothing) if any solution is not Optimal. */
cuopt_int_t cuOptSolutionAdjointBatch(cuopt_int_t count,
                                      const cuOptOptimizationProblem* problems,
                                      const cuOptSolution* solutions,
                                      const cuopt_float_t* const* dl_dx,
                                      const cuopt_float_t* const* dl_dy,
                                      cuopt_float_t* const* dl_dc,
                                      cuopt_float_t* const* dl_dlower,
                                      cuopt_float_t* const* dl_dupper,
                                      cuopt_float_t* const* dl_dvalues);

/* KKT errors of a given point, computed without allocating device memory (no counterpart in the
 * reference).  For an LP in device memory (user's CSR order, as for cuOptSolveDevice) and a point
 * (d_primal n, d_dual m, d_reduced_cost n, signs as cuOptSolveDevice returns them), writes to the
 * device array d_out (9 doubles), in stream order: l2 primal residual, l2 dual residual, primal
 * objective, dual objective, gap, relative primal residual, relative dual residual, relative gap
 * (the quantities of cuOptPDLPStatistics), and the count of malformed entries found (column
 * indices outside [0, n), rows whose offsets decrease or start below 0; when it is non-zero the
 * eight values are NaN).  d_row_offsets must start at 0 and end at the length of d_column_indices
 * and d_values: offsets past the arrays' end cannot be detected and are read as given.
 * For callers that cannot allocate: a memory pool that is already fully reserved, or a loop that
 * must not pay cudaMalloc's implicit synchronisation.
 * Scratch is a fixed static device array (about 4 MiB) held by every device that loads this
 * library until the process exits: num_variables may be at most 524288 (larger sizes return
 * CUOPT_INVALID_ARGUMENT with a message on stderr); constraints and non-zeros are not bounded.
 * The CUDA runtime loads the library's device code on a device at the first call that needs it,
 * so the first call on a device is when the static scratch takes its device memory: make it
 * before reserving the rest of the device's memory, and before any stream capture.  Calls that
 * overlap in time on one device share the scratch and race; order them.  A^T y is summed with
 * double-precision atomics, so the dual residual, the relative dual residual and the values
 * derived from them are not bit-reproducible between calls (they agree to rounding). */
cuopt_int_t cuOptComputeKKTErrorsNoAlloc(cuopt_int_t num_constraints,
                                         cuopt_int_t num_variables,
                                         cuopt_int_t objective_sense,
                                         cuopt_float_t objective_offset,
                                         const cuopt_float_t* d_objective_coefficients,
                                         const cuopt_int_t* d_row_offsets,
                                         const cuopt_int_t* d_column_indices,
                                         const cuopt_float_t* d_values,
                                         const cuopt_float_t* d_constraint_lower_bounds,
                                         const cuopt_float_t* d_constraint_upper_bounds,
                                         const cuopt_float_t* d_primal,
                                         const cuopt_float_t* d_dual,
                                         const cuopt_float_t* d_reduced_cost,
                                         void* stream,
                                         cuopt_float_t* d_out);

#ifdef __cplusplus
}
#endif

#endif /* CUOPT_B200_H */
