/*
 * cuopt_b200 — constants of the cuOpt LP C interface.
 *
 * The names and numeric values below must equal those of cuOpt 26.04
 * (cpp/include/cuopt/linear_programming/constants.h:17-160) so that code written against the
 * cuOpt C API compiles and behaves the same when linked against libcuopt_b200.so instead of
 * libcuopt.so.  Only the LP subset is implemented by this library; MIP / QP / barrier names are
 * kept so that existing callers still compile, and the library answers them with
 * CUOPT_INVALID_ARGUMENT or a validation-error solution.
 */
#ifndef CUOPT_CONSTANTS_H
#define CUOPT_CONSTANTS_H

#ifdef __cplusplus
#include <limits>
#else
#include <math.h>
#endif

#define CUOPT_INSTANTIATE_FLOAT  0
#define CUOPT_INSTANTIATE_DOUBLE 1
#define CUOPT_INSTANTIATE_INT32  1
#define CUOPT_INSTANTIATE_INT64  0

/* Parameter names (reference constants.h:23-76) */
#define CUOPT_ABSOLUTE_DUAL_TOLERANCE         "absolute_dual_tolerance"
#define CUOPT_RELATIVE_DUAL_TOLERANCE         "relative_dual_tolerance"
#define CUOPT_ABSOLUTE_PRIMAL_TOLERANCE       "absolute_primal_tolerance"
#define CUOPT_RELATIVE_PRIMAL_TOLERANCE       "relative_primal_tolerance"
#define CUOPT_ABSOLUTE_GAP_TOLERANCE          "absolute_gap_tolerance"
#define CUOPT_RELATIVE_GAP_TOLERANCE          "relative_gap_tolerance"
#define CUOPT_INFEASIBILITY_DETECTION         "infeasibility_detection"
#define CUOPT_STRICT_INFEASIBILITY            "strict_infeasibility"
#define CUOPT_PRIMAL_INFEASIBLE_TOLERANCE     "primal_infeasible_tolerance"
#define CUOPT_DUAL_INFEASIBLE_TOLERANCE       "dual_infeasible_tolerance"
#define CUOPT_ITERATION_LIMIT                 "iteration_limit"
#define CUOPT_TIME_LIMIT                      "time_limit"
#define CUOPT_WORK_LIMIT                      "work_limit"
#define CUOPT_PDLP_SOLVER_MODE                "pdlp_solver_mode"
#define CUOPT_METHOD                          "method"
#define CUOPT_PER_CONSTRAINT_RESIDUAL         "per_constraint_residual"
#define CUOPT_SAVE_BEST_PRIMAL_SO_FAR         "save_best_primal_so_far"
#define CUOPT_FIRST_PRIMAL_FEASIBLE           "first_primal_feasible"
#define CUOPT_LOG_FILE                        "log_file"
#define CUOPT_LOG_TO_CONSOLE                  "log_to_console"
#define CUOPT_CROSSOVER                       "crossover"
#define CUOPT_FOLDING                         "folding"
#define CUOPT_AUGMENTED                       "augmented"
#define CUOPT_DUALIZE                         "dualize"
#define CUOPT_ORDERING                        "ordering"
#define CUOPT_BARRIER_DUAL_INITIAL_POINT      "barrier_dual_initial_point"
#define CUOPT_ELIMINATE_DENSE_COLUMNS         "eliminate_dense_columns"
#define CUOPT_CUDSS_DETERMINISTIC             "cudss_deterministic"
#define CUOPT_PRESOLVE                        "presolve"
#define CUOPT_DUAL_POSTSOLVE                  "dual_postsolve"
#define CUOPT_MIP_DETERMINISM_MODE            "mip_determinism_mode"
#define CUOPT_MIP_ABSOLUTE_TOLERANCE          "mip_absolute_tolerance"
#define CUOPT_MIP_RELATIVE_TOLERANCE          "mip_relative_tolerance"
#define CUOPT_MIP_INTEGRALITY_TOLERANCE       "mip_integrality_tolerance"
#define CUOPT_MIP_ABSOLUTE_GAP                "mip_absolute_gap"
#define CUOPT_MIP_RELATIVE_GAP                "mip_relative_gap"
#define CUOPT_MIP_HEURISTICS_ONLY             "mip_heuristics_only"
#define CUOPT_MIP_SCALING                     "mip_scaling"
#define CUOPT_MIP_PRESOLVE                    "mip_presolve"
#define CUOPT_MIP_RELIABILITY_BRANCHING       "mip_reliability_branching"
#define CUOPT_MIP_CUT_PASSES                  "mip_cut_passes"
#define CUOPT_MIP_MIXED_INTEGER_ROUNDING_CUTS "mip_mixed_integer_rounding_cuts"
#define CUOPT_MIP_MIXED_INTEGER_GOMORY_CUTS   "mip_mixed_integer_gomory_cuts"
#define CUOPT_MIP_KNAPSACK_CUTS               "mip_knapsack_cuts"
#define CUOPT_MIP_STRONG_CHVATAL_GOMORY_CUTS  "mip_strong_chvatal_gomory_cuts"
#define CUOPT_MIP_REDUCED_COST_STRENGTHENING  "mip_reduced_cost_strengthening"
#define CUOPT_MIP_CUT_CHANGE_THRESHOLD        "mip_cut_change_threshold"
#define CUOPT_MIP_CUT_MIN_ORTHOGONALITY       "mip_cut_min_orthogonality"
#define CUOPT_MIP_BATCH_PDLP_STRONG_BRANCHING "mip_batch_pdlp_strong_branching"
#define CUOPT_SOLUTION_FILE                   "solution_file"
#define CUOPT_NUM_CPU_THREADS                 "num_cpu_threads"
#define CUOPT_NUM_GPUS                        "num_gpus"
#define CUOPT_USER_PROBLEM_FILE               "user_problem_file"
#define CUOPT_RANDOM_SEED                     "random_seed"

/* Parameters added by this library (no counterpart in the reference).  "pdlp_precision" picks the
 * arithmetic of the PDHG iterations: 0 = FP64 throughout (the reference's behaviour, default),
 * 1 = mixed (FP32 matrix and iterates, FP64 termination/restart/step ratio).
 * "pdlp_refinement_passes" (default 0 = off; any positive value = on) makes a mixed-precision solve
 * that reached its tolerances continue in FP64 from its solution (same scaling, step size and
 * primal weight) until "pdlp_refinement_tolerance" (default 1e-8) holds for all six relative
 * tolerances on the original LP, within the iteration and time limits. */
#define CUOPT_PDLP_PRECISION            "pdlp_precision"
#define CUOPT_PDLP_REFINEMENT_PASSES    "pdlp_refinement_passes"
#define CUOPT_PDLP_REFINEMENT_TOLERANCE "pdlp_refinement_tolerance"
#define CUOPT_PDLP_TILED_SWEEPS         "pdlp_tiled_sweeps"
#define CUOPT_PDLP_PRECISION_FP64  0
#define CUOPT_PDLP_PRECISION_MIXED 1
/* pdlp_tiled_sweeps (mixed precision): -1 chooses per sweep by timing both forms at setup,
 * 0 always uses the sliced-ELL sweeps, 1 uses the tiled sweeps wherever the matrix allows them */
#define CUOPT_PDLP_TILED_SWEEPS_AUTO -1
#define CUOPT_PDLP_TILED_SWEEPS_OFF  0
#define CUOPT_PDLP_TILED_SWEEPS_ON   1
/* pdlp_persistent_iterations: the runs of plain iterations between termination checks are
 * replayed from CUDA graphs (0), run by one persistent cooperative kernel launch with a grid
 * barrier after every sweep (1), or, for LPs whose two gathered vectors fit in one block's shared
 * memory, by one thread-block cluster that keeps them there (2; single LPs, not batches); -1
 * times the available forms on the first check-to-check cycles of a solve (the iterates are the
 * same either way) and keeps the fastest, remembered per problem shape.  A form that cannot run
 * on the problem falls back to 0. */
#define CUOPT_PDLP_PERSISTENT_ITERATIONS         "pdlp_persistent_iterations"
#define CUOPT_PDLP_PERSISTENT_ITERATIONS_AUTO    -1
#define CUOPT_PDLP_PERSISTENT_ITERATIONS_OFF     0
#define CUOPT_PDLP_PERSISTENT_ITERATIONS_ON      1
#define CUOPT_PDLP_PERSISTENT_ITERATIONS_CLUSTER 2
/* pdlp_sweep_warps_per_block: block shape of the plain sliced-ELL sweeps.  0 (default) chooses
 * 4, 8 or 16 warps per block by timing each sweep at the first solve of a problem shape; 4, 8 or
 * 16 fixes it (other values are a validation error).  The shape does not change any row's
 * arithmetic, so the iterates are the same for every choice. */
#define CUOPT_PDLP_SWEEP_WARPS_PER_BLOCK "pdlp_sweep_warps_per_block"

#define CUOPT_MODE_OPPORTUNISTIC 0
#define CUOPT_MODE_DETERMINISTIC 1

/* Termination status (reference constants.h:83-93; spelling kept as in the reference) */
#define CUOPT_TERIMINATION_STATUS_NO_TERMINATION   0
#define CUOPT_TERIMINATION_STATUS_OPTIMAL          1
#define CUOPT_TERIMINATION_STATUS_INFEASIBLE       2
#define CUOPT_TERIMINATION_STATUS_UNBOUNDED        3
#define CUOPT_TERIMINATION_STATUS_ITERATION_LIMIT  4
#define CUOPT_TERIMINATION_STATUS_TIME_LIMIT       5
#define CUOPT_TERIMINATION_STATUS_NUMERICAL_ERROR  6
#define CUOPT_TERIMINATION_STATUS_PRIMAL_FEASIBLE  7
#define CUOPT_TERIMINATION_STATUS_FEASIBLE_FOUND   8
#define CUOPT_TERIMINATION_STATUS_CONCURRENT_LIMIT 9
#define CUOPT_TERIMINATION_STATUS_WORK_LIMIT       10

#define CUOPT_MINIMIZE 1
#define CUOPT_MAXIMIZE -1

#define CUOPT_LESS_THAN    'L'
#define CUOPT_GREATER_THAN 'G'
#define CUOPT_EQUAL        'E'

#define CUOPT_CONTINUOUS 'C'
#define CUOPT_INTEGER    'I'

#ifdef __cplusplus
#define CUOPT_INFINITY std::numeric_limits<double>::infinity()
#else
#define CUOPT_INFINITY INFINITY
#endif

#define CUOPT_PDLP_SOLVER_MODE_STABLE1     0
#define CUOPT_PDLP_SOLVER_MODE_STABLE2     1
#define CUOPT_PDLP_SOLVER_MODE_METHODICAL1 2
#define CUOPT_PDLP_SOLVER_MODE_FAST1       3
#define CUOPT_PDLP_SOLVER_MODE_STABLE3     4

#define CUOPT_METHOD_CONCURRENT   0
#define CUOPT_METHOD_PDLP         1
#define CUOPT_METHOD_DUAL_SIMPLEX 2
#define CUOPT_METHOD_BARRIER      3

#define CUOPT_FILE_FORMAT_MPS 0

/* Return codes (reference constants.h:132-138) */
#define CUOPT_SUCCESS          0
#define CUOPT_INVALID_ARGUMENT 1
#define CUOPT_MPS_FILE_ERROR   2
#define CUOPT_MPS_PARSE_ERROR  3
#define CUOPT_VALIDATION_ERROR 4
#define CUOPT_OUT_OF_MEMORY    5
#define CUOPT_RUNTIME_ERROR    6

#define CUOPT_PRESOLVE_DEFAULT -1
#define CUOPT_PRESOLVE_OFF     0
#define CUOPT_PRESOLVE_PAPILO  1
#define CUOPT_PRESOLVE_PSLP    2

#endif /* CUOPT_CONSTANTS_H */
