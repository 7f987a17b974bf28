/*
 * cuopt_b200 — the cuOpt LP C interface, implemented for NVIDIA B200 (sm_100a).
 *
 * Every declaration below has the same name, signature, argument meaning, ownership rule and
 * return-code behaviour as in cuOpt 26.04's cpp/include/cuopt/linear_programming/cuopt_c.h
 * (the line of each counterpart is cited), so an existing C/C++ caller, or a ctypes / cffi /
 * JNI binding generated from that header, can switch libraries by relinking.
 *
 * Scope: linear programs solved by PDLP (primal-dual hybrid gradient, default mode Stable3).
 *  - Arrays passed to the create functions are copied (host or device pointers are accepted).
 *  - Getters copy into caller buffers and return after the copy completed.
 *  - Handles are owned by the library and released with the cuOptDestroy* functions.
 *  - MIP, quadratic objectives and MPS writing are outside this library's scope: those calls
 *    return CUOPT_INVALID_ARGUMENT (or a solution whose error status is CUOPT_VALIDATION_ERROR),
 *    never a wrong answer.
 */
#ifndef CUOPT_C_H
#define CUOPT_C_H

#include <cuopt/linear_programming/constants.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque handles (reference cuopt_c.h:25, :32, :38) */
typedef void* cuOptOptimizationProblem;
typedef void* cuOptSolverSettings;
typedef void* cuOptSolution;

/* Scalar types (reference cuopt_c.h:46-71; this library is built with double / int32) */
typedef double cuopt_float_t;
typedef int32_t cuopt_int_t;

/* reference cuopt_c.h:78, :84 */
int8_t cuOptGetFloatSize();
int8_t cuOptGetIntSize();

/* reference cuopt_c.h:98 */
cuopt_int_t cuOptGetVersion(cuopt_int_t* version_major,
                            cuopt_int_t* version_minor,
                            cuopt_int_t* version_patch);

/* reference cuopt_c.h:112 — reads free or fixed MPS (ROWS/COLUMNS/RHS/RANGES/BOUNDS/OBJSENSE).
 * Returns CUOPT_MPS_FILE_ERROR if the file cannot be opened, CUOPT_MPS_PARSE_ERROR on bad input. */
cuopt_int_t cuOptReadProblem(const char* filename, cuOptOptimizationProblem* problem_ptr);

/* reference cuopt_c.h:124 — writes the problem as free MPS. */
cuopt_int_t cuOptWriteProblem(cuOptOptimizationProblem problem,
                              const char* filename,
                              cuopt_int_t format);

/* reference cuopt_c.h:171 — constraints given by sense ('E','L','G') and right-hand side. */
cuopt_int_t cuOptCreateProblem(cuopt_int_t num_constraints,
                               cuopt_int_t num_variables,
                               cuopt_int_t objective_sense,
                               cuopt_float_t objective_offset,
                               const cuopt_float_t* objective_coefficients,
                               const cuopt_int_t* constraint_matrix_row_offsets,
                               const cuopt_int_t* constraint_matrix_column_indices,
                               const cuopt_float_t* constraint_matrix_coefficent_values,
                               const char* constraint_sense,
                               const cuopt_float_t* rhs,
                               const cuopt_float_t* lower_bounds,
                               const cuopt_float_t* upper_bounds,
                               const char* variable_types,
                               cuOptOptimizationProblem* problem_ptr);

/* reference cuopt_c.h:240 — constraints given as lower <= A x <= upper. */
cuopt_int_t cuOptCreateRangedProblem(cuopt_int_t num_constraints,
                                     cuopt_int_t num_variables,
                                     cuopt_int_t objective_sense,
                                     cuopt_float_t objective_offset,
                                     const cuopt_float_t* objective_coefficients,
                                     const cuopt_int_t* constraint_matrix_row_offsets,
                                     const cuopt_int_t* constraint_matrix_column_indices,
                                     const cuopt_float_t* constraint_matrix_coefficients,
                                     const cuopt_float_t* constraint_lower_bounds,
                                     const cuopt_float_t* constraint_upper_bounds,
                                     const cuopt_float_t* variable_lower_bounds,
                                     const cuopt_float_t* variable_upper_bounds,
                                     const char* variable_types,
                                     cuOptOptimizationProblem* problem_ptr);

/* reference cuopt_c.h:309, :391 — quadratic objectives are outside this library's scope:
 * both return CUOPT_INVALID_ARGUMENT. */
cuopt_int_t cuOptCreateQuadraticProblem(
  cuopt_int_t num_constraints,
  cuopt_int_t num_variables,
  cuopt_int_t objective_sense,
  cuopt_float_t objective_offset,
  const cuopt_float_t* objective_coefficients,
  const cuopt_int_t* quadratic_objective_matrix_row_offsets,
  const cuopt_int_t* quadratic_objective_matrix_column_indices,
  const cuopt_float_t* quadratic_objective_matrix_coefficent_values,
  const cuopt_int_t* constraint_matrix_row_offsets,
  const cuopt_int_t* constraint_matrix_column_indices,
  const cuopt_float_t* constraint_matrix_coefficent_values,
  const char* constraint_sense,
  const cuopt_float_t* rhs,
  const cuopt_float_t* lower_bounds,
  const cuopt_float_t* upper_bounds,
  cuOptOptimizationProblem* problem_ptr);

cuopt_int_t cuOptCreateQuadraticRangedProblem(
  cuopt_int_t num_constraints,
  cuopt_int_t num_variables,
  cuopt_int_t objective_sense,
  cuopt_float_t objective_offset,
  const cuopt_float_t* objective_coefficients,
  const cuopt_int_t* quadratic_objective_matrix_row_offsets,
  const cuopt_int_t* quadratic_objective_matrix_column_indices,
  const cuopt_float_t* quadratic_objective_matrix_coefficent_values,
  const cuopt_int_t* constraint_matrix_row_offsets,
  const cuopt_int_t* constraint_matrix_column_indices,
  const cuopt_float_t* constraint_matrix_coefficients,
  const cuopt_float_t* constraint_lower_bounds,
  const cuopt_float_t* constraint_upper_bounds,
  const cuopt_float_t* variable_lower_bounds,
  const cuopt_float_t* variable_upper_bounds,
  cuOptOptimizationProblem* problem_ptr);

/* reference cuopt_c.h:414 */
void cuOptDestroyProblem(cuOptOptimizationProblem* problem_ptr);

/* Problem getters (reference cuopt_c.h:425-562) */
cuopt_int_t cuOptGetNumConstraints(cuOptOptimizationProblem problem,
                                   cuopt_int_t* num_constraints_ptr);
cuopt_int_t cuOptGetNumVariables(cuOptOptimizationProblem problem, cuopt_int_t* num_variables_ptr);
cuopt_int_t cuOptGetObjectiveSense(cuOptOptimizationProblem problem,
                                   cuopt_int_t* objective_sense_ptr);
cuopt_int_t cuOptGetObjectiveOffset(cuOptOptimizationProblem problem,
                                    cuopt_float_t* objective_offset_ptr);
cuopt_int_t cuOptGetObjectiveCoefficients(cuOptOptimizationProblem problem,
                                          cuopt_float_t* objective_coefficients_ptr);
cuopt_int_t cuOptGetNumNonZeros(cuOptOptimizationProblem problem, cuopt_int_t* num_non_zeros_ptr);
cuopt_int_t cuOptGetConstraintMatrix(cuOptOptimizationProblem problem,
                                     cuopt_int_t* constraint_matrix_row_offsets_ptr,
                                     cuopt_int_t* constraint_matrix_column_indices_ptr,
                                     cuopt_float_t* constraint_matrix_coefficients_ptr);
cuopt_int_t cuOptGetConstraintSense(cuOptOptimizationProblem problem, char* constraint_sense_ptr);
cuopt_int_t cuOptGetConstraintRightHandSide(cuOptOptimizationProblem problem,
                                            cuopt_float_t* rhs_ptr);
cuopt_int_t cuOptGetConstraintLowerBounds(cuOptOptimizationProblem problem,
                                          cuopt_float_t* lower_bounds_ptr);
cuopt_int_t cuOptGetConstraintUpperBounds(cuOptOptimizationProblem problem,
                                          cuopt_float_t* upper_bounds_ptr);
cuopt_int_t cuOptGetVariableLowerBounds(cuOptOptimizationProblem problem,
                                        cuopt_float_t* lower_bounds_ptr);
cuopt_int_t cuOptGetVariableUpperBounds(cuOptOptimizationProblem problem,
                                        cuopt_float_t* upper_bounds_ptr);
cuopt_int_t cuOptGetVariableTypes(cuOptOptimizationProblem problem, char* variable_types_ptr);

/* Settings (reference cuopt_c.h:601-690) */
cuopt_int_t cuOptCreateSolverSettings(cuOptSolverSettings* settings_ptr);
void cuOptDestroySolverSettings(cuOptSolverSettings* settings_ptr);
cuopt_int_t cuOptSetParameter(cuOptSolverSettings settings,
                              const char* parameter_name,
                              const char* parameter_value);
cuopt_int_t cuOptGetParameter(cuOptSolverSettings settings,
                              const char* parameter_name,
                              cuopt_int_t parameter_value_size,
                              char* parameter_value);
cuopt_int_t cuOptSetIntegerParameter(cuOptSolverSettings settings,
                                     const char* parameter_name,
                                     cuopt_int_t parameter_value);
cuopt_int_t cuOptGetIntegerParameter(cuOptSolverSettings settings,
                                     const char* parameter_name,
                                     cuopt_int_t* parameter_value);
cuopt_int_t cuOptSetFloatParameter(cuOptSolverSettings settings,
                                   const char* parameter_name,
                                   cuopt_float_t parameter_value);
cuopt_int_t cuOptGetFloatParameter(cuOptSolverSettings settings,
                                   const char* parameter_name,
                                   cuopt_float_t* parameter_value);

/* MIP callbacks (reference cuopt_c.h:653-705): MIP is outside this library's scope; both setters
 * return CUOPT_INVALID_ARGUMENT. */
typedef void (*cuOptMIPGetSolutionCallback)(const cuopt_float_t* solution,
                                            const cuopt_float_t* objective_value,
                                            const cuopt_float_t* solution_bound,
                                            void* user_data);
typedef void (*cuOptMIPSetSolutionCallback)(cuopt_float_t* solution,
                                            cuopt_float_t* objective_value,
                                            const cuopt_float_t* solution_bound,
                                            void* user_data);
cuopt_int_t cuOptSetMIPGetSolutionCallback(cuOptSolverSettings settings,
                                           cuOptMIPGetSolutionCallback callback,
                                           void* user_data);
cuopt_int_t cuOptSetMIPSetSolutionCallback(cuOptSolverSettings settings,
                                           cuOptMIPSetSolutionCallback callback,
                                           void* user_data);

/* reference cuopt_c.h:781-798 — initial iterates for PDLP (copied). */
cuopt_int_t cuOptSetInitialPrimalSolution(cuOptSolverSettings settings,
                                          const cuopt_float_t* primal_solution,
                                          cuopt_int_t num_variables);
cuopt_int_t cuOptSetInitialDualSolution(cuOptSolverSettings settings,
                                        const cuopt_float_t* dual_solution,
                                        cuopt_int_t num_constraints);

/* reference cuopt_c.h:814 — MIP starts: returns CUOPT_INVALID_ARGUMENT. */
cuopt_int_t cuOptAddMIPStart(cuOptSolverSettings settings,
                             const cuopt_float_t* solution,
                             cuopt_int_t num_variables);

/* reference cuopt_c.h:824 */
cuopt_int_t cuOptIsMIP(cuOptOptimizationProblem problem, cuopt_int_t* is_mip_ptr);

/* reference cuopt_c.h:844 — returns the solution's error status (CUOPT_SUCCESS when the solver
 * ran, whatever its termination status). */
cuopt_int_t cuOptSolve(cuOptOptimizationProblem problem,
                       cuOptSolverSettings settings,
                       cuOptSolution* solution_ptr);

/* Solution access (reference cuopt_c.h:852-978) */
void cuOptDestroySolution(cuOptSolution* solution_ptr);
cuopt_int_t cuOptGetTerminationStatus(cuOptSolution solution, cuopt_int_t* termination_status_ptr);
cuopt_int_t cuOptGetErrorStatus(cuOptSolution solution, cuopt_int_t* error_status_ptr);
cuopt_int_t cuOptGetErrorString(cuOptSolution solution,
                                char* error_string_ptr,
                                cuopt_int_t error_string_size);
cuopt_int_t cuOptGetPrimalSolution(cuOptSolution solution, cuopt_float_t* solution_values);
cuopt_int_t cuOptGetObjectiveValue(cuOptSolution solution, cuopt_float_t* objective_value_ptr);
cuopt_int_t cuOptGetSolveTime(cuOptSolution solution, cuopt_float_t* solve_time_ptr);
cuopt_int_t cuOptGetMIPGap(cuOptSolution solution, cuopt_float_t* mip_gap_ptr);
cuopt_int_t cuOptGetSolutionBound(cuOptSolution solution, cuopt_float_t* solution_bound_ptr);
cuopt_int_t cuOptGetDualSolution(cuOptSolution solution, cuopt_float_t* dual_solution_ptr);
cuopt_int_t cuOptGetDualObjectiveValue(cuOptSolution solution,
                                       cuopt_float_t* dual_objective_value_ptr);
cuopt_int_t cuOptGetReducedCosts(cuOptSolution solution, cuopt_float_t* reduced_cost_ptr);

#ifdef __cplusplus
}
#endif

#endif /* CUOPT_C_H */
