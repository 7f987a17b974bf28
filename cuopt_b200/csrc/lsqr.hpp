// Matrix-free sparse least-squares solves on the GPU (the adjoint and the vertex polish).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace cuopt_b200 {

// One problem  min |Op z - b|_2  (the minimum-norm solution in the equilibrated variables when Op
// lacks full column rank), with Op given in CSR (rows x cols).
struct lsqr_problem {
  int rows = 0, cols = 0;
  std::vector<int64_t> off;  // rows + 1
  std::vector<int> idx;
  std::vector<double> val;
  std::vector<double> b;  // rows
};

struct lsqr_result {
  std::vector<double> z;  // cols
  int iterations = 0;
  // 0: b = 0 (z = 0), 1: residual test met, 2: least-squares (normal-equation) test met,
  // 3: iteration limit.
  int flag      = 0;
  double rnorm  = 0.0;  // |b - Op z| of the equilibrated system (LSQR's estimate)
  double arnorm = 0.0;  // |Op^T (b - Op z)| of the equilibrated system (LSQR's estimate)
};

// Solves every problem with LSQR (Paige and Saunders, ACM TOMS 8(1), 1982) after a two-sided
// diagonal equilibration of each operator.  One thread block per problem runs the whole
// iteration; nothing is launched per iteration.  `tol` is LSQR's atol = btol; `max_iter` <= 0
// chooses 20 x (rows + cols), at most 200000.
std::vector<lsqr_result> lsqr_solve_batch(const std::vector<const lsqr_problem*>& ps,
                                          cudaStream_t s, double tol = 1e-14, int max_iter = 0);

}  // namespace cuopt_b200
