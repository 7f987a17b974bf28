// The cuOpt LP C interface (see include/cuopt/linear_programming/cuopt_c.h).
//
// Behaviour mirrors the reference's cpp/src/pdlp/cuopt_c.cpp: the same null-argument checks, the
// same return codes, input arrays copied at creation, getters copying into caller buffers.
#include <cuopt/linear_programming/cuopt_c.h>
#include <cuopt_b200.h>

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <new>
#include <algorithm>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "common.cuh"
#include "host_io.hpp"
#include "lp_model.hpp"

using cuopt_b200::lp_problem;
using cuopt_b200::lp_settings;
using cuopt_b200::lp_solution;

namespace {

constexpr int kVersionMajor = 26, kVersionMinor = 4, kVersionPatch = 0;

// Copies n elements from a host or device pointer (the reference accepts both).
template <typename T, typename A>
void copy_in(std::vector<T, A>& dst, const T* src, size_t n)
{
  if (n == 0) {
    dst.clear();
    return;
  }
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, src) == cudaSuccess &&
      (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged)) {
    dst.resize(n);
    if (cudaMemcpy(dst.data(), src, n * sizeof(T), cudaMemcpyDefault) != cudaSuccess)
      throw std::invalid_argument("cannot read device array");
    return;
  }
  cudaGetLastError();  // clear a "no device" / "invalid value" answer for plain host memory
  dst.resize(n);
  cuopt_b200::parallel_memcpy(dst.data(), src, n * sizeof(T));
}

template <typename T, typename A>
void copy_out(T* dst, const std::vector<T, A>& src)
{
  if (src.empty()) return;
  cudaPointerAttributes attr{};
  if (cudaPointerGetAttributes(&attr, dst) == cudaSuccess &&
      (attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged)) {
    cudaMemcpy(dst, src.data(), src.size() * sizeof(T), cudaMemcpyDefault);
    return;
  }
  cudaGetLastError();
  cuopt_b200::parallel_memcpy(dst, src.data(), src.size() * sizeof(T));
}

// Runs the body of a C entry point; no exception crosses the C ABI (they become return codes).
template <class F>
cuopt_int_t guarded(F&& body) noexcept
{
  try {
    return body();
  } catch (const std::bad_alloc&) {
    return CUOPT_OUT_OF_MEMORY;
  } catch (...) {
    return CUOPT_RUNTIME_ERROR;
  }
}

lp_problem* P(cuOptOptimizationProblem p) { return static_cast<lp_problem*>(p); }
lp_settings* S(cuOptSolverSettings s) { return static_cast<lp_settings*>(s); }
lp_solution* R(cuOptSolution s) { return static_cast<lp_solution*>(s); }

// Device copy of a new problem's arrays (see device_problem), started before the host copies
// when every array is pinned host memory or memory of the current device, so that the DMA engine
// reads them while host threads make the library's own copies.  finish() waits for it (the caller
// may free its arrays once the create call returns); on any failure there is simply no copy.
class device_copy {
 public:
  struct array {
    const void* src;
    size_t bytes;
  };
  explicit device_copy(const std::vector<array>& arrays)
  {
    if (!start(arrays)) fail();
  }
  ~device_copy()
  {
    if (s_) {
      cudaStreamSynchronize(s_);
      cudaStreamDestroy(s_);
    }
  }
  // The copy's arrays in the order given, once they have arrived (null: no copy).
  std::shared_ptr<cuopt_b200::device_problem> finish(std::vector<void*>& dst)
  {
    if (!s_ || !dev_) return nullptr;
    const bool ok = cudaStreamSynchronize(s_) == cudaSuccess;
    cudaStreamDestroy(s_);
    s_ = nullptr;
    if (!ok) {
      fail();
      return nullptr;
    }
    dst = dst_;
    return std::move(dev_);
  }

 private:
  bool start(const std::vector<array>& arrays)
  {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    size_t total = 0;
    for (const array& a : arrays) {
      if (!a.src || a.bytes == 0) continue;
      cudaPointerAttributes attr{};
      if (cudaPointerGetAttributes(&attr, a.src) != cudaSuccess) return false;
      const bool pinned = attr.type == cudaMemoryTypeHost;
      const bool local  = attr.type == cudaMemoryTypeDevice && attr.device == dev;
      if (!pinned && !local) return false;
      total += (a.bytes + 255) / 256 * 256;
    }
    if (total == 0) return true;
    cuopt_b200::configure_pool_once();
    if (cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking) != cudaSuccess) {
      s_ = nullptr;
      return false;
    }
    dev_         = std::make_shared<cuopt_b200::device_problem>();
    dev_->device = dev;
    if (cudaMallocAsync(&dev_->base, total, s_) != cudaSuccess) {
      dev_->base = nullptr;
      return false;
    }
    size_t at = 0;
    for (const array& a : arrays) {
      void* dst = nullptr;
      if (a.src && a.bytes) {
        dst = static_cast<char*>(dev_->base) + at;
        if (cudaMemcpyAsync(dst, a.src, a.bytes, cudaMemcpyDefault, s_) != cudaSuccess)
          return false;
        at += (a.bytes + 255) / 256 * 256;
      }
      dst_.push_back(dst);
    }
    return true;
  }
  // No copy: copies in flight finish before the allocation is released.
  void fail()
  {
    if (s_) cudaStreamSynchronize(s_);
    cudaGetLastError();
    dev_.reset();
  }
  cudaStream_t s_ = nullptr;
  std::shared_ptr<cuopt_b200::device_problem> dev_;
  std::vector<void*> dst_;
};

cuopt_int_t create_common(cuopt_int_t m, cuopt_int_t n, cuopt_int_t sense, cuopt_float_t offset,
                          const cuopt_float_t* c, const cuopt_int_t* off, const cuopt_int_t* idx,
                          const cuopt_float_t* val, const cuopt_float_t* vlo,
                          const cuopt_float_t* vup, const char* vtypes, const cuopt_float_t* clo,
                          const cuopt_float_t* cup, lp_problem* p)
{
  if (m < 0 || n < 0) return CUOPT_INVALID_ARGUMENT;
  p->m          = m;
  p->n          = n;
  p->maximize   = sense == CUOPT_MAXIMIZE;
  p->obj_offset = offset;
  copy_in(p->c, c, n);
  copy_in(p->row_off, off, (size_t)m + 1);
  const int64_t nnz = p->row_off[m];
  if (nnz < 0) return CUOPT_INVALID_ARGUMENT;
  const bool ranged = clo && cup;
  device_copy copy({{off, ((size_t)m + 1) * sizeof(int)},
                    {idx, (size_t)nnz * sizeof(int)},
                    {val, (size_t)nnz * sizeof(double)},
                    {c, (size_t)n * sizeof(double)},
                    {vlo, (size_t)n * sizeof(double)},
                    {vup, (size_t)n * sizeof(double)},
                    {ranged ? clo : nullptr, (size_t)m * sizeof(double)},
                    {ranged ? cup : nullptr, (size_t)m * sizeof(double)}});
  copy_in(p->col_idx, idx, (size_t)nnz);
  copy_in(p->val, val, (size_t)nnz);
  copy_in(p->var_lo, vlo, n);
  copy_in(p->var_up, vup, n);
  if (ranged) {
    p->ranged = true;
    copy_in(p->con_lo, clo, m);
    copy_in(p->con_up, cup, m);
  }
  std::vector<void*> d;
  if (auto dp = copy.finish(d); dp && m > 0 && n > 0 && nnz > 0) {
    dp->row_off = static_cast<const int*>(d[0]);
    dp->col_idx = static_cast<const int*>(d[1]);
    dp->val     = static_cast<const double*>(d[2]);
    dp->c       = static_cast<const double*>(d[3]);
    dp->var_lo  = static_cast<const double*>(d[4]);
    dp->var_up  = static_cast<const double*>(d[5]);
    dp->con_lo  = static_cast<const double*>(d[6]);
    dp->con_up  = static_cast<const double*>(d[7]);
    p->dev.p    = std::move(dp);
  }
  if (vtypes) {
    std::vector<char> t;
    copy_in(t, vtypes, n);
    p->var_types.resize(n);
    for (int j = 0; j < n; ++j) p->var_types[j] = t[j] == CUOPT_CONTINUOUS ? 'C' : 'I';
  } else {
    p->var_types.assign(n, 'C');
  }
  return CUOPT_SUCCESS;
}

}  // namespace

extern "C" {

int8_t cuOptGetFloatSize() { return sizeof(cuopt_float_t); }
int8_t cuOptGetIntSize() { return sizeof(cuopt_int_t); }

cuopt_int_t cuOptGetVersion(cuopt_int_t* major, cuopt_int_t* minor, cuopt_int_t* patch)
{
  if (!major || !minor || !patch) return CUOPT_INVALID_ARGUMENT;
  *major = kVersionMajor;
  *minor = kVersionMinor;
  *patch = kVersionPatch;
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptReadProblem(const char* filename, cuOptOptimizationProblem* problem_ptr)
{
  if (!filename || !problem_ptr) return CUOPT_INVALID_ARGUMENT;
  auto* p = new (std::nothrow) lp_problem();
  if (!p) return CUOPT_OUT_OF_MEMORY;
  std::string err;
  const cuopt_int_t rc = guarded([&] { return (cuopt_int_t)cuopt_b200::read_mps(filename, *p, err); });
  if (rc != CUOPT_SUCCESS) {
    delete p;
    *problem_ptr = nullptr;
    return rc;
  }
  *problem_ptr = p;
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptWriteProblem(cuOptOptimizationProblem problem, const char* filename,
                              cuopt_int_t format)
{
  if (!problem || !filename || std::strlen(filename) == 0) return CUOPT_INVALID_ARGUMENT;
  if (format != CUOPT_FILE_FORMAT_MPS) return CUOPT_INVALID_ARGUMENT;
  return guarded([&] { return (cuopt_int_t)cuopt_b200::write_mps(*P(problem), filename); });
}

cuopt_int_t cuOptCreateProblem(cuopt_int_t num_constraints, cuopt_int_t num_variables,
                               cuopt_int_t objective_sense, cuopt_float_t objective_offset,
                               const cuopt_float_t* objective_coefficients,
                               const cuopt_int_t* constraint_matrix_row_offsets,
                               const cuopt_int_t* constraint_matrix_column_indices,
                               const cuopt_float_t* constraint_matrix_coefficent_values,
                               const char* constraint_sense, const cuopt_float_t* rhs,
                               const cuopt_float_t* lower_bounds,
                               const cuopt_float_t* upper_bounds, const char* variable_types,
                               cuOptOptimizationProblem* problem_ptr)
{
  if (!problem_ptr || !objective_coefficients || !constraint_matrix_row_offsets ||
      !constraint_matrix_column_indices || !constraint_matrix_coefficent_values ||
      !constraint_sense || !rhs || !lower_bounds || !upper_bounds || !variable_types)
    return CUOPT_INVALID_ARGUMENT;
  auto* p = new (std::nothrow) lp_problem();
  if (!p) return CUOPT_OUT_OF_MEMORY;
  try {
    cuopt_int_t rc = create_common(num_constraints, num_variables, objective_sense,
                                   objective_offset, objective_coefficients,
                                   constraint_matrix_row_offsets, constraint_matrix_column_indices,
                                   constraint_matrix_coefficent_values, lower_bounds, upper_bounds,
                                   variable_types, nullptr, nullptr, p);
    if (rc != CUOPT_SUCCESS) {
      delete p;
      return rc;
    }
    p->ranged = false;
    copy_in(p->row_types, constraint_sense, num_constraints);
    copy_in(p->rhs, rhs, num_constraints);
  } catch (const std::exception&) {
    delete p;
    return CUOPT_INVALID_ARGUMENT;
  }
  *problem_ptr = p;
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptCreateRangedProblem(cuopt_int_t num_constraints, cuopt_int_t num_variables,
                                     cuopt_int_t objective_sense, cuopt_float_t objective_offset,
                                     const cuopt_float_t* objective_coefficients,
                                     const cuopt_int_t* constraint_matrix_row_offsets,
                                     const cuopt_int_t* constraint_matrix_column_indices,
                                     const cuopt_float_t* constraint_matrix_coefficients,
                                     const cuopt_float_t* constraint_lower_bounds,
                                     const cuopt_float_t* constraint_upper_bounds,
                                     const cuopt_float_t* variable_lower_bounds,
                                     const cuopt_float_t* variable_upper_bounds,
                                     const char* variable_types,
                                     cuOptOptimizationProblem* problem_ptr)
{
  if (!problem_ptr || !objective_coefficients || !constraint_matrix_row_offsets ||
      !constraint_matrix_column_indices || !constraint_matrix_coefficients ||
      !constraint_lower_bounds || !constraint_upper_bounds || !variable_lower_bounds ||
      !variable_upper_bounds || !variable_types)
    return CUOPT_INVALID_ARGUMENT;
  auto* p = new (std::nothrow) lp_problem();
  if (!p) return CUOPT_OUT_OF_MEMORY;
  try {
    cuopt_int_t rc =
      create_common(num_constraints, num_variables, objective_sense, objective_offset,
                    objective_coefficients, constraint_matrix_row_offsets,
                    constraint_matrix_column_indices, constraint_matrix_coefficients,
                    variable_lower_bounds, variable_upper_bounds, variable_types,
                    constraint_lower_bounds, constraint_upper_bounds, p);
    if (rc != CUOPT_SUCCESS) {
      delete p;
      return rc;
    }
  } catch (const std::exception&) {
    delete p;
    return CUOPT_INVALID_ARGUMENT;
  }
  *problem_ptr = p;
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptCreateQuadraticProblem(cuopt_int_t, cuopt_int_t, cuopt_int_t, cuopt_float_t,
                                        const cuopt_float_t*, const cuopt_int_t*,
                                        const cuopt_int_t*, const cuopt_float_t*,
                                        const cuopt_int_t*, const cuopt_int_t*,
                                        const cuopt_float_t*, const char*, const cuopt_float_t*,
                                        const cuopt_float_t*, const cuopt_float_t*,
                                        cuOptOptimizationProblem* problem_ptr)
{
  if (problem_ptr) *problem_ptr = nullptr;
  return CUOPT_INVALID_ARGUMENT;
}

cuopt_int_t cuOptCreateQuadraticRangedProblem(
  cuopt_int_t, cuopt_int_t, cuopt_int_t, cuopt_float_t, const cuopt_float_t*, const cuopt_int_t*,
  const cuopt_int_t*, const cuopt_float_t*, const cuopt_int_t*, const cuopt_int_t*,
  const cuopt_float_t*, const cuopt_float_t*, const cuopt_float_t*, const cuopt_float_t*,
  const cuopt_float_t*, cuOptOptimizationProblem* problem_ptr)
{
  if (problem_ptr) *problem_ptr = nullptr;
  return CUOPT_INVALID_ARGUMENT;
}

void cuOptDestroyProblem(cuOptOptimizationProblem* problem_ptr)
{
  if (!problem_ptr || !*problem_ptr) return;
  delete P(*problem_ptr);
  *problem_ptr = nullptr;
}

#define CHECK2(a, b) \
  if (!(a) || !(b)) return CUOPT_INVALID_ARGUMENT

cuopt_int_t cuOptGetNumConstraints(cuOptOptimizationProblem problem, cuopt_int_t* v)
{
  CHECK2(problem, v);
  *v = P(problem)->m;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetNumVariables(cuOptOptimizationProblem problem, cuopt_int_t* v)
{
  CHECK2(problem, v);
  *v = P(problem)->n;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetObjectiveSense(cuOptOptimizationProblem problem, cuopt_int_t* v)
{
  CHECK2(problem, v);
  *v = P(problem)->maximize ? CUOPT_MAXIMIZE : CUOPT_MINIMIZE;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetObjectiveOffset(cuOptOptimizationProblem problem, cuopt_float_t* v)
{
  CHECK2(problem, v);
  *v = P(problem)->obj_offset;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetObjectiveCoefficients(cuOptOptimizationProblem problem, cuopt_float_t* v)
{
  CHECK2(problem, v);
  copy_out(v, P(problem)->c);
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetNumNonZeros(cuOptOptimizationProblem problem, cuopt_int_t* v)
{
  CHECK2(problem, v);
  *v = (cuopt_int_t)P(problem)->val.size();
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetConstraintMatrix(cuOptOptimizationProblem problem, cuopt_int_t* off,
                                     cuopt_int_t* idx, cuopt_float_t* val)
{
  if (!problem || !off || !idx || !val) return CUOPT_INVALID_ARGUMENT;
  copy_out(val, P(problem)->val);
  copy_out(idx, P(problem)->col_idx);
  copy_out(off, P(problem)->row_off);
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetConstraintSense(cuOptOptimizationProblem problem, char* v)
{
  CHECK2(problem, v);
  copy_out(v, P(problem)->row_types);
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetConstraintRightHandSide(cuOptOptimizationProblem problem, cuopt_float_t* v)
{
  CHECK2(problem, v);
  copy_out(v, P(problem)->rhs);
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetConstraintLowerBounds(cuOptOptimizationProblem problem, cuopt_float_t* v)
{
  CHECK2(problem, v);
  copy_out(v, P(problem)->con_lo);
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetConstraintUpperBounds(cuOptOptimizationProblem problem, cuopt_float_t* v)
{
  CHECK2(problem, v);
  copy_out(v, P(problem)->con_up);
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetVariableLowerBounds(cuOptOptimizationProblem problem, cuopt_float_t* v)
{
  CHECK2(problem, v);
  copy_out(v, P(problem)->var_lo);
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetVariableUpperBounds(cuOptOptimizationProblem problem, cuopt_float_t* v)
{
  CHECK2(problem, v);
  copy_out(v, P(problem)->var_up);
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetVariableTypes(cuOptOptimizationProblem problem, char* v)
{
  CHECK2(problem, v);
  copy_out(v, P(problem)->var_types);
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptCreateSolverSettings(cuOptSolverSettings* settings_ptr)
{
  if (!settings_ptr) return CUOPT_INVALID_ARGUMENT;
  auto* s = new (std::nothrow) lp_settings();
  if (!s) return CUOPT_OUT_OF_MEMORY;
  *settings_ptr = s;
  return CUOPT_SUCCESS;
}
void cuOptDestroySolverSettings(cuOptSolverSettings* settings_ptr)
{
  if (!settings_ptr) return;
  delete S(*settings_ptr);
  *settings_ptr = nullptr;
}
cuopt_int_t cuOptSetParameter(cuOptSolverSettings settings, const char* name, const char* value)
{
  if (!settings || !name || !value) return CUOPT_INVALID_ARGUMENT;
  return S(settings)->set_from_string(name, value);
}
cuopt_int_t cuOptGetParameter(cuOptSolverSettings settings, const char* name, cuopt_int_t size,
                              char* value)
{
  if (!settings || !name || !value || size <= 0) return CUOPT_INVALID_ARGUMENT;
  std::string v;
  if (S(settings)->get_as_string(name, v) != CUOPT_SUCCESS) return CUOPT_INVALID_ARGUMENT;
  std::snprintf(value, size, "%s", v.c_str());
  return CUOPT_SUCCESS;
}
// Integer setter falls back to the boolean registry (reference cuopt_c.cpp:642-660).
cuopt_int_t cuOptSetIntegerParameter(cuOptSolverSettings settings, const char* name,
                                     cuopt_int_t value)
{
  if (!settings || !name) return CUOPT_INVALID_ARGUMENT;
  if (S(settings)->set_int(name, value) == CUOPT_SUCCESS) return CUOPT_SUCCESS;
  return S(settings)->set_bool(name, value != 0);
}
cuopt_int_t cuOptGetIntegerParameter(cuOptSolverSettings settings, const char* name,
                                     cuopt_int_t* value)
{
  if (!settings || !name || !value) return CUOPT_INVALID_ARGUMENT;
  int32_t v;
  if (S(settings)->get_int(name, v) == CUOPT_SUCCESS) {
    *value = v;
    return CUOPT_SUCCESS;
  }
  bool bv;
  if (S(settings)->get_bool(name, bv) == CUOPT_SUCCESS) {
    *value = bv ? 1 : 0;
    return CUOPT_SUCCESS;
  }
  return CUOPT_INVALID_ARGUMENT;
}
cuopt_int_t cuOptSetFloatParameter(cuOptSolverSettings settings, const char* name,
                                   cuopt_float_t value)
{
  if (!settings || !name) return CUOPT_INVALID_ARGUMENT;
  return S(settings)->set_float(name, value);
}
cuopt_int_t cuOptGetFloatParameter(cuOptSolverSettings settings, const char* name,
                                   cuopt_float_t* value)
{
  if (!settings || !name || !value) return CUOPT_INVALID_ARGUMENT;
  return S(settings)->get_float(name, *value);
}

cuopt_int_t cuOptSetMIPGetSolutionCallback(cuOptSolverSettings, cuOptMIPGetSolutionCallback,
                                           void*)
{
  return CUOPT_INVALID_ARGUMENT;
}
cuopt_int_t cuOptSetMIPSetSolutionCallback(cuOptSolverSettings, cuOptMIPSetSolutionCallback,
                                           void*)
{
  return CUOPT_INVALID_ARGUMENT;
}

cuopt_int_t cuOptSetInitialPrimalSolution(cuOptSolverSettings settings,
                                          const cuopt_float_t* primal, cuopt_int_t n)
{
  if (!settings || !primal || n <= 0) return CUOPT_INVALID_ARGUMENT;
  try {
    copy_in(S(settings)->initial_primal, primal, n);
  } catch (const std::exception&) {
    return CUOPT_INVALID_ARGUMENT;
  }
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptSetInitialDualSolution(cuOptSolverSettings settings, const cuopt_float_t* dual,
                                        cuopt_int_t m)
{
  if (!settings || !dual || m <= 0) return CUOPT_INVALID_ARGUMENT;
  try {
    copy_in(S(settings)->initial_dual, dual, m);
  } catch (const std::exception&) {
    return CUOPT_INVALID_ARGUMENT;
  }
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptAddMIPStart(cuOptSolverSettings, const cuopt_float_t*, cuopt_int_t)
{
  return CUOPT_INVALID_ARGUMENT;
}

cuopt_int_t cuOptIsMIP(cuOptOptimizationProblem problem, cuopt_int_t* is_mip)
{
  CHECK2(problem, is_mip);
  *is_mip = P(problem)->is_mip() ? 1 : 0;
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptSolve(cuOptOptimizationProblem problem, cuOptSolverSettings settings,
                       cuOptSolution* solution_ptr)
{
  if (!problem || !settings || !solution_ptr) return CUOPT_INVALID_ARGUMENT;
  auto* sol = new (std::nothrow) lp_solution();
  if (!sol) return CUOPT_OUT_OF_MEMORY;
  cuopt_b200::trace("cuOptSolve: enter");
  const cuopt_int_t rc = guarded([&] {
    // user_problem_file / solution_file, as the reference's solve_lp writes them
    // (cpp/src/pdlp/solve.cu:1282-1284, 1327-1329).
    std::string problem_file, solution_file;
    S(settings)->get_as_string(CUOPT_USER_PROBLEM_FILE, problem_file);
    S(settings)->get_as_string(CUOPT_SOLUTION_FILE, solution_file);
    if (!problem_file.empty()) cuopt_b200::write_mps(*P(problem), problem_file);
    *sol = cuopt_b200::solve_problem(*P(problem), *S(settings));
    if (!solution_file.empty() && sol->error_code == CUOPT_SUCCESS)
      cuopt_b200::write_sol_file(*P(problem), *sol, solution_file);
    return CUOPT_SUCCESS;
  });
  if (rc != CUOPT_SUCCESS) {
    delete sol;
    return rc;
  }
  cuopt_b200::trace("cuOptSolve: solve_problem");
  *solution_ptr = sol;
  return sol->error_code;
}

void cuOptDestroySolution(cuOptSolution* solution_ptr)
{
  if (!solution_ptr || !*solution_ptr) return;
  delete R(*solution_ptr);
  *solution_ptr = nullptr;
}

cuopt_int_t cuOptGetTerminationStatus(cuOptSolution solution, cuopt_int_t* v)
{
  CHECK2(solution, v);
  *v = R(solution)->r.status;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetErrorStatus(cuOptSolution solution, cuopt_int_t* v)
{
  CHECK2(solution, v);
  *v = R(solution)->error_code;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetErrorString(cuOptSolution solution, char* buf, cuopt_int_t size)
{
  CHECK2(solution, buf);
  std::snprintf(buf, size, "%s", R(solution)->error_message.c_str());
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetPrimalSolution(cuOptSolution solution, cuopt_float_t* v)
{
  CHECK2(solution, v);
  return guarded([&] {
    const auto& r = R(solution)->r;
    if (r.dev)
      cuopt_b200::copy_solution_vector(r, 0, v);
    else
      copy_out(v, r.x);
    return CUOPT_SUCCESS;
  });
}
cuopt_int_t cuOptGetObjectiveValue(cuOptSolution solution, cuopt_float_t* v)
{
  CHECK2(solution, v);
  *v = R(solution)->r.primal_obj;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetSolveTime(cuOptSolution solution, cuopt_float_t* v)
{
  CHECK2(solution, v);
  *v = R(solution)->r.solve_time;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetMIPGap(cuOptSolution solution, cuopt_float_t* v)
{
  CHECK2(solution, v);
  return CUOPT_INVALID_ARGUMENT;  // LP solution (reference cuopt_c.cpp:1030-1045)
}
cuopt_int_t cuOptGetSolutionBound(cuOptSolution solution, cuopt_float_t* v)
{
  CHECK2(solution, v);
  return CUOPT_INVALID_ARGUMENT;
}
cuopt_int_t cuOptGetDualSolution(cuOptSolution solution, cuopt_float_t* v)
{
  CHECK2(solution, v);
  return guarded([&] {
    const auto& r = R(solution)->r;
    if (r.dev)
      cuopt_b200::copy_solution_vector(r, 1, v);
    else
      copy_out(v, r.y);
    return CUOPT_SUCCESS;
  });
}
cuopt_int_t cuOptGetDualObjectiveValue(cuOptSolution solution, cuopt_float_t* v)
{
  CHECK2(solution, v);
  *v = R(solution)->r.dual_obj;
  return CUOPT_SUCCESS;
}
cuopt_int_t cuOptGetReducedCosts(cuOptSolution solution, cuopt_float_t* v)
{
  CHECK2(solution, v);
  return guarded([&] {
    const auto& r = R(solution)->r;
    if (r.dev)
      cuopt_b200::copy_solution_vector(r, 2, v);
    else
      copy_out(v, r.rc);
    return CUOPT_SUCCESS;
  });
}

cuopt_int_t cuOptGetPDLPStatistics(cuOptSolution solution, cuOptPDLPStatistics* st)
{
  CHECK2(solution, st);
  const auto& r                       = R(solution)->r;
  st->number_of_steps_taken           = (cuopt_int_t)r.iterations;
  st->total_number_of_attempted_steps = (cuopt_int_t)r.iterations;
  st->l2_primal_residual              = r.l2_primal;
  st->l2_relative_primal_residual     = r.rel_primal;
  st->l2_dual_residual                = r.l2_dual;
  st->l2_relative_dual_residual       = r.rel_dual;
  st->primal_objective                = r.primal_obj;
  st->dual_objective                  = r.dual_obj;
  st->gap                             = r.gap;
  st->relative_gap                    = r.rel_gap;
  st->solve_time                      = r.solve_time;
  st->solved_by_pdlp                  = R(solution)->solved_by_pdlp ? 1 : 0;
  st->restarts                        = r.restarts;
  st->power_iterations                = r.power_iterations;
  st->refinement_passes               = r.refinement_passes;
  st->step_size                       = r.step_size;
  st->primal_weight                   = r.primal_weight;
  st->setup_time                      = r.setup_time;
  st->loop_time                       = r.loop_time;
  st->kernel_launches                 = r.kernel_launches;
  st->crossover                       = r.crossover ? 1 : 0;
  st->plain_iteration_form            = r.plain_form;
  st->persistent_blocks               = r.persistent_blocks;
  st->plain_iteration_us_graphs       = r.us_plain_graphs;
  st->plain_iteration_us_persistent   = r.us_plain_persistent;
  st->plain_iteration_us_cluster      = r.us_plain_cluster;
  st->sweep_warps_per_block_primal    = r.wpb_primal;
  st->sweep_warps_per_block_dual      = r.wpb_dual;
  for (int q = 0; q < 6; ++q) st->sweep_block_shape_ms[q] = r.wpb_ms[q / 3][q % 3];
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptSolveDevice(cuopt_int_t m, cuopt_int_t n, cuopt_int_t sense, cuopt_float_t offset,
                             const cuopt_float_t* d_c, const cuopt_int_t* d_off,
                             const cuopt_int_t* d_idx, const cuopt_float_t* d_val,
                             const cuopt_float_t* d_lo, const cuopt_float_t* d_up,
                             const cuopt_float_t* d_vlo, const cuopt_float_t* d_vup,
                             cuOptSolverSettings settings, void* stream, cuopt_float_t* d_x,
                             cuopt_float_t* d_y, cuopt_float_t* d_rc, cuOptPDLPStatistics* stats,
                             cuopt_int_t* termination_status)
{
  if (!settings || !d_c || !d_off || !d_lo || !d_up || !d_vlo || !d_vup || !d_x || !d_y || !d_rc)
    return CUOPT_INVALID_ARGUMENT;
  if (m <= 0 || n <= 0) return CUOPT_INVALID_ARGUMENT;
  lp_solution sol;
  try {
    cuopt_b200::lp_device_input in;
    in.m          = m;
    in.n          = n;
    in.row_off    = d_off;
    in.col_idx    = d_idx;
    in.val        = d_val;
    in.c          = d_c;
    in.con_lo     = d_lo;
    in.con_up     = d_up;
    in.var_lo     = d_vlo;
    in.var_up     = d_vup;
    in.obj_offset = offset;
    in.maximize   = sense == CUOPT_MAXIMIZE;
    const std::string mode_err = cuopt_b200::solver_mode_error(*S(settings));
    if (!mode_err.empty()) throw std::invalid_argument(mode_err);
    cuopt_b200::pdlp_params prm = cuopt_b200::params_from_settings(*S(settings));
    prm.log_to_console          = false;
    sol.r = cuopt_b200::pdlp_solve_device(in, prm, static_cast<cudaStream_t>(stream), d_x, d_y, d_rc);
  } catch (const std::bad_alloc&) {
    std::fprintf(stderr, "cuOptSolveDevice: out of memory\n");
    return CUOPT_OUT_OF_MEMORY;
  } catch (const std::invalid_argument& e) {
    std::fprintf(stderr, "cuOptSolveDevice: %s\n", e.what());
    return CUOPT_VALIDATION_ERROR;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptSolveDevice: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  if (termination_status) *termination_status = sol.r.status;
  if (stats) cuOptGetPDLPStatistics(&sol, stats);
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptProfilePDHGSweeps(cuopt_int_t m, cuopt_int_t n, const cuopt_float_t* d_c,
                                   const cuopt_int_t* d_off, const cuopt_int_t* d_idx,
                                   const cuopt_float_t* d_val, const cuopt_float_t* d_lo,
                                   const cuopt_float_t* d_up, const cuopt_float_t* d_vlo,
                                   const cuopt_float_t* d_vup, cuOptSolverSettings settings,
                                   void* stream, cuopt_int_t iterations, double* ms_primal,
                                   double* ms_dual, double* bytes_primal, double* bytes_dual)
{
  if (!settings || !d_c || !d_off || !d_lo || !d_up || !d_vlo || !d_vup || m <= 0 || n <= 0 ||
      iterations <= 0 || !ms_primal || !ms_dual || !bytes_primal || !bytes_dual)
    return CUOPT_INVALID_ARGUMENT;
  try {
    cuopt_b200::lp_device_input in;
    in.m       = m;
    in.n       = n;
    in.row_off = d_off;
    in.col_idx = d_idx;
    in.val     = d_val;
    in.c       = d_c;
    in.con_lo  = d_lo;
    in.con_up  = d_up;
    in.var_lo  = d_vlo;
    in.var_up  = d_vup;
    auto prm   = cuopt_b200::params_from_settings(*S(settings));
    auto prof  = cuopt_b200::pdlp_profile_sweeps(in, prm, static_cast<cudaStream_t>(stream),
                                                 iterations);
    *ms_primal    = prof.ms_primal;
    *ms_dual      = prof.ms_dual;
    *bytes_primal = prof.bytes_primal;
    *bytes_dual   = prof.bytes_dual;
  } catch (const std::bad_alloc&) {
    return CUOPT_OUT_OF_MEMORY;
  } catch (const std::invalid_argument& e) {
    std::fprintf(stderr, "cuOptProfilePDHGSweeps: %s\n", e.what());
    return CUOPT_VALIDATION_ERROR;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptProfilePDHGSweeps: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptProfileSweepClasses(cuopt_int_t m, cuopt_int_t n, const cuopt_float_t* d_c,
                                     const cuopt_int_t* d_off, const cuopt_int_t* d_idx,
                                     const cuopt_float_t* d_val, const cuopt_float_t* d_lo,
                                     const cuopt_float_t* d_up, const cuopt_float_t* d_vlo,
                                     const cuopt_float_t* d_vup, cuOptSolverSettings settings,
                                     void* stream, cuopt_int_t iterations, double* out)
{
  if (!settings || !d_c || !d_off || !d_lo || !d_up || !d_vlo || !d_vup || m <= 0 || n <= 0 ||
      iterations <= 0 || !out)
    return CUOPT_INVALID_ARGUMENT;
  try {
    cuopt_b200::lp_device_input in;
    in.m       = m;
    in.n       = n;
    in.row_off = d_off;
    in.col_idx = d_idx;
    in.val     = d_val;
    in.c       = d_c;
    in.con_lo  = d_lo;
    in.con_up  = d_up;
    in.var_lo  = d_vlo;
    in.var_up  = d_vup;
    auto prm   = cuopt_b200::params_from_settings(*S(settings));
    auto prof  = cuopt_b200::pdlp_profile_sweeps(in, prm, static_cast<cudaStream_t>(stream),
                                                 iterations);
    for (int s = 0; s < 2; ++s)
      for (int q = 0; q < 7; ++q) out[7 * s + q] = prof.classes[s][q];
  } catch (const std::bad_alloc&) {
    return CUOPT_OUT_OF_MEMORY;
  } catch (const std::invalid_argument& e) {
    std::fprintf(stderr, "cuOptProfileSweepClasses: %s\n", e.what());
    return CUOPT_VALIDATION_ERROR;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptProfileSweepClasses: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptBatchSolve(const cuOptOptimizationProblem* problems, cuopt_int_t count,
                            cuOptSolverSettings settings, cuOptSolution* solutions)
{
  if (!problems || !settings || !solutions || count < 0) return CUOPT_INVALID_ARGUMENT;
  std::vector<const cuopt_b200::lp_problem*> ps(count);
  for (cuopt_int_t i = 0; i < count; ++i) {
    solutions[i] = nullptr;
    if (!problems[i]) return CUOPT_INVALID_ARGUMENT;
    ps[i] = P(problems[i]);
  }
  std::vector<lp_solution> rs;
  try {
    rs = cuopt_b200::solve_batch(ps, *S(settings));
  } catch (const std::bad_alloc&) {
    return CUOPT_OUT_OF_MEMORY;
  } catch (...) {
    return CUOPT_RUNTIME_ERROR;
  }
  cuopt_int_t first_error = CUOPT_SUCCESS;
  for (cuopt_int_t i = 0; i < count; ++i) {
    auto* sol = new (std::nothrow) lp_solution(std::move(rs[i]));
    if (!sol) {
      for (cuopt_int_t j = 0; j < i; ++j) cuOptDestroySolution(&solutions[j]);
      return CUOPT_OUT_OF_MEMORY;
    }
    solutions[i] = sol;
    if (sol->error_code != CUOPT_SUCCESS && first_error == CUOPT_SUCCESS) first_error = sol->error_code;
  }
  return first_error;
}

namespace {
cuopt_int_t climbers_to_solutions(std::vector<lp_solution>&& rs, cuOptSolution* solutions)
{
  cuopt_int_t first_error = CUOPT_SUCCESS;
  for (size_t i = 0; i < rs.size(); ++i) {
    auto* sol = new (std::nothrow) lp_solution(std::move(rs[i]));
    if (!sol) {
      for (size_t j = 0; j < i; ++j) cuOptDestroySolution(&solutions[j]);
      return CUOPT_OUT_OF_MEMORY;
    }
    solutions[i] = sol;
    if (sol->error_code != CUOPT_SUCCESS && first_error == CUOPT_SUCCESS)
      first_error = sol->error_code;
  }
  return first_error;
}
}  // namespace

cuopt_int_t cuOptSolveClimbers(cuOptOptimizationProblem problem, cuOptSolverSettings settings,
                               cuopt_int_t count, const cuopt_int_t* variable_indices,
                               const cuopt_float_t* lower_bounds,
                               const cuopt_float_t* upper_bounds, cuOptSolution* solutions)
{
  if (!problem || !settings || !solutions || count <= 0 || !variable_indices || !lower_bounds ||
      !upper_bounds)
    return CUOPT_INVALID_ARGUMENT;
  for (cuopt_int_t i = 0; i < count; ++i) solutions[i] = nullptr;
  std::vector<int> var;
  std::vector<double> lo, up;
  try {
    copy_in(var, variable_indices, count);
    copy_in(lo, lower_bounds, count);
    copy_in(up, upper_bounds, count);
    return climbers_to_solutions(cuopt_b200::solve_climbers(*P(problem), *S(settings), var, lo, up),
                                 solutions);
  } catch (const std::bad_alloc&) {
    return CUOPT_OUT_OF_MEMORY;
  } catch (const std::exception&) {
    return CUOPT_INVALID_ARGUMENT;
  }
}

cuopt_int_t cuOptBatchPDLPStrongBranching(cuOptOptimizationProblem problem,
                                          cuOptSolverSettings settings, cuopt_int_t count,
                                          const cuopt_int_t* fractional,
                                          const cuopt_float_t* root_solution,
                                          cuOptSolution* solutions)
{
  if (!problem || !settings || !solutions || count <= 0 || !fractional || !root_solution)
    return CUOPT_INVALID_ARGUMENT;
  const lp_problem& p = *P(problem);
  for (cuopt_int_t i = 0; i < 2 * count; ++i) solutions[i] = nullptr;
  try {
    std::vector<int> frac;
    std::vector<double> root;
    copy_in(frac, fractional, count);
    copy_in(root, root_solution, count);
    for (cuopt_int_t i = 0; i < count; ++i)
      if (frac[i] < 0 || frac[i] >= p.n) return CUOPT_INVALID_ARGUMENT;
    // Down branches (upper bound floor(x)) then up branches (lower bound ceil(x)), started from a
    // solve of the LP itself, as batch_pdlp_solve / run_batch_pdlp do (reference
    // solve.cu:743-919).
    return climbers_to_solutions(cuopt_b200::solve_strong_branching(p, *S(settings), frac, root),
                                 solutions);
  } catch (const std::bad_alloc&) {
    return CUOPT_OUT_OF_MEMORY;
  } catch (const std::exception&) {
    return CUOPT_INVALID_ARGUMENT;
  }
}

cuopt_int_t cuOptSolutionAdjointBatch(cuopt_int_t count, const cuOptOptimizationProblem* problems,
                                      const cuOptSolution* solutions,
                                      const cuopt_float_t* const* dl_dx,
                                      const cuopt_float_t* const* dl_dy,
                                      cuopt_float_t* const* dl_dc, cuopt_float_t* const* dl_dlower,
                                      cuopt_float_t* const* dl_dupper,
                                      cuopt_float_t* const* dl_dvalues)
{
  if (count < 0 || (count > 0 && (!problems || !solutions || !dl_dx)))
    return CUOPT_INVALID_ARGUMENT;
  struct host_grads {
    std::vector<double> gx, gy, dc, dlo, dup, dval;
  };
  std::vector<host_grads> g(count);
  std::vector<cuopt_b200::adjoint_job> jobs;
  try {
    for (int i = 0; i < count; ++i) {
      if (!problems[i] || !solutions[i] || !dl_dx[i]) return CUOPT_INVALID_ARGUMENT;
      lp_solution* sol = R(solutions[i]);
      if (sol->error_code != CUOPT_SUCCESS || sol->r.status != CUOPT_TERIMINATION_STATUS_OPTIMAL)
        return CUOPT_INVALID_ARGUMENT;
      const lp_problem& p = *P(problems[i]);
      cuopt_b200::ensure_host(sol->r);
      if ((int)sol->r.x.size() != p.n || (int)sol->r.y.size() != p.m) return CUOPT_INVALID_ARGUMENT;
      host_grads& h = g[i];
      copy_in(h.gx, dl_dx[i], p.n);
      const bool has_gy = dl_dy && dl_dy[i];
      if (has_gy) copy_in(h.gy, dl_dy[i], p.m);
      h.dc.resize(dl_dc && dl_dc[i] ? p.n : 0);
      h.dlo.resize(dl_dlower && dl_dlower[i] ? p.m : 0);
      h.dup.resize(dl_dupper && dl_dupper[i] ? p.m : 0);
      h.dval.resize(dl_dvalues && dl_dvalues[i] ? p.val.size() : 0);
      jobs.push_back(cuopt_b200::adjoint_job{
        &p, &sol->r, h.gx.data(), has_gy ? h.gy.data() : nullptr,
        h.dc.empty() ? nullptr : h.dc.data(), h.dlo.empty() ? nullptr : h.dlo.data(),
        h.dup.empty() ? nullptr : h.dup.data(), h.dval.empty() ? nullptr : h.dval.data()});
    }
    cuopt_b200::solution_adjoint_batch(jobs);
    for (int i = 0; i < count; ++i) {
      if (!g[i].dc.empty()) copy_out(dl_dc[i], g[i].dc);
      if (!g[i].dlo.empty()) copy_out(dl_dlower[i], g[i].dlo);
      if (!g[i].dup.empty()) copy_out(dl_dupper[i], g[i].dup);
      if (!g[i].dval.empty()) copy_out(dl_dvalues[i], g[i].dval);
    }
  } catch (const std::bad_alloc&) {
    return CUOPT_OUT_OF_MEMORY;
  } catch (const std::invalid_argument& e) {
    std::fprintf(stderr, "cuOptSolutionAdjointBatch: %s\n", e.what());
    return CUOPT_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptSolutionAdjointBatch: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}

cuopt_int_t cuOptSolutionAdjoint(cuOptOptimizationProblem problem, cuOptSolution solution,
                                 const cuopt_float_t* dl_dx, const cuopt_float_t* dl_dy,
                                 cuopt_float_t* dl_dc, cuopt_float_t* dl_dlower,
                                 cuopt_float_t* dl_dupper, cuopt_float_t* dl_dvalues)
{
  if (!problem || !solution || !dl_dx) return CUOPT_INVALID_ARGUMENT;
  lp_solution* sol = R(solution);
  if (sol->error_code != CUOPT_SUCCESS || sol->r.status != CUOPT_TERIMINATION_STATUS_OPTIMAL)
    return CUOPT_INVALID_ARGUMENT;
  const lp_problem& p = *P(problem);
  try {
    cuopt_b200::ensure_host(sol->r);
  } catch (const std::exception&) {
    return CUOPT_RUNTIME_ERROR;
  }
  if ((int)sol->r.x.size() != p.n || (int)sol->r.y.size() != p.m) return CUOPT_INVALID_ARGUMENT;
  try {
    std::vector<double> gx, gy;
    copy_in(gx, dl_dx, p.n);
    if (dl_dy) copy_in(gy, dl_dy, p.m);
    std::vector<double> dc(dl_dc ? p.n : 0), dlo(dl_dlower ? p.m : 0), dup(dl_dupper ? p.m : 0),
      dval(dl_dvalues ? p.val.size() : 0);
    cuopt_b200::solution_adjoint(p, sol->r, gx.data(), dl_dy ? gy.data() : nullptr,
                                 dl_dc ? dc.data() : nullptr, dl_dlower ? dlo.data() : nullptr,
                                 dl_dupper ? dup.data() : nullptr,
                                 dl_dvalues ? dval.data() : nullptr);
    if (dl_dc) copy_out(dl_dc, dc);
    if (dl_dlower) copy_out(dl_dlower, dlo);
    if (dl_dupper) copy_out(dl_dupper, dup);
    if (dl_dvalues) copy_out(dl_dvalues, dval);
  } catch (const std::bad_alloc&) {
    return CUOPT_OUT_OF_MEMORY;
  } catch (const std::invalid_argument& e) {
    std::fprintf(stderr, "cuOptSolutionAdjoint: %s\n", e.what());
    return CUOPT_INVALID_ARGUMENT;
  } catch (const std::exception& e) {
    std::fprintf(stderr, "cuOptSolutionAdjoint: %s\n", e.what());
    return CUOPT_RUNTIME_ERROR;
  }
  return CUOPT_SUCCESS;
}

}  // extern "C"
