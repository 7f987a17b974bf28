// TEST INFRASTRUCTURE: a command-line driver around the reference's own CPU dual simplex
// (dual_simplex::solve_linear_program, cpp/src/dual_simplex/solve.cpp:665 in the cuOpt project),
// which oracle/ref.mk compiles from the reference's unmodified sources into
// oracle/_ref/ref_dual_simplex.  Used only by tests/ and by bench.py's CPU baseline legs, never by
// the product library.
//
// Input (binary file, little endian): int32 m, n, nnz, maximize, threads; float64 time_limit;
// int32 row_off[m + 1], col_idx[nnz]; float64 val[nnz], c[n], con_lo[m], con_up[m], var_lo[n],
// var_up[n].  Rows must be equalities (con_lo == con_up) or one-sided (one bound infinite).
// Output (stdout, one JSON line): status (the reference's lp_status_t name), objective (in the
// caller's sense), solve_seconds (wall clock of the solve call alone), primal_residual
// (|A x - b|_2 over the rows against their violated bound), threads; with a second argument, x is
// written to that file as float64.
#include <dual_simplex/solve.hpp>
#include <dual_simplex/user_problem.hpp>

#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

namespace ds = cuopt::linear_programming::dual_simplex;

namespace {

template <typename T>
bool read_vec(std::ifstream& f, std::vector<T>& v, size_t n)
{
  v.resize(n);
  return n == 0 || (bool)f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T)));
}

}  // namespace

int main(int argc, char** argv)
{
  if (argc < 2) {
    std::fprintf(stderr, "usage: ref_dual_simplex <lp file> [x output file]\n");
    return 2;
  }
  std::ifstream f(argv[1], std::ios::binary);
  int32_t hdr[5];
  double time_limit = 0.0;
  if (!f.read(reinterpret_cast<char*>(hdr), sizeof(hdr)) ||
      !f.read(reinterpret_cast<char*>(&time_limit), sizeof(double))) {
    std::fprintf(stderr, "ref_dual_simplex: short header\n");
    return 2;
  }
  const int m = hdr[0], n = hdr[1], nnz = hdr[2], maximize = hdr[3], threads = hdr[4];
  std::vector<int32_t> off, idx;
  std::vector<double> val, c, lo, up, vl, vu;
  if (!read_vec(f, off, (size_t)m + 1) || !read_vec(f, idx, nnz) || !read_vec(f, val, nnz) ||
      !read_vec(f, c, n) || !read_vec(f, lo, m) || !read_vec(f, up, m) || !read_vec(f, vl, n) ||
      !read_vec(f, vu, n)) {
    std::fprintf(stderr, "ref_dual_simplex: short body\n");
    return 2;
  }
  raft::handle_t handle{};
  ds::user_problem_t<int, double> p(&handle);
  p.num_rows = m;
  p.num_cols = n;
  p.objective.resize(n);
  for (int j = 0; j < n; ++j) p.objective[j] = maximize ? -c[j] : c[j];
  // CSC copy of the CSR matrix.
  p.A.m      = m;
  p.A.n      = n;
  p.A.nz_max = nnz;
  p.A.reallocate(nnz);
  std::vector<int> cs(n + 1, 0);
  for (int k = 0; k < nnz; ++k) ++cs[idx[k] + 1];
  for (int j = 0; j < n; ++j) cs[j + 1] += cs[j];
  p.A.col_start.resize(n + 1);
  for (int j = 0; j <= n; ++j) p.A.col_start[j] = cs[j];
  {
    std::vector<int> pos(cs.begin(), cs.end() - 1);
    for (int i = 0; i < m; ++i)
      for (int k = off[i]; k < off[i + 1]; ++k) {
        const int q = pos[idx[k]]++;
        p.A.i[q]    = i;
        p.A.x[q]    = val[k];
      }
  }
  p.rhs.resize(m);
  p.row_sense.resize(m);
  for (int i = 0; i < m; ++i) {
    if (lo[i] == up[i]) {
      p.row_sense[i] = 'E';
      p.rhs[i]       = lo[i];
    } else if (!std::isfinite(lo[i]) && std::isfinite(up[i])) {
      p.row_sense[i] = 'L';
      p.rhs[i]       = up[i];
    } else if (std::isfinite(lo[i]) && !std::isfinite(up[i])) {
      p.row_sense[i] = 'G';
      p.rhs[i]       = lo[i];
    } else {
      std::fprintf(stderr, "ref_dual_simplex: row %d is ranged or free (not supported)\n", i);
      return 3;
    }
  }
  p.lower.assign(vl.begin(), vl.end());
  p.upper.assign(vu.begin(), vu.end());
  for (int j = 0; j < n; ++j) {
    if (std::isinf(p.lower[j])) p.lower[j] = -ds::inf;
    if (std::isinf(p.upper[j])) p.upper[j] = ds::inf;
  }
  p.num_range_rows = 0;
  p.problem_name   = "lp";
  p.row_names.resize(m);
  p.col_names.resize(n);
  for (int i = 0; i < m; ++i) p.row_names[i] = "r" + std::to_string(i);
  for (int j = 0; j < n; ++j) p.col_names[j] = "x" + std::to_string(j);
  p.obj_constant = 0.0;
  p.var_types.assign(n, ds::variable_type_t::CONTINUOUS);

  ds::simplex_solver_settings_t<int, double> settings;
  settings.set_log(false);
  if (time_limit > 0.0) settings.time_limit = time_limit;
  if (threads > 0) settings.num_threads = threads;
  ds::lp_solution_t<int, double> sol(m, n);
  const auto t0       = std::chrono::steady_clock::now();
  const auto status   = ds::solve_linear_program(p, settings, sol);
  const double secs   = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  double r2 = 0.0;
  if ((int)sol.x.size() == n)
    for (int i = 0; i < m; ++i) {
      double ax = 0.0;
      for (int k = off[i]; k < off[i + 1]; ++k) ax += val[k] * sol.x[idx[k]];
      const double d = ax < lo[i] ? lo[i] - ax : (ax > up[i] ? ax - up[i] : 0.0);
      r2 += d * d;
    }
  double obj = 0.0;
  for (int j = 0; j < n && (int)sol.x.size() == n; ++j) obj += c[j] * sol.x[j];
  std::printf("{\"status\": \"%s\", \"objective\": %.17g, \"solve_seconds\": %.6f, "
              "\"primal_residual\": %.6g, \"threads\": %d}\n",
              ds::lp_status_to_string(status).c_str(), obj, secs, std::sqrt(r2),
              settings.num_threads);
  if (argc > 2 && (int)sol.x.size() == n) {
    std::ofstream out(argv[2], std::ios::binary);
    out.write(reinterpret_cast<const char*>(sol.x.data()), (std::streamsize)(n * sizeof(double)));
  }
  return 0;
}
