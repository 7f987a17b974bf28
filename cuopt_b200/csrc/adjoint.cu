// Reverse-mode sensitivities of an optimal LP solution (implicit differentiation of the KKT
// conditions on the solution's active set), and the crossover of an optimal solution to the
// vertex of its active set.  No counterpart in the reference for the adjoint; the reference's
// crossover (dual_simplex/crossover.cpp, called from pdlp/solve.cu:601-680) is replaced by the
// active-set vertex below.
//
// At an optimum, with F the variables strictly inside their bounds and R the constraints held at
// a bound (equalities included), the solution satisfies
//     M x_F = b_R - A_{R,N} x_N      (M = A_{R,F}; x_N sits on its bounds)
//     M^T y_R = c_F                  (stationarity of the free variables; y is 0 off R)
// For a loss L with gradients g_x = dL/dx and g_y = dL/dy, and lambda = M^-T g_x,F,
// mu = M^-1 g_y,R:
//     dL/db_R  = lambda,     dL/dc_F = mu,
//     dL/dA_ij = -lambda_i x_j  (i in R)   - mu_j y_i  (i in R, j in F),
// and every other entry is 0.  When M is square and non-singular (a non-degenerate vertex) these
// are the exact derivatives; otherwise lambda and mu are LSQR's minimum-norm least-squares
// solutions (in the equilibrated variables), the derivatives of the minimum-norm response.
//
// Every solve with M or M^T is matrix-free: LSQR on the GPU with one thread block per system
// (lsqr.cu), all the systems of a batch of instances in one launch.
#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"
#include "host_io.hpp"
#include "lp_model.hpp"
#include "lsqr.hpp"

namespace cuopt_b200 {

namespace {

constexpr double kBoundTol  = 1e-9;   // a variable within this (relative) distance is on its bound
constexpr double kActiveTol = 1e-7;   // a row within this (relative) distance is held at a bound
// Vertex polish: a PDLP solution at its tolerances identifies the active set with looser tests.
constexpr double kPolishBoundTol = 1e-9;
constexpr double kPolishRowTol   = 1e-5;
constexpr double kPolishFeasTol  = 1e-9;
// LSQR tolerance (atol = btol) of the active-set solves: close to FP64 resolution, so that
// square systems are solved to the accuracy of a direct factorisation.
constexpr double kSolveTol = 1e-14;
// Iterative-refinement steps of the vertex polish (its vertex is returned as the solution, so it
// is solved to FP64 resolution; the adjoint's multipliers need no refinement).
constexpr int kPolishRefinements = 2;
// Variables strictly inside their bounds (F) and constraints held at a bound (R) at a point x.
struct active_set {
  std::vector<int> F, R, fpos, rpos;
  std::vector<char> rkind;  // per row: 0 inactive, 1 lower bound (or equality), 2 upper bound
};

template <class X>
active_set classify(const lp_problem& p, const std::vector<double>& lo,
                    const std::vector<double>& up, const X& x, const std::vector<double>& ax,
                    double bound_tol, double row_tol)
{
  active_set a;
  a.fpos.assign(p.n, -1);
  a.rpos.assign(p.m, -1);
  a.rkind.assign(p.m, 0);
  for (int j = 0; j < p.n; ++j) {
    const double l = p.var_lo[j], u = p.var_up[j];
    const bool at_l = std::isfinite(l) && std::fabs(x[j] - l) <= bound_tol * (1.0 + std::fabs(l));
    const bool at_u = std::isfinite(u) && std::fabs(x[j] - u) <= bound_tol * (1.0 + std::fabs(u));
    if (!at_l && !at_u) {
      a.fpos[j] = (int)a.F.size();
      a.F.push_back(j);
    }
  }
  for (int i = 0; i < p.m; ++i) {
    const double l = lo[i], u = up[i];
    char kind = 0;
    if (l == u)
      kind = 1;
    else if (std::isfinite(l) && std::fabs(ax[i] - l) <= row_tol * (1.0 + std::fabs(l)))
      kind = 1;
    else if (std::isfinite(u) && std::fabs(ax[i] - u) <= row_tol * (1.0 + std::fabs(u)))
      kind = 2;
    if (kind) {
      a.rkind[i] = kind;
      a.rpos[i]  = (int)a.R.size();
      a.R.push_back(i);
    }
  }
  return a;
}

template <class X>
std::vector<double> row_products(const lp_problem& p, const X& x)
{
  std::vector<double> ax(p.m, 0.0);
  for (int i = 0; i < p.m; ++i)
    for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) ax[i] += p.val[k] * x[p.col_idx[k]];
  return ax;
}

// Replaces r by the vertex (x_F on the free variables, y_R on the active rows) when it is primal
// and dual feasible; false (r unchanged) otherwise.
bool accept_vertex(const lp_problem& p, pdlp_result& r, const active_set& a,
                   const std::vector<double>& lo, const std::vector<double>& up,
                   const std::vector<double>& xF, const std::vector<double>& yR)
{
  const int m = p.m, n = p.n;
  const int nr = (int)a.R.size(), nf = (int)a.F.size();
  const double sgn = p.maximize ? -1.0 : 1.0;
  // Candidate vertex; accepted only if primal and dual feasible.
  std::vector<double> x(r.x.begin(), r.x.end()), y(m, 0.0);
  for (int q = 0; q < nf; ++q) x[a.F[q]] = xF[q];
  for (int q = 0; q < nr; ++q) y[a.R[q]] = yR[q];
  for (int j : a.F) {
    const double tol = kPolishFeasTol * (1.0 + std::fabs(x[j]));
    if (!(x[j] >= p.var_lo[j] - tol && x[j] <= p.var_up[j] + tol)) return false;
  }
  const std::vector<double> ax = row_products(p, x);
  for (int i = 0; i < m; ++i) {
    const double tol = kPolishFeasTol * (1.0 + std::fabs(ax[i]));
    if (!(ax[i] >= lo[i] - tol && ax[i] <= up[i] + tol)) return false;
    // dual sign: y >= 0 on a lower bound, <= 0 on an upper bound (minimisation form)
    if (lo[i] != up[i] && a.rkind[i] == 1 && y[i] < -kPolishFeasTol) return false;
    if (lo[i] != up[i] && a.rkind[i] == 2 && y[i] > kPolishFeasTol) return false;
  }
  std::vector<double> s(n);
  for (int j = 0; j < n; ++j) s[j] = sgn * p.c[j];
  for (int i = 0; i < m; ++i)
    for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) s[p.col_idx[k]] -= p.val[k] * y[i];
  double cnorm = 0.0;
  for (int j = 0; j < n; ++j) cnorm = std::max(cnorm, std::fabs(p.c[j]));
  for (int j = 0; j < n; ++j) {
    if (a.fpos[j] >= 0) {
      s[j] = 0.0;
      continue;
    }
    const bool at_l = std::isfinite(p.var_lo[j]) && r.x[j] <= p.var_lo[j];
    const double tol = kPolishFeasTol * (1.0 + cnorm);
    if (at_l ? s[j] < -tol : s[j] > tol) return false;
  }
  // Accept: user-form duals / reduced costs and the statistics of the vertex.
  double pobj = 0.0, dobj = 0.0;
  for (int j = 0; j < n; ++j) pobj += p.c[j] * x[j];
  for (int i = 0; i < m; ++i)
    dobj += std::max(y[i], 0.0) * (std::isfinite(lo[i]) ? lo[i] : 0.0) +
            std::min(y[i], 0.0) * (std::isfinite(up[i]) ? up[i] : 0.0);
  for (int j = 0; j < n; ++j) dobj += s[j] * x[j];
  dobj = sgn * dobj;
  r.x.assign(x.begin(), x.end());
  r.y.resize(m);
  r.rc.resize(n);
  for (int i = 0; i < m; ++i) r.y[i] = sgn * y[i];
  for (int j = 0; j < n; ++j) r.rc[j] = sgn * s[j];
  r.primal_obj = pobj + p.obj_offset;
  r.dual_obj   = dobj + p.obj_offset;
  r.gap        = std::fabs(r.primal_obj - r.dual_obj);
  r.rel_gap    = r.gap / (1.0 + std::fabs(r.primal_obj) + std::fabs(r.dual_obj));
  double rp2 = 0.0;
  for (int i = 0; i < m; ++i) {
    const double d = ax[i] - std::min(std::max(ax[i], lo[i]), up[i]);
    rp2 += d * d;
  }
  r.l2_primal = std::sqrt(rp2);
  r.l2_dual   = 0.0;
  r.rel_dual  = 0.0;
  double bn2 = 0.0;
  for (int i = 0; i < m; ++i) {
    if (std::isfinite(lo[i]) && lo[i] != up[i]) bn2 += lo[i] * lo[i];
    if (std::isfinite(up[i])) bn2 += up[i] * up[i];
  }
  r.rel_primal = r.l2_primal / (1.0 + std::sqrt(bn2));
  return true;
}


// M = A_{R,F} (transposed = false) or its transpose, as an LSQR operator with right-hand side b.
lsqr_problem active_operator(const lp_problem& p, const active_set& a, bool transposed,
                             std::vector<double> b)
{
  const int nr = (int)a.R.size(), nf = (int)a.F.size();
  lsqr_problem q;
  q.rows = transposed ? nf : nr;
  q.cols = transposed ? nr : nf;
  q.off.assign(q.rows + 1, 0);
  if (!transposed) {
    for (int r = 0; r < nr; ++r) {
      const int i = a.R[r];
      int64_t cnt = 0;
      for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k)
        if (a.fpos[p.col_idx[k]] >= 0) ++cnt;
      q.off[r + 1] = q.off[r] + cnt;
    }
    q.idx.resize(q.off[nr]);
    q.val.resize(q.off[nr]);
    for (int r = 0; r < nr; ++r) {
      const int i = a.R[r];
      int64_t e   = q.off[r];
      for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) {
        const int f = a.fpos[p.col_idx[k]];
        if (f < 0) continue;
        q.idx[e]   = f;
        q.val[e++] = p.val[k];
      }
    }
  } else {
    for (int r = 0; r < nr; ++r) {
      const int i = a.R[r];
      for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) {
        const int f = a.fpos[p.col_idx[k]];
        if (f >= 0) ++q.off[f + 1];
      }
    }
    for (int f = 0; f < nf; ++f) q.off[f + 1] += q.off[f];
    q.idx.resize(q.off[nf]);
    q.val.resize(q.off[nf]);
    std::vector<int64_t> pos(q.off.begin(), q.off.end() - 1);
    for (int r = 0; r < nr; ++r) {  // rows of M in order, so every row of M^T is sorted
      const int i = a.R[r];
      for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) {
        const int f = a.fpos[p.col_idx[k]];
        if (f < 0) continue;
        const int64_t e = pos[f]++;
        q.idx[e]        = r;
        q.val[e]        = p.val[k];
      }
    }
  }
  q.b = std::move(b);
  return q;
}

// Own stream and allocation scope for one batch of solves.
struct scoped_stream {
  cudaStream_t s = nullptr;
  scoped_stream() { B200_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~scoped_stream() { cudaStreamDestroy(s); }
};

// b - Op z with the row sums accumulated in long double (the residual of a refinement step).
std::vector<double> residual(const lsqr_problem& q, const std::vector<double>& z)
{
  std::vector<double> r(q.rows);
  for (int i = 0; i < q.rows; ++i) {
    long double acc = q.b[i];
    for (int64_t e = q.off[i]; e < q.off[i + 1]; ++e) acc -= (long double)q.val[e] * z[q.idx[e]];
    r[i] = (double)acc;
  }
  return r;
}

std::vector<lsqr_result> solve_all(const std::vector<lsqr_problem>& sys);

// `rounds` steps of iterative refinement of every solution: LSQR on the residual system, added
// back.  Each step multiplies the error by about LSQR's relative accuracy on the system.
void refine(const std::vector<lsqr_problem>& sys, std::vector<lsqr_result>& res, int rounds)
{
  for (int round = 0; round < rounds && !sys.empty(); ++round) {
    std::vector<lsqr_problem> corr(sys.size());
    for (size_t q = 0; q < sys.size(); ++q) {
      corr[q]   = sys[q];
      corr[q].b = residual(sys[q], res[q].z);
    }
    const std::vector<lsqr_result> d = solve_all(corr);
    for (size_t q = 0; q < sys.size(); ++q) {
      for (size_t j = 0; j < res[q].z.size(); ++j) res[q].z[j] += d[q].z[j];
      if (d[q].flag == 3) res[q].flag = 3;
    }
  }
}

std::vector<lsqr_result> solve_all(const std::vector<lsqr_problem>& sys)
{
  if (sys.empty()) return {};
  scoped_stream ss;
  configure_pool_once();
  std::vector<const lsqr_problem*> ptrs;
  for (const auto& q : sys) ptrs.push_back(&q);
  return lsqr_solve_batch(ptrs, ss.s, kSolveTol);
}

}  // namespace

void solution_adjoint_batch(const std::vector<adjoint_job>& jobs)
{
  struct prepared {
    active_set a;
    int lam = -1, mu = -1;  // indices of the instance's systems
  };
  std::vector<prepared> prep(jobs.size());
  std::vector<lsqr_problem> sys;
  std::vector<std::vector<double>> lo(jobs.size()), up(jobs.size());
  for (size_t t = 0; t < jobs.size(); ++t) {
    const adjoint_job& J = jobs[t];
    const lp_problem& p  = *J.p;
    if ((int)J.sol->x.size() != p.n || (int)J.sol->y.size() != p.m)
      throw std::invalid_argument("adjoint: the solution holds no primal / dual vectors");
    p.constraint_bounds(lo[t], up[t]);
    prep[t].a = classify(p, lo[t], up[t], J.sol->x, row_products(p, J.sol->x), kBoundTol,
                         kActiveTol);
    const active_set& a = prep[t].a;
    if (a.R.empty() || a.F.empty()) continue;
    std::vector<double> gF(a.F.size());
    for (size_t q = 0; q < a.F.size(); ++q) gF[q] = J.gx[a.F[q]];
    prep[t].lam = (int)sys.size();
    sys.push_back(active_operator(p, a, true, std::move(gF)));  // M^T lambda = g_F
    if (J.gy) {
      std::vector<double> gR(a.R.size());
      for (size_t q = 0; q < a.R.size(); ++q) gR[q] = J.gy[a.R[q]];
      prep[t].mu = (int)sys.size();
      sys.push_back(active_operator(p, a, false, std::move(gR)));  // M mu = g_R
    }
  }
  const std::vector<lsqr_result> res = solve_all(sys);
  for (size_t t = 0; t < jobs.size(); ++t) {
    const adjoint_job& J = jobs[t];
    const lp_problem& p  = *J.p;
    const active_set& a  = prep[t].a;
    const int m = p.m, n = p.n;
    std::vector<double> lam(a.R.size(), 0.0), mu(a.F.size(), 0.0);
    if (prep[t].lam >= 0) lam = res[prep[t].lam].z;
    if (prep[t].mu >= 0) mu = res[prep[t].mu].z;
    const host_array<double>& x = J.sol->x;
    const host_array<double>& y = J.sol->y;
    if (J.dc)
      for (int j = 0; j < n; ++j) J.dc[j] = (J.gy && a.fpos[j] >= 0) ? mu[a.fpos[j]] : 0.0;
    if (J.dlo || J.dup)
      for (int i = 0; i < m; ++i) {
        const double v = a.rpos[i] >= 0 ? lam[a.rpos[i]] : 0.0;
        if (J.dlo) J.dlo[i] = a.rkind[i] == 1 ? v : 0.0;
        if (J.dup) J.dup[i] = a.rkind[i] == 2 ? v : 0.0;
      }
    if (J.dval)
      for (int i = 0; i < m; ++i)
        for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) {
          double g = 0.0;
          if (a.rpos[i] >= 0) {
            const int j = p.col_idx[k];
            g -= lam[a.rpos[i]] * x[j];
            if (J.gy && a.fpos[j] >= 0) g -= mu[a.fpos[j]] * y[i];
          }
          J.dval[k] = g;
        }
  }
}

void solution_adjoint(const lp_problem& p, const pdlp_result& sol, const double* gx,
                      const double* gy, double* dc, double* dlo, double* dup, double* dval)
{
  solution_adjoint_batch({adjoint_job{&p, &sol, gx, gy, dc, dlo, dup, dval}});
}

std::vector<bool> vertex_polish_batch(const std::vector<const lp_problem*>& ps,
                                      const std::vector<pdlp_result*>& rs)
{
  const size_t count = ps.size();
  std::vector<bool> ok(count, false);
  struct prepared {
    active_set a;
    std::vector<double> lo, up;
    int xs = -1, ys = -1;
  };
  std::vector<prepared> prep(count);
  std::vector<lsqr_problem> sys;
  for (size_t t = 0; t < count; ++t) {
    const lp_problem& p = *ps[t];
    pdlp_result& r      = *rs[t];
    if ((int)r.x.size() != p.n || (int)r.y.size() != p.m || p.m == 0) continue;
    prepared& P = prep[t];
    p.constraint_bounds(P.lo, P.up);
    P.a = classify(p, P.lo, P.up, r.x, row_products(p, r.x), kPolishBoundTol, kPolishRowTol);
    const int nr = (int)P.a.R.size(), nf = (int)P.a.F.size();
    if (nr != nf || nr == 0) continue;  // degenerate: no unique vertex on this active set
    const double sgn = p.maximize ? -1.0 : 1.0;
    // M x_F = b_R - A_{R,N} x_N ;  M^T y_R = c_F  (in the minimisation form: c -> sgn c).
    std::vector<double> rhs(nr), cF(nf);
    for (int q = 0; q < nr; ++q) {
      const int i = P.a.R[q];
      double v    = P.a.rkind[i] == 2 ? P.up[i] : P.lo[i];
      for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) {
        const int j = p.col_idx[k];
        if (P.a.fpos[j] < 0) v -= p.val[k] * r.x[j];
      }
      rhs[q] = v;
    }
    for (int q = 0; q < nf; ++q) cF[q] = sgn * p.c[P.a.F[q]];
    P.xs = (int)sys.size();
    sys.push_back(active_operator(p, P.a, false, std::move(rhs)));
    P.ys = (int)sys.size();
    sys.push_back(active_operator(p, P.a, true, std::move(cF)));
  }
  std::vector<lsqr_result> res = solve_all(sys);
  refine(sys, res, kPolishRefinements);
  for (size_t t = 0; t < count; ++t) {
    prepared& P = prep[t];
    if (P.xs < 0) continue;
    if (res[P.xs].flag == 3 || res[P.ys].flag == 3) continue;  // not solved to the tolerance
    ok[t] = accept_vertex(*ps[t], *rs[t], P.a, P.lo, P.up, res[P.xs].z, res[P.ys].z);
  }
  return ok;
}

bool vertex_polish(const lp_problem& p, pdlp_result& r)
{
  return vertex_polish_batch({&p}, {&r})[0];
}

}  // namespace cuopt_b200
