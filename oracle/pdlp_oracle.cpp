// CPU oracle for the PDLP LP path — TEST INFRASTRUCTURE ONLY.
//
// This file restates, in plain FP64 C++, the algorithm cuOpt 26.04 runs on the GPU for
// `solve_lp` with method=PDLP and the default solver mode Stable3 (restarted, reflected Halpern
// PDHG with the cuPDLPx restart scheme).  It exists so the tests, `__graft_entry__.smoke()` and the
// CPU leg of `bench.py` can check the CUDA product path against an independent restatement.  The
// product library never links, loads or calls it.
//
// Each routine cites the reference file:line it follows (paths inside the cuOpt project):
//   hyper-parameters        cpp/src/pdlp/solve.cu:167-209, pdlp_hyper_params.cuh:12-56
//   main loop               cpp/src/pdlp/pdlp.cu:2013-2457 (run_solver), utils.cuh:63-81
//   reflected PDHG step     cpp/src/pdlp/pdhg.cu:431-530, 785-1030
//   Halpern update          cpp/src/pdlp/pdlp.cu:2506-2563
//   fixed-point error       cpp/src/pdlp/pdlp.cu:1401-1421, 1749-1857;
//                           step_size_strategy/adaptive_step_size_strategy.cu:352-518
//   cuPDLPx restart + PID   restart_strategy/pdlp_restart_strategy.cu:689-986, 1196-1259, 1398-1419
//   power iteration         cpp/src/pdlp/pdlp.cu:2587-2739
//   primal weight           cpp/src/pdlp/pdlp.cu:2742-2832
//   scaling                 initial_scaling_strategy/initial_scaling.cu:95-569, 684-790
//   residuals / objectives  termination_strategy/convergence_information.cu:327-811
//   termination test        termination_strategy/termination_strategy.cu:222-376
//   limits / return         cpp/src/pdlp/pdlp.cu:336-495, 839-1238; solve.cu:556-590
//
// Parallelism: row-parallel loops use OpenMP; every reduction is done over a fixed number of
// chunks and then summed in chunk order, so results do not depend on the thread count.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using vec = std::vector<double>;
constexpr double kInf = std::numeric_limits<double>::infinity();

struct csr_t {
  int rows = 0, cols = 0;
  std::vector<int> off, idx;
  vec val;
};

csr_t transpose(const csr_t& a)
{
  csr_t t;
  t.rows = a.cols;
  t.cols = a.rows;
  t.off.assign(a.cols + 1, 0);
  for (int k = 0; k < (int)a.idx.size(); ++k) t.off[a.idx[k] + 1]++;
  for (int j = 0; j < a.cols; ++j) t.off[j + 1] += t.off[j];
  t.idx.resize(a.idx.size());
  t.val.resize(a.val.size());
  std::vector<int> fill(t.off.begin(), t.off.end() - 1);
  for (int i = 0; i < a.rows; ++i)
    for (int k = a.off[i]; k < a.off[i + 1]; ++k) {
      int dst      = fill[a.idx[k]]++;
      t.idx[dst]   = i;
      t.val[dst]   = a.val[k];
    }
  return t;
}

// y = A x, each row summed left to right.
void spmv(const csr_t& a, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
  for (int i = 0; i < a.rows; ++i) {
    double s = 0.0;
    for (int k = a.off[i]; k < a.off[i + 1]; ++k) s += a.val[k] * x[a.idx[k]];
    y[i] = s;
  }
}

// Deterministic chunked sum of f(i) for i in [0, n).
template <typename F>
double chunk_sum(int n, F f)
{
  constexpr int kChunks = 256;
  double part[kChunks];
#pragma omp parallel for schedule(static)
  for (int c = 0; c < kChunks; ++c) {
    long lo = (long)n * c / kChunks, hi = (long)n * (c + 1) / kChunks;
    double s = 0.0;
    for (long i = lo; i < hi; ++i) s += f((int)i);
    part[c] = s;
  }
  double s = 0.0;
  for (int c = 0; c < kChunks; ++c) s += part[c];
  return s;
}

double dot(const vec& a, const vec& b)
{
  return chunk_sum((int)a.size(), [&](int i) { return a[i] * b[i]; });
}
double nrm2(const vec& a) { return std::sqrt(dot(a, a)); }
inline double finite_or_zero(double v) { return std::isfinite(v) ? v : 0.0; }

// sqrt(sum_i  [l_i finite & l_i != u_i] l_i^2 + [u_i finite] u_i^2)   (utils.cuh:251-296)
double bound_norm(const vec& lo, const vec& up)
{
  return std::sqrt(chunk_sum((int)lo.size(), [&](int i) {
    double s = 0.0;
    if (std::isfinite(lo[i]) && lo[i] != up[i]) s += lo[i] * lo[i];
    if (std::isfinite(up[i])) s += up[i] * up[i];
    return s;
  }));
}

// conditional_major (utils.cuh:63-81): 10 below 1e3, 100 below 1e4, ...
long conditional_major(long k)
{
  long step = 10, threshold = 1000;
  while (k >= threshold) {
    step *= 10;
    threshold *= 10;
  }
  return step;
}

struct hyper_t {
  int ruiz_iterations;
  bool do_ruiz, do_pock_chambolle;
  double pc_alpha;
  bool bound_objective_rescaling;
  bool step_from_max_singular_value;  // power iteration vs 1/max|A|
  bool primal_weight_before_scaling;
  bool primal_weight_combined_bounds;
  double primal_importance;
  int major_iteration;
  double artificial_restart_threshold;
  double sufficient_reduction, necessary_reduction;
  double k_p, k_i, k_d, i_smooth;
  double reflection_coefficient;
};

// solve.cu:167-209
hyper_t stable3()
{
  hyper_t h{};
  h.ruiz_iterations               = 10;
  h.do_ruiz                       = true;
  h.do_pock_chambolle             = true;
  h.pc_alpha                      = 1.0;
  h.bound_objective_rescaling     = true;
  h.step_from_max_singular_value  = true;
  h.primal_weight_before_scaling  = true;
  h.primal_weight_combined_bounds = false;
  h.primal_importance             = 1.0;
  h.major_iteration               = 200;
  h.artificial_restart_threshold  = 0.36;
  h.sufficient_reduction          = 0.2;
  h.necessary_reduction           = 0.8;
  h.k_p                           = 0.99;
  h.k_i                           = 0.01;
  h.k_d                           = 0.0;
  h.i_smooth                      = 0.3;
  h.reflection_coefficient        = 1.0;
  return h;
}

// solve.cu:212-248 (only the fields that shape the initial step size / primal weight)
hyper_t methodical1()
{
  hyper_t h                       = stable3();
  h.ruiz_iterations               = 5;
  h.bound_objective_rescaling     = false;
  h.step_from_max_singular_value  = false;
  h.primal_weight_before_scaling  = false;
  h.primal_weight_combined_bounds = true;
  return h;
}

// The problem as PDLP sees it after problem_t construction: minimisation, bounds explicit.
struct lp_t {
  csr_t a, at;
  vec c, con_lo, con_up, var_lo, var_up;
  double obj_scale = 1.0, obj_offset = 0.0;  // presolve_data (problem_helpers.cuh:132-151)
  bool maximize    = false;
};

struct scaling_t {
  vec dr, dc;             // cumulative constraint / variable scaling
  double beta  = 1.0;     // bound rescaling
  double gamma = 1.0;     // objective rescaling
};

// Ruiz inf-norm passes and Pock-Chambolle (initial_scaling.cu:152-365)
scaling_t compute_scaling(const lp_t& p, const hyper_t& h)
{
  const int m = p.a.rows, n = p.a.cols;
  scaling_t s;
  s.dr.assign(m, 1.0);
  s.dc.assign(n, 1.0);
  if (h.do_ruiz) {
    for (int it = 0; it < h.ruiz_iterations; ++it) {
      vec rmax(m, 0.0), cmax(n, 0.0);
      for (int i = 0; i < m; ++i)
        for (int k = p.a.off[i]; k < p.a.off[i + 1]; ++k) {
          int j    = p.a.idx[k];
          double v = std::fabs((p.a.val[k] * s.dr[i]) * s.dc[j]);
          rmax[i]  = std::max(rmax[i], v);
          cmax[j]  = std::max(cmax[j], v);
        }
      for (int i = 0; i < m; ++i)
        if (rmax[i] > 0) s.dr[i] = s.dr[i] / std::sqrt(rmax[i]);
      for (int j = 0; j < n; ++j)
        if (cmax[j] > 0) s.dc[j] = s.dc[j] / std::sqrt(cmax[j]);
    }
  }
  if (h.do_pock_chambolle) {
    const double alpha = h.pc_alpha;
    vec rsum(m, 0.0), csum(n, 0.0);
    for (int i = 0; i < m; ++i)
      for (int k = p.a.off[i]; k < p.a.off[i + 1]; ++k) {
        double v = std::fabs((p.a.val[k] * s.dr[i]) * s.dc[p.a.idx[k]]);
        rsum[i] += std::pow(v, alpha);
      }
    for (int j = 0; j < n; ++j)
      for (int k = p.at.off[j]; k < p.at.off[j + 1]; ++k) {
        double v = std::fabs((p.at.val[k] * s.dr[p.at.idx[k]]) * s.dc[j]);
        csum[j] += std::pow(v, 2.0 - alpha);
      }
    for (int i = 0; i < m; ++i)
      if (rsum[i] > 0) s.dr[i] = s.dr[i] / std::sqrt(rsum[i]);
    for (int j = 0; j < n; ++j)
      if (csum[j] > 0) s.dc[j] = s.dc[j] / std::sqrt(csum[j]);
  }
  return s;
}

// scale_problem (initial_scaling.cu:417-569): returns the scaled copy, fills beta/gamma.
lp_t scale_problem(const lp_t& p, scaling_t& s, const hyper_t& h)
{
  lp_t q = p;
  for (int i = 0; i < q.a.rows; ++i)
    for (int k = q.a.off[i]; k < q.a.off[i + 1]; ++k)
      q.a.val[k] = q.a.val[k] * s.dr[i] * s.dc[q.a.idx[k]];
  for (int j = 0; j < q.at.rows; ++j)
    for (int k = q.at.off[j]; k < q.at.off[j + 1]; ++k)
      q.at.val[k] = q.at.val[k] * s.dc[j] * s.dr[q.at.idx[k]];
  for (int j = 0; j < q.a.cols; ++j) {
    q.c[j] = q.c[j] * s.dc[j];
    if (s.dc[j] != 0) {  // divide_check_zero (utils.cuh:330-339)
      q.var_lo[j] = q.var_lo[j] / s.dc[j];
      q.var_up[j] = q.var_up[j] / s.dc[j];
    } else {
      q.var_lo[j] = 0.0;
      q.var_up[j] = 0.0;
    }
  }
  for (int i = 0; i < q.a.rows; ++i) {
    q.con_lo[i] = q.con_lo[i] * s.dr[i];
    q.con_up[i] = q.con_up[i] * s.dr[i];
  }
  if (h.bound_objective_rescaling) {
    // bound_objective_rescaling (initial_scaling.cu:95-149), computed on the D-scaled values
    s.beta  = 1.0 / (bound_norm(q.con_lo, q.con_up) + 1.0);
    s.gamma = 1.0 / (nrm2(q.c) + 1.0);
    for (int i = 0; i < q.a.rows; ++i) {
      q.con_lo[i] *= s.beta;
      q.con_up[i] *= s.beta;
    }
    for (int j = 0; j < q.a.cols; ++j) {
      q.var_lo[j] *= s.beta;
      q.var_up[j] *= s.beta;
      q.c[j] *= s.gamma;
    }
  }
  return q;
}

// unscale_solutions / scale_solutions (initial_scaling.cu:571-790)
void unscale(const scaling_t& s, vec& x, vec& y, vec& slack)
{
  const double ib = 1.0 / s.beta, ig = 1.0 / s.gamma;
  for (size_t j = 0; j < x.size(); ++j) x[j] = (x[j] * s.dc[j]) * ib;
  for (size_t i = 0; i < y.size(); ++i) y[i] = (y[i] * s.dr[i]) * ig;
  for (size_t j = 0; j < slack.size(); ++j) {
    double v = s.dc[j] != 0 ? slack[j] / s.dc[j] : slack[j];
    slack[j] = v * ig;
  }
}
void rescale(const scaling_t& s, vec& x, vec& y, vec& slack)
{
  for (size_t j = 0; j < x.size(); ++j) {
    double v = s.dc[j] != 0 ? x[j] / s.dc[j] : x[j];
    x[j]     = v * s.beta;
  }
  for (size_t i = 0; i < y.size(); ++i) {
    double v = s.dr[i] != 0 ? y[i] / s.dr[i] : y[i];
    y[i]     = v * s.gamma;
  }
  for (size_t j = 0; j < slack.size(); ++j) slack[j] = (slack[j] * s.dc[j]) * s.gamma;
}

// Power iteration on A A^T (pdlp.cu:2620-2731): returns sigma_max^2.
double power_iteration(const lp_t& q, int* iters_out)
{
  const int m = q.a.rows, n = q.a.cols;
  vec z(m), qv(m), atq(n);
  std::mt19937 gen(1);
  std::normal_distribution<double> dist(0.0, 1.0);
  for (int i = 0; i < m; ++i) z[i] = dist(gen);
  double s2 = 0.0;
  int it    = 0;
  for (int i = 0; i < 5000; ++i) {
    ++it;
    qv        = z;
    double nq = nrm2(qv);
    for (int r = 0; r < m; ++r) qv[r] = qv[r] / nq;
    spmv(q.at, qv.data(), atq.data());
    spmv(q.a, atq.data(), z.data());
    s2 = dot(qv, z);
    for (int r = 0; r < m; ++r) qv[r] = qv[r] * -s2 + z[r];
    if (nrm2(qv) < 1e-4) break;
  }
  if (iters_out) *iters_out = it;
  return s2;
}

struct conv_t {
  double l2_primal = 0, l2_dual = 0, primal_obj = 0, dual_obj = 0, gap = 0, abs_obj = 0;
  // per_constraint_residual: max(0, max_i r_i - rel * rhs_i), rhs = combined bound / c_j
  double linf_primal = 0, linf_dual = 0;
};

// compute_convergence_information for the reflected variant (convergence_information.cu:327-811);
// the per-constraint forms follow :390-420, :453-470 with relative_residual_t (utils.cuh:578-590)
// and combine_finite_abs_bounds (utils.cuh:180-188).
conv_t convergence(const lp_t& p, const vec& x, const vec& y, const vec& slack, double rel_primal,
                   double rel_dual)
{
  const int m = p.a.rows, n = p.a.cols;
  conv_t r;
  vec ax(m), aty(n), rp(m), pslack(m), rd(n);
  spmv(p.a, x.data(), ax.data());
  for (int i = 0; i < m; ++i) {
    double cl = std::max(p.con_lo[i], std::min(ax[i], p.con_up[i]));
    rp[i]     = ax[i] - cl;
    pslack[i] = std::max(y[i], 0.0) * finite_or_zero(p.con_lo[i]) +
                std::min(y[i], 0.0) * finite_or_zero(p.con_up[i]);
  }
  r.l2_primal  = nrm2(rp);
  r.primal_obj = dot(x, p.c);
  spmv(p.at, y.data(), aty.data());
  for (int j = 0; j < n; ++j) rd[j] = (p.c[j] - aty[j]) - slack[j];
  r.l2_dual = nrm2(rd);
  for (int i = 0; i < m; ++i) {
    double cb = 0.0;
    if (std::isfinite(p.con_up[i])) cb = std::max(cb, std::fabs(p.con_up[i]));
    if (std::isfinite(p.con_lo[i])) cb = std::max(cb, std::fabs(p.con_lo[i]));
    r.linf_primal = std::max(r.linf_primal, rp[i] - rel_primal * cb);
  }
  for (int j = 0; j < n; ++j) r.linf_dual = std::max(r.linf_dual, rd[j] - rel_dual * p.c[j]);
  r.dual_obj =
    dot(slack, x) + chunk_sum(m, [&](int i) { return pslack[i]; });
  if (p.obj_scale != 1.0 || p.obj_offset != 0.0) {
    r.primal_obj = p.obj_scale * (r.primal_obj + p.obj_offset);
    r.dual_obj   = p.obj_scale * (r.dual_obj + p.obj_offset);
  }
  r.gap     = std::fabs(r.primal_obj - r.dual_obj);
  r.abs_obj = std::fabs(r.primal_obj) + std::fabs(r.dual_obj);
  return r;
}

}  // namespace

extern "C" {

struct oracle_lp {
  int m, n, nnz;
  const int* row_off;
  const int* col_idx;
  const double* val;
  const double* c;
  const double* con_lo;
  const double* con_up;
  const double* var_lo;
  const double* var_up;
  double obj_offset;
  int maximize;
  const double* initial_primal;  // optional (n), user order; null: start from zero
  const double* initial_dual;    // optional (m)
  // Optional (NaN: not given): a step size that replaces the power iteration and a primal weight
  // that replaces the initial 1, as the reference's strong-branching batch passes them
  // (solve.cu:835-842, pdlp.cu:2027-2083).
  double initial_step_size;
  double initial_primal_weight;
};

struct oracle_settings {
  double abs_primal, rel_primal, abs_dual, rel_dual, abs_gap, rel_gap;
  long iteration_limit;
  double time_limit;
  int threads;
  int detect_infeasibility;                                   // CUOPT_INFEASIBILITY_DETECTION
  double primal_infeasible_tolerance, dual_infeasible_tolerance;
  int per_constraint_residual;                                // CUOPT_PER_CONSTRAINT_RESIDUAL
};

struct oracle_result {
  int status;  // CUOPT_TERIMINATION_STATUS_* values
  int iterations;
  double primal_obj, dual_obj, l2_primal, l2_dual, rel_primal, rel_dual, gap, rel_gap;
  double step_size, primal_weight;
  int restarts;
  int power_iterations;
  double solve_time;
};

}  // extern "C"

namespace {

lp_t build(const oracle_lp* in)
{
  lp_t p;
  p.a.rows = in->m;
  p.a.cols = in->n;
  p.a.off.assign(in->row_off, in->row_off + in->m + 1);
  p.a.idx.assign(in->col_idx, in->col_idx + in->nnz);
  p.a.val.assign(in->val, in->val + in->nnz);
  p.at = transpose(p.a);
  p.c.assign(in->c, in->c + in->n);
  p.con_lo.assign(in->con_lo, in->con_lo + in->m);
  p.con_up.assign(in->con_up, in->con_up + in->m);
  p.var_lo.assign(in->var_lo, in->var_lo + in->n);
  p.var_up.assign(in->var_up, in->var_up + in->n);
  p.maximize   = in->maximize != 0;
  p.obj_offset = in->obj_offset;
  if (p.maximize) {  // convert_to_maximization_problem (problem_helpers.cuh:132-151)
    for (auto& v : p.c) v = -v;
    p.obj_scale  = -1.0;
    p.obj_offset = -p.obj_offset;
  }
  return p;
}

enum { kNoTermination = 0, kOptimal = 1, kInfeasible = 2, kUnbounded = 3, kIterationLimit = 4,
       kTimeLimit = 5,
       kNumericalError = 6, kPrimalFeasible = 7 };

}  // namespace

extern "C" {

// Initial step size and primal weight as computed before the first iteration, for the Stable3
// (mode 4) or Methodical1 (mode 2) hyper-parameter sets (pdlp.cu:2013-2097).
int oracle_initial_step_and_weight(const oracle_lp* in, int mode, double* step, double* weight)
{
  lp_t p    = build(in);
  hyper_t h = mode == 2 ? methodical1() : stable3();
  scaling_t s = compute_scaling(p, h);
  double omega = 1.0;
  auto primal_weight = [&](const lp_t& q) {
    double cn = std::sqrt(chunk_sum(q.a.cols, [&](int j) { return q.c[j] * q.c[j]; }));
    double bn;
    if (h.primal_weight_combined_bounds) {
      bn = std::sqrt(chunk_sum(q.a.rows, [&](int i) {
        double v = 0.0;
        if (std::isfinite(q.con_up[i])) v = std::max(v, std::fabs(q.con_up[i]));
        if (std::isfinite(q.con_lo[i])) v = std::max(v, std::fabs(q.con_lo[i]));
        return v * v;
      }));
    } else if (h.bound_objective_rescaling) {
      return 1.0;
    } else {
      bn = bound_norm(q.con_lo, q.con_up);
    }
    return (bn > 0 && cn > 0) ? h.primal_importance * (cn / bn) : h.primal_importance;
  };
  if (h.primal_weight_before_scaling) omega = primal_weight(p);
  lp_t q = scale_problem(p, s, h);
  if (!h.primal_weight_before_scaling) omega = primal_weight(q);
  double eta;
  if (h.step_from_max_singular_value) {
    double s2 = power_iteration(q, nullptr);
    eta       = 0.998 / std::sqrt(s2);
  } else {
    double amax = 0.0;
    for (double v : q.a.val) amax = std::max(amax, std::fabs(v));
    eta = amax != 0 ? 1.0 / amax : 0.0;
  }
  *step   = eta;
  *weight = omega;
  return 0;
}

// Full Stable3 solve.  x_out[n], y_out[m], rc_out[n] receive the returned (unscaled) iterates.
int oracle_pdlp_solve(const oracle_lp* in, const oracle_settings* st, oracle_result* res,
                      double* x_out, double* y_out, double* rc_out)
{
#ifdef _OPENMP
  if (st->threads > 0) omp_set_num_threads(st->threads);
#endif
  auto t0 = std::chrono::steady_clock::now();
  auto elapsed = [&]() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  };
  std::memset(res, 0, sizeof(*res));
  const int m = in->m, n = in->n;
  if (m == 0) {  // run_pdlp_solver refuses problems without constraints (solve.cu:562-567)
    res->status = kNumericalError;
    return 0;
  }
  const hyper_t h = stable3();
  lp_t p          = build(in);

  // Constant norms of the unscaled problem (convergence_information.cu:92-106)
  const double c_norm = nrm2(p.c);
  const double b_norm = bound_norm(p.con_lo, p.con_up);

  // Initial primal weight before scaling: bound_objective_rescaling => 1 (pdlp.cu:2799-2810),
  // unless one is given; it also seeds the PID controller's best weight (pdlp.cu:2061-2083).
  double omega = std::isfinite(in->initial_primal_weight) ? in->initial_primal_weight : 1.0;
  double best_omega = omega;
  scaling_t s  = compute_scaling(p, h);
  lp_t q       = scale_problem(p, s, h);
  int piters   = 0;
  // A given step size skips compute_initial_step_size (pdlp.cu:2036-2059).
  const double eta = std::isfinite(in->initial_step_size)
                       ? in->initial_step_size
                       : 0.998 / std::sqrt(power_iteration(q, &piters));
  if (!(std::isfinite(eta) && eta > 0)) {
    res->status = kNumericalError;
    return 0;
  }
  double tau = eta / omega, sigma = eta * omega;

  vec x(n, 0.0), y(m, 0.0), x_hat(n, 0.0), y_hat(m, 0.0), slack(n, 0.0), x_bar(n, 0.0),
    y_bar(m, 0.0), x_anchor(n, 0.0), y_anchor(m, 0.0), aty(n, 0.0), ax(m, 0.0), next_aty(n, 0.0);
  // Initial solution (pdlp.cu:1236-1400, set_initial_primal_solution :305-330): x, the
  // potential next iterate and the restart anchor take it, scaled by scale_solutions
  // (initial_scaling.cu:571-640).
  if (in->initial_primal)
    for (int j = 0; j < n; ++j) {
      const double v = s.dc[j] != 0 ? in->initial_primal[j] / s.dc[j] : in->initial_primal[j];
      x[j] = x_hat[j] = x_anchor[j] = v * s.beta;
    }
  if (in->initial_dual)
    for (int i = 0; i < m; ++i) {
      const double v = s.dr[i] != 0 ? in->initial_dual[i] / s.dr[i] : in->initial_dual[i];
      y[i] = y_hat[i] = y_anchor[i] = v * s.gamma;
    }
  // project_initial_primal (pdlp.cu:2237-2262): only x, not the anchor
  for (int j = 0; j < n; ++j) x[j] = std::min(std::max(x[j], q.var_lo[j]), q.var_up[j]);

  const double qnan = std::numeric_limits<double>::quiet_NaN();
  double fpe = qnan, fpe0 = qnan, last_trial = kInf;
  // Ray statistics of the infeasibility test (infeasibility_information.cu:220-490, cuPDLPx
  // branch); zero until first computed, then kept between computations.
  double primal_ray_obj = 0.0, max_primal_ray_inf = 0.0, dual_ray_obj = 0.0, max_dual_ray_inf = 0.0;
  double pid_sum = 0.0, pid_last = 0.0, best_gap = kInf;
  long iters_since_restart = 0;
  int restarts = 0;

  auto finish = [&](int status, const conv_t& cv, long internal_iters) {
    res->status      = status;
    res->iterations  = (int)internal_iters;
    res->primal_obj  = cv.primal_obj;
    res->dual_obj    = cv.dual_obj;
    // With per_constraint_residual the statistics carry the per-constraint forms
    // (termination_strategy.cu:540-566).
    res->l2_primal   = st->per_constraint_residual ? cv.linf_primal : cv.l2_primal;
    res->l2_dual     = st->per_constraint_residual ? cv.linf_dual : cv.l2_dual;
    res->rel_primal  = cv.l2_primal / (1.0 + b_norm);
    res->rel_dual    = cv.l2_dual / (1.0 + c_norm);
    res->gap         = cv.gap;
    res->rel_gap     = cv.gap / (1.0 + cv.abs_obj);
    res->step_size   = eta;
    res->primal_weight = omega;
    res->restarts    = restarts;
    res->power_iterations = piters;
    // x_hat / y_hat / slack are unscaled in place at this point
    const double sgn = p.maximize ? -1.0 : 1.0;  // solve.cu:584-588
    if (x_out) std::copy(x_hat.begin(), x_hat.end(), x_out);
    if (y_out) for (int i = 0; i < m; ++i) y_out[i] = sgn * y_hat[i];
    if (rc_out) for (int j = 0; j < n; ++j) rc_out[j] = sgn * slack[j];
    res->solve_time = elapsed();
    return 0;
  };

  for (long k = 0;; ++k) {
    const bool is_major = (k % h.major_iteration == 0 && k > 0) || k <= 0;
    const bool is_cond  = (k % conditional_major(k)) == 0;
    std::vector<int> restarted(1, 0);
    if (is_major || is_cond) {
      unscale(s, x_hat, y_hat, slack);
      conv_t cv = convergence(p, x_hat, y_hat, slack, st->rel_primal, st->rel_dual);
      int status = kNoTermination;
      // check_termination_criteria_kernel (termination_strategy.cu:311-352)
      const bool pcr       = st->per_constraint_residual != 0;
      const bool primal_ok = pcr ? cv.linf_primal <= st->abs_primal
                                 : cv.l2_primal <= st->abs_primal + st->rel_primal * b_norm;
      const bool dual_ok   = pcr ? cv.linf_dual <= st->abs_dual
                                 : cv.l2_dual <= st->abs_dual + st->rel_dual * c_norm;
      if (dual_ok && primal_ok && cv.gap <= st->abs_gap + st->rel_gap * cv.abs_obj)
        status = kOptimal;
      else if (primal_ok)
        status = kPrimalFeasible;
      if (k > 1 && status == kOptimal) return finish(kOptimal, cv, k);
      // check_termination_criteria_kernel (termination_strategy.cu:354-376); Stable3 returns any
      // current infeasibility (never_restart_to_average, pdlp.cu:1089-1109).
      if (st->detect_infeasibility && status == kNoTermination) {
        if (dual_ray_obj > 0.0 && max_dual_ray_inf / dual_ray_obj <= st->primal_infeasible_tolerance)
          return finish(kInfeasible, cv, k);
        if (primal_ray_obj < 0.0 &&
            max_primal_ray_inf / -primal_ray_obj <= st->dual_infeasible_tolerance)
          return finish(kUnbounded, cv, k);
      }
      if (elapsed() >= st->time_limit) return finish(kTimeLimit, cv, k);
      if (k >= st->iteration_limit) return finish(kIterationLimit, cv, k);
      rescale(s, x_hat, y_hat, slack);

      if (is_major) {
        // should_cupdlpx_restart (pdlp_restart_strategy.cu:689-754)
        bool do_restart = false;
        if (k == h.major_iteration)
          do_restart = true;
        else if (k > h.major_iteration) {
          if (fpe <= h.sufficient_reduction * fpe0)
            do_restart = true;
          else if (fpe <= h.necessary_reduction * fpe0 && fpe > last_trial)
            do_restart = true;
          else if ((double)iters_since_restart >= h.artificial_restart_threshold * (double)k)
            do_restart = true;
        }
        last_trial = fpe;
        if (do_restart) {
          // cupdlpx_restart (pdlp_restart_strategy.cu:868-986)
          double pd = 0.0, dd = 0.0;
          pd = chunk_sum(n, [&](int j) { double d = x_anchor[j] - x_hat[j]; return d * d; });
          dd = chunk_sum(m, [&](int i) { double d = y_anchor[i] - y_hat[i]; return d * d; });
          const double rel_dual   = cv.l2_dual / (1.0 + c_norm);
          const double rel_primal = cv.l2_primal / (1.0 + b_norm);
          const double lp = std::sqrt(pd), ld = std::sqrt(dd);
          const double ratio = rel_primal == 0.0 ? kInf : rel_dual / rel_primal;
          if (lp > 1e-16 && ld > 1e-16 && lp < 1e12 && ld < 1e12 && ratio > 1e-8 && ratio < 1e8) {
            const double err = std::log(ld) - std::log(lp) - std::log(omega);
            pid_sum          = pid_sum * h.i_smooth + err;
            const double derr = err - pid_last;
            omega    = std::exp(h.k_p * err + h.k_i * pid_sum + h.k_d * derr) * omega;
            pid_last = err;
          } else {
            omega    = best_omega;
            pid_sum  = 0.0;
            pid_last = 0.0;
          }
          tau   = eta / omega;
          sigma = eta * omega;
          const double rgap = std::fabs(std::log10(ratio));
          if (rgap < best_gap) {
            best_gap   = rgap;
            best_omega = omega;
          }
          x_anchor = x_hat;
          x        = x_hat;
          y_anchor = y_hat;
          y        = y_hat;
          iters_since_restart = 0;
          last_trial          = kInf;
          restarted[0]        = 1;
          ++restarts;
        }
      }
    }

    // take_step: reflected PDHG (pdhg.cu:785-999, 1002-1030)
    const bool major_step = ((k + 1) % h.major_iteration == 0) ||
                            ((k + 2) % conditional_major(k + 2)) == 0;
    spmv(q.at, y.data(), aty.data());
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j) {
      const double next    = x[j] - tau * (q.c[j] - aty[j]);
      const double clamped = std::max(std::min(next, q.var_up[j]), q.var_lo[j]);
      if (major_step) {
        x_hat[j] = clamped;
        slack[j] = (clamped - next) / tau;
      }
      x_bar[j] = 2.0 * clamped - x[j];
    }
    spmv(q.a, x_bar.data(), ax.data());
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m; ++i) {
      const double t      = y[i] / sigma - ax[i];
      const double tp     = std::max(-q.con_up[i], std::min(t, -q.con_lo[i]));
      const double next_y = (t - tp) * sigma;
      if (major_step) y_hat[i] = next_y;
      y_bar[i] = 2.0 * next_y - y[i];
    }

    // compute_fixed_error (pdlp.cu:1749-1857)
    if ((k + 1) % h.major_iteration == 0 || restarted[0]) {
      spmv(q.at, y_bar.data(), next_aty.data());
      const double inter = chunk_sum(n, [&](int j) { return (next_aty[j] - aty[j]) * (x_bar[j] - x[j]); });
      const double ndx   = chunk_sum(n, [&](int j) { double d = x_bar[j] - x[j]; return d * d; });
      const double ndy   = chunk_sum(m, [&](int i) { double d = y_bar[i] - y[i]; return d * d; });
      const double movement = ndx * omega + ndy / omega;
      fpe = std::sqrt(movement + 2.0 * inter * eta);
      if (restarted[0]) fpe0 = fpe;
      // Infeasibility information from the deltas of this step, for the checks at iterations 200
      // and 400 only (termination_strategy.cu:187-199; infeasibility_information.cu:230-490).
      if (st->detect_infeasibility && (k + 1) % h.major_iteration == 0 &&
          (k + 1) < 3 * h.major_iteration) {
        vec d(n), e(m), ad(m), ate(n);
        for (int j = 0; j < n; ++j) {
          double v = x_bar[j] - x[j];
          if (std::isfinite(q.var_lo[j])) v = std::max(v, 0.0);
          if (std::isfinite(q.var_up[j])) v = std::min(v, 0.0);
          d[j] = v;
        }
        double nd = 0.0, ne = 0.0;
        for (int j = 0; j < n; ++j) nd = std::max(nd, std::fabs(d[j]));
        for (int i = 0; i < m; ++i) {
          double v = y_bar[i] - y[i];
          if (!std::isfinite(q.con_lo[i])) v = std::min(v, 0.0);
          if (!std::isfinite(q.con_up[i])) v = std::max(v, 0.0);
          e[i] = v;
          ne   = std::max(ne, std::fabs(v));
        }
        if (nd > 0.0)
          for (int j = 0; j < n; ++j) d[j] /= nd;
        spmv(q.a, d.data(), ad.data());
        spmv(q.at, e.data(), ate.data());
        const double br = s.beta * s.gamma;
        const auto fin  = [](double v) { return std::isfinite(v) ? v : 0.0; };
        primal_ray_obj  = chunk_sum(n, [&](int j) { return q.c[j] * d[j]; }) / br;
        const double sum_ps = chunk_sum(m, [&](int i) {
          return std::max(e[i], 0.0) * fin(q.con_lo[i]) + std::min(e[i], 0.0) * fin(q.con_up[i]);
        });
        const double sum_ds = chunk_sum(n, [&](int j) {
          return std::max(-ate[j], 0.0) * fin(q.var_lo[j]) + std::min(-ate[j], 0.0) * fin(q.var_up[j]);
        });
        max_primal_ray_inf = 0.0;
        for (int i = 0; i < m; ++i) {
          const double v = (std::max(-ad[i], 0.0) * (std::isfinite(q.con_lo[i]) ? 1.0 : 0.0) +
                            std::max(ad[i], 0.0) * (std::isfinite(q.con_up[i]) ? 1.0 : 0.0)) *
                           s.dr[i];
          max_primal_ray_inf = std::max(max_primal_ray_inf, std::fabs(v));
        }
        double mdi = 0.0;
        for (int j = 0; j < n; ++j) {
          const double v = (std::max(-ate[j], 0.0) * (std::isfinite(q.var_lo[j]) ? 0.0 : 1.0) -
                            std::min(-ate[j], 0.0) * (std::isfinite(q.var_up[j]) ? 0.0 : 1.0)) *
                           s.dc[j];
          mdi = std::max(mdi, std::fabs(v));
        }
        const double sf = std::max(mdi, ne);
        if (sf > 0.0) {
          max_dual_ray_inf = mdi / sf;
          dual_ray_obj     = ((sum_ps + sum_ds) / br) / sf;
        } else {
          max_dual_ray_inf = 0.0;
          dual_ray_obj     = 0.0;
        }
      }
    }

    // halpern_update (pdlp.cu:2506-2563)
    const double w  = double(iters_since_restart + 1) / double(iters_since_restart + 2);
    const double rc = h.reflection_coefficient;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j) x[j] = w * (rc * x_bar[j] + (1.0 - rc) * x[j]) + (1.0 - w) * x_anchor[j];
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m; ++i) y[i] = w * (rc * y_bar[i] + (1.0 - rc) * y[i]) + (1.0 - w) * y_anchor[i];
    ++iters_since_restart;
  }
}

// A plain count of PDHG iterations per second on the given problem, for the CPU baseline: runs
// `iterations` reflected steps (no termination checks) and returns the wall time in seconds.
double oracle_pdhg_iterations(const oracle_lp* in, int iterations, int threads)
{
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#endif
  const hyper_t h = stable3();
  lp_t p          = build(in);
  scaling_t s     = compute_scaling(p, h);
  lp_t q          = scale_problem(p, s, h);
  const int m = q.a.rows, n = q.a.cols;
  const double eta = 1.0, tau = eta, sigma = eta;
  vec x(n, 0.0), y(m, 0.0), x_bar(n), aty(n), ax(m), x_anchor(n, 0.0), y_anchor(m, 0.0);
  auto t0 = std::chrono::steady_clock::now();
  for (int k = 0; k < iterations; ++k) {
    spmv(q.at, y.data(), aty.data());
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j) {
      const double next    = x[j] - tau * (q.c[j] - aty[j]);
      const double clamped = std::max(std::min(next, q.var_up[j]), q.var_lo[j]);
      x_bar[j]             = 2.0 * clamped - x[j];
    }
    spmv(q.a, x_bar.data(), ax.data());
    const double w = double(k + 1) / double(k + 2);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < m; ++i) {
      const double t  = y[i] / sigma - ax[i];
      const double tp = std::max(-q.con_up[i], std::min(t, -q.con_lo[i]));
      const double yb = 2.0 * (t - tp) * sigma - y[i];
      y[i]            = w * yb + (1.0 - w) * y_anchor[i];
    }
#pragma omp parallel for schedule(static)
    for (int j = 0; j < n; ++j) x[j] = w * x_bar[j] + (1.0 - w) * x_anchor[j];
  }
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

int oracle_max_threads()
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
