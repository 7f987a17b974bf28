// Reverse-mode sensitivities of an optimal LP solution (implicit differentiation of the KKT
// conditions on the solution's active set).  No counterpart in the reference.
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
// are the exact derivatives; otherwise lambda and mu are the least-squares solutions of the
// regularised normal equations, i.e. the derivatives of the minimum-norm response.
//
// M is assembled densely on the GPU and factorised with cuSOLVER (LU when square, Cholesky of
// M M^T otherwise); this is a one-off linear solve per call, not part of the PDLP iteration.
// cuSOLVER and cuBLAS are loaded with dlopen on the first call, so the library itself depends on
// nothing but the driver.
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <dlfcn.h>

#include <algorithm>
#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "common.cuh"
#include "host_io.hpp"
#include "lp_model.hpp"

namespace cuopt_b200 {

namespace {

#define B200_SOLVER_CHECK(expr)                                                          \
  do {                                                                                  \
    const int _st = (int)(expr);                                                        \
    if (_st != 0)                                                                       \
      throw cuda_error(std::string("cuSOLVER/cuBLAS status ") + std::to_string(_st) +  \
                       " at " + __FILE__ + ":" + std::to_string(__LINE__));             \
  } while (0)

constexpr double kBoundTol  = 1e-9;   // a variable within this (relative) distance is on its bound
constexpr double kActiveTol = 1e-7;   // a row within this (relative) distance is held at a bound
constexpr size_t kMaxDenseBytes = size_t(6) << 30;
// Vertex polish: a PDLP solution at its tolerances identifies the active set with looser tests.
constexpr double kPolishBoundTol = 1e-9;
constexpr double kPolishRowTol   = 1e-5;
constexpr double kPolishFeasTol  = 1e-9;

// Dense column-major M (rows x cols, zeroed) from (row, col, value) triplets.
__global__ void scatter_dense_kernel(const int* r, const int* c, const double* v, int count,
                                     int ld, double* M)
{
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x)
    M[(size_t)c[k] * ld + r[k]] += v[k];
}

__global__ void add_diagonal_kernel(double* N, int n, double delta)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    N[(size_t)i * n + i] += delta;
}

// Entry points of the dynamically loaded cuSOLVER / cuBLAS.
struct solver_api {
  decltype(&cusolverDnCreate) dn_create;
  decltype(&cusolverDnDestroy) dn_destroy;
  decltype(&cusolverDnSetStream) dn_set_stream;
  decltype(&cusolverDnDgetrf_bufferSize) getrf_buffer;
  decltype(&cusolverDnDgetrf) getrf;
  decltype(&cusolverDnDgetrs) getrs;
  decltype(&cusolverDnDpotrf_bufferSize) potrf_buffer;
  decltype(&cusolverDnDpotrf) potrf;
  decltype(&cusolverDnDpotrs) potrs;
  decltype(&cublasCreate_v2) blas_create;
  decltype(&cublasDestroy_v2) blas_destroy;
  decltype(&cublasSetStream_v2) blas_set_stream;
  decltype(&cublasDgemm_v2) gemm;
  decltype(&cublasDgemv_v2) gemv;
};

void* open_first(const char* const* names)
{
  for (; *names; ++names)
    if (void* h = dlopen(*names, RTLD_NOW | RTLD_LOCAL)) return h;
  return nullptr;
}

template <typename F>
void bind(void* lib, const char* name, F& f)
{
  f = reinterpret_cast<F>(dlsym(lib, name));
  if (!f) throw std::runtime_error(std::string("adjoint: missing symbol ") + name);
}

const solver_api& api()
{
  static const solver_api a = [] {
    static const char* const solver_names[] = {"libcusolver.so.11", "libcusolver.so", nullptr};
    static const char* const blas_names[]   = {"libcublas.so.12", "libcublas.so", nullptr};
    void* ls = open_first(solver_names);
    void* lb = open_first(blas_names);
    if (!ls || !lb) throw std::runtime_error("adjoint: cannot load cuSOLVER / cuBLAS");
    solver_api r{};
    bind(ls, "cusolverDnCreate", r.dn_create);
    bind(ls, "cusolverDnDestroy", r.dn_destroy);
    bind(ls, "cusolverDnSetStream", r.dn_set_stream);
    bind(ls, "cusolverDnDgetrf_bufferSize", r.getrf_buffer);
    bind(ls, "cusolverDnDgetrf", r.getrf);
    bind(ls, "cusolverDnDgetrs", r.getrs);
    bind(ls, "cusolverDnDpotrf_bufferSize", r.potrf_buffer);
    bind(ls, "cusolverDnDpotrf", r.potrf);
    bind(ls, "cusolverDnDpotrs", r.potrs);
    bind(lb, "cublasCreate_v2", r.blas_create);
    bind(lb, "cublasDestroy_v2", r.blas_destroy);
    bind(lb, "cublasSetStream_v2", r.blas_set_stream);
    bind(lb, "cublasDgemm_v2", r.gemm);
    bind(lb, "cublasDgemv_v2", r.gemv);
    return r;
  }();
  return a;
}

struct handles {
  cusolverDnHandle_t solver = nullptr;
  cublasHandle_t blas       = nullptr;
  ~handles()
  {
    if (solver) api().dn_destroy(solver);
    if (blas) api().blas_destroy(blas);
  }
};

handles& thread_handles()
{
  static thread_local handles h;
  if (!h.solver) B200_SOLVER_CHECK(api().dn_create(&h.solver));
  if (!h.blas) B200_SOLVER_CHECK(api().blas_create(&h.blas));
  return h;
}

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

// The dense |R| x |F| matrix M = A_{R,F} on the device, factorised once (LU when square, Cholesky
// of M M^T + delta I otherwise), then used for any number of solves.
class active_system {
 public:
  active_system(const lp_problem& p, const active_set& a, cudaStream_t s)
    : s_(s), nr_((int)a.R.size()), nf_((int)a.F.size())
  {
    if ((size_t)nr_ * (size_t)std::max(nf_, nr_) * sizeof(double) > kMaxDenseBytes)
      throw std::invalid_argument("the active set (" + std::to_string(nr_) + " rows x " +
                                  std::to_string(nf_) + " free variables) exceeds the dense limit");
    std::vector<int> tr, tc;
    std::vector<double> tv;
    for (int i : a.R)
      for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) {
        const int j = p.col_idx[k];
        if (a.fpos[j] < 0) continue;
        tr.push_back(a.rpos[i]);
        tc.push_back(a.fpos[j]);
        tv.push_back(p.val[k]);
        fro2_ += p.val[k] * p.val[k];
      }
    M_.resize((size_t)std::max(nr_, 1) * std::max(nf_, 1));
    M_.zero(s_);
    const int cnt = (int)tv.size();
    if (cnt > 0) {
      dbuf<int> dr(cnt), dcl(cnt);
      dbuf<double> dv(cnt);
      dr.upload(tr.data(), cnt, s_);
      dcl.upload(tc.data(), cnt, s_);
      dv.upload(tv.data(), cnt, s_);
      scatter_dense_kernel<<<std::max(1, std::min(4096, (cnt + 255) / 256)), 256, 0, s_>>>(
        dr.data(), dcl.data(), dv.data(), cnt, std::max(nr_, 1), M_.data());
      B200_LAUNCH_CHECK();
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    }
    info_.resize(1);
    if (nr_ > 0 && nf_ > 0) factor();
  }

  bool square() const { return nr_ == nf_; }
  bool ok() const { return ok_; }

  // Least-squares solution of M^T v = g (|F| values in, |R| out).
  std::vector<double> solve_transposed(const std::vector<double>& g)
  {
    std::vector<double> out(nr_, 0.0);
    if (nr_ == 0 || nf_ == 0) return out;
    const solver_api& A = api();
    handles& h          = thread_handles();
    const double one = 1.0, zero = 0.0;
    if (square()) {
      dbuf<double> v(nr_);
      v.upload(g.data(), nr_, s_);
      B200_SOLVER_CHECK(A.getrs(h.solver, CUBLAS_OP_T, nr_, 1, M_.data(), nr_, piv_.data(),
                                v.data(), nr_, info_.data()));
      v.download(out.data(), nr_, s_);
    } else {
      dbuf<double> vF(nf_), vR(nr_);
      vF.upload(g.data(), nf_, s_);
      B200_SOLVER_CHECK(A.gemv(h.blas, CUBLAS_OP_N, nr_, nf_, &one, M_.data(), nr_, vF.data(),
                               1, &zero, vR.data(), 1));
      B200_SOLVER_CHECK(A.potrs(h.solver, CUBLAS_FILL_MODE_LOWER, nr_, 1, N_.data(), nr_,
                                vR.data(), nr_, info_.data()));
      vR.download(out.data(), nr_, s_);
    }
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    return out;
  }

  // Least-squares solution of M v = g (|R| values in, |F| out).
  std::vector<double> solve(const std::vector<double>& g)
  {
    std::vector<double> out(nf_, 0.0);
    if (nr_ == 0 || nf_ == 0) return out;
    const solver_api& A = api();
    handles& h          = thread_handles();
    const double one = 1.0, zero = 0.0;
    if (square()) {
      dbuf<double> v(nr_);
      v.upload(g.data(), nr_, s_);
      B200_SOLVER_CHECK(A.getrs(h.solver, CUBLAS_OP_N, nr_, 1, M_.data(), nr_, piv_.data(),
                                v.data(), nr_, info_.data()));
      v.download(out.data(), nr_, s_);
    } else {
      dbuf<double> vF(nf_), vR(nr_);
      vR.upload(g.data(), nr_, s_);
      B200_SOLVER_CHECK(A.potrs(h.solver, CUBLAS_FILL_MODE_LOWER, nr_, 1, N_.data(), nr_,
                                vR.data(), nr_, info_.data()));
      B200_SOLVER_CHECK(A.gemv(h.blas, CUBLAS_OP_T, nr_, nf_, &one, M_.data(), nr_, vR.data(),
                               1, &zero, vF.data(), 1));
      vF.download(out.data(), nf_, s_);
    }
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    return out;
  }

 private:
  void factor()
  {
    const solver_api& A = api();
    handles& h          = thread_handles();
    B200_SOLVER_CHECK(A.dn_set_stream(h.solver, s_));
    B200_SOLVER_CHECK(A.blas_set_stream(h.blas, s_));
    int lwork = 0, hinfo = 0;
    if (square()) {
      B200_SOLVER_CHECK(A.getrf_buffer(h.solver, nr_, nr_, M_.data(), nr_, &lwork));
      dbuf<double> work(std::max(lwork, 1));
      piv_.resize(nr_);
      B200_SOLVER_CHECK(A.getrf(h.solver, nr_, nr_, M_.data(), nr_, work.data(), piv_.data(),
                                info_.data()));
    } else {
      // delta = 1e-12 x the mean diagonal of M M^T (|M|_F^2 / |R|) keeps the system positive
      // definite when M lacks full row rank.
      const double one = 1.0, zero = 0.0;
      N_.resize((size_t)nr_ * nr_);
      B200_SOLVER_CHECK(A.gemm(h.blas, CUBLAS_OP_N, CUBLAS_OP_T, nr_, nr_, nf_, &one, M_.data(),
                               nr_, M_.data(), nr_, &zero, N_.data(), nr_));
      add_diagonal_kernel<<<std::max(1, std::min(1024, (nr_ + 255) / 256)), 256, 0, s_>>>(
        N_.data(), nr_, 1e-12 * std::max(fro2_ / nr_, 1e-300));
      B200_LAUNCH_CHECK();
      B200_SOLVER_CHECK(
        A.potrf_buffer(h.solver, CUBLAS_FILL_MODE_LOWER, nr_, N_.data(), nr_, &lwork));
      dbuf<double> work(std::max(lwork, 1));
      B200_SOLVER_CHECK(A.potrf(h.solver, CUBLAS_FILL_MODE_LOWER, nr_, N_.data(), nr_,
                                work.data(), lwork, info_.data()));
    }
    info_.download(&hinfo, 1, s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    ok_ = hinfo == 0;
  }

  cudaStream_t s_;
  int nr_, nf_;
  double fro2_ = 0.0;
  bool ok_     = false;
  dbuf<double> M_, N_;
  dbuf<int> piv_, info_;
};

// Own stream and allocation scope for one adjoint / polish call.
struct scoped_stream {
  cudaStream_t s = nullptr;
  scoped_stream() { B200_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~scoped_stream() { cudaStreamDestroy(s); }
};

}  // namespace

void solution_adjoint(const lp_problem& p, const pdlp_result& sol, const double* gx,
                      const double* gy, double* dc, double* dlo, double* dup, double* dval)
{
  const int m = p.m, n = p.n;
  if ((int)sol.x.size() != n || (int)sol.y.size() != m)
    throw std::invalid_argument("adjoint: the solution holds no primal / dual vectors");
  std::vector<double> lo, up;
  p.constraint_bounds(lo, up);
  const host_array<double>& x = sol.x;
  const host_array<double>& y = sol.y;
  const active_set a = classify(p, lo, up, x, row_products(p, x), kBoundTol, kActiveTol);
  const int nr = (int)a.R.size(), nf = (int)a.F.size();

  scoped_stream ss;
  alloc_scope scope(ss.s);
  configure_pool_once();
  std::vector<double> lam(nr, 0.0), mu(nf, 0.0);
  {
    active_system sys(p, a, ss.s);
    if (nr > 0 && nf > 0 && !sys.ok())
      throw std::runtime_error("adjoint: the active-set system is singular");
    std::vector<double> gF(nf);
    for (int q = 0; q < nf; ++q) gF[q] = gx[a.F[q]];
    lam = sys.solve_transposed(gF);
    if (gy) {
      std::vector<double> gR(nr);
      for (int q = 0; q < nr; ++q) gR[q] = gy[a.R[q]];
      mu = sys.solve(gR);
    }
  }

  if (dc)
    for (int j = 0; j < n; ++j) dc[j] = (gy && a.fpos[j] >= 0) ? mu[a.fpos[j]] : 0.0;
  if (dlo || dup)
    for (int i = 0; i < m; ++i) {
      const double v = a.rpos[i] >= 0 ? lam[a.rpos[i]] : 0.0;
      if (dlo) dlo[i] = a.rkind[i] == 1 ? v : 0.0;
      if (dup) dup[i] = a.rkind[i] == 2 ? v : 0.0;
    }
  if (dval)
    for (int i = 0; i < m; ++i)
      for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) {
        double g = 0.0;
        if (a.rpos[i] >= 0) {
          const int j = p.col_idx[k];
          g -= lam[a.rpos[i]] * x[j];
          if (gy && a.fpos[j] >= 0) g -= mu[a.fpos[j]] * y[i];
        }
        dval[k] = g;
      }
}

bool vertex_polish(const lp_problem& p, pdlp_result& r)
{
  const int m = p.m, n = p.n;
  if ((int)r.x.size() != n || (int)r.y.size() != m || m == 0) return false;
  std::vector<double> lo, up;
  p.constraint_bounds(lo, up);
  const active_set a = classify(p, lo, up, r.x, row_products(p, r.x), kPolishBoundTol,
                                kPolishRowTol);
  const int nr = (int)a.R.size(), nf = (int)a.F.size();
  if (nr != nf || nr == 0) return false;  // degenerate: no unique vertex on this active set
  const double sgn = p.maximize ? -1.0 : 1.0;

  scoped_stream ss;
  alloc_scope scope(ss.s);
  configure_pool_once();
  std::vector<double> xF, yR;
  {
    active_system sys(p, a, ss.s);
    if (!sys.ok()) return false;
    // M x_F = b_R - A_{R,N} x_N ;  M^T y_R = c_F  (in the minimisation form: c -> sgn c).
    std::vector<double> rhs(nr), cF(nf);
    for (int q = 0; q < nr; ++q) {
      const int i = a.R[q];
      double v    = a.rkind[i] == 2 ? up[i] : lo[i];
      for (int k = p.row_off[i]; k < p.row_off[i + 1]; ++k) {
        const int j = p.col_idx[k];
        if (a.fpos[j] < 0) v -= p.val[k] * r.x[j];
      }
      rhs[q] = v;
    }
    for (int q = 0; q < nf; ++q) cF[q] = sgn * p.c[a.F[q]];
    xF = sys.solve(rhs);
    yR = sys.solve_transposed(cF);
  }
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

}  // namespace cuopt_b200
