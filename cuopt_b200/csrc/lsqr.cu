// Batched LSQR on sm_100a: many small sparse least-squares systems, one thread block each.
//
// The KKT adjoint and the vertex polish both need solves with the active-set matrix M = A_{R,F}
// (rows held at a bound x variables strictly inside their bounds) or its transpose.  These are
// non-symmetric and, on random sparse LPs, ill-conditioned (condition numbers 1e4 - 1e5 for the
// 5000 x 5000 bases of the 64-LP adjoint workload), where restarted GMRES and BiCGStab stall and
// LSQR converges in 7 000 - 11 000 iterations.  A batch of such systems would need two kernel
// boundaries and a reduction per system per iteration if each iteration were a grid-wide launch,
// so instead every system gets one thread block that runs its whole LSQR loop:
//   * the iterate vectors u (rows), v, x and w (cols) live in shared memory when they fit
//     (rows + 3 cols doubles <= kSmemBudget), else in a global scratch slice of the block's own;
//   * the operator and its transpose are stored as 32-row sliced ELL (lane t of a warp owns row t
//     of a slice and reads element k at base + 32 k + t, so a warp reads 32 contiguous values per
//     step), rows sorted by length, so each product is a coalesced stream from L2 with gathers
//     from shared memory;
//   * the two norms of an iteration are block reductions in a fixed order, computed identically by
//     every thread, so the scalar recurrence and the stopping decision are uniform and the result
//     is deterministic;
//   * the x / w update of an iteration is applied in the next transpose product by the thread that
//     owns the row, so an iteration costs two products and two block synchronisations.
// Each block stops at LSQR's tests or at its iteration limit: there are no waits between blocks.
#include "common.cuh"
#include "lsqr.hpp"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>
#include <thread>

namespace cuopt_b200 {

namespace {

constexpr int kLsqrThreads = 512;
constexpr int kLsqrWarps   = kLsqrThreads / kWarp;
constexpr size_t kSmemBudget = 200 * 1024;
constexpr int kEquilibrationPasses = 10;

struct lsqr_desc {
  int rows, cols;           // u has `rows` entries, v / x / w have `cols`
  int slices_p, slices_q;   // slices of P (= Op, rows x cols) and Q (= Op^T, cols x rows)
  const int64_t* p_slice;   // slices_p + 1 element offsets
  const int* p_idx;
  const double* p_val;
  const int64_t* q_slice;   // slices_q + 1
  const int* q_idx;
  const double* q_val;
  const double* b;          // rows (sorted, equilibrated)
  double* z;                // cols (sorted, equilibrated)
  double* scratch;          // rows + 3 cols doubles when the vectors are not in shared memory
  int max_iter;
  double tol;
};

struct lsqr_out {
  int iterations;
  int flag;
  double rnorm;
  double arnorm;
};

// Sum over the block of K per-thread values; every thread gets the same totals (fixed order).
template <int K>
__device__ __forceinline__ void block_sums(const double (&v)[K], double* part, double (&out)[K])
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < K; ++q) {
    const double s = warp_sum(v[q]);
    if (lane == 0) part[warp * K + q] = s;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < K; ++q) {
    double s = 0.0;
    for (int w = 0; w < kLsqrWarps; ++w) s += part[w * K + q];
    out[q] = s;
  }
}

// acc_r = sum_k val[r, k] vec[idx[r, k]] for the rows of a sliced-ELL matrix; f(r, acc_r) for the
// rows this thread owns (row s * 32 + lane of slice s, slices dealt to warps round-robin).
template <class F>
__device__ __forceinline__ void slice_products(int slices, int rows, const int64_t* __restrict__ so,
                                               const int* __restrict__ idx,
                                               const double* __restrict__ val,
                                               const double* vec, F&& f)
{
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int s = warp; s < slices; s += kLsqrWarps) {
    const int64_t base = so[s];
    const int len      = (int)((so[s + 1] - base) >> 5);
    const int* ip      = idx + base + lane;
    const double* vp   = val + base + lane;
    double acc         = 0.0;
    int k              = 0;
    for (; k + 2 <= len; k += 2) {
      const int i0 = ip[32 * k], i1 = ip[32 * k + 32];
      const double a0 = vp[32 * k], a1 = vp[32 * k + 32];
      acc += a0 * vec[i0];
      acc += a1 * vec[i1];
    }
    if (k < len) acc += vp[32 * k] * vec[ip[32 * k]];
    const int r = s * kWarp + lane;
    if (r < rows) f(r, acc);
  }
}

template <bool SMEM>
__global__ void __launch_bounds__(kLsqrThreads) lsqr_kernel(const lsqr_desc* __restrict__ descs,
                                                            lsqr_out* __restrict__ outs)
{
  extern __shared__ double dyn[];
  __shared__ double part_a[kLsqrWarps * 2], part_b[kLsqrWarps * 2];
  const lsqr_desc d = descs[blockIdx.x];
  double* u = SMEM ? dyn : d.scratch;
  double* v = u + d.rows;
  double* x = v + d.cols;
  double* w = x + d.cols;
  const int T = kLsqrThreads;

  // u = b, beta = |b|
  double t1[1] = {0.0}, r1[1];
  for (int r = threadIdx.x; r < d.rows; r += T) {
    const double bv = d.b[r];
    u[r]            = bv;
    t1[0] += bv * bv;
  }
  block_sums<1>(t1, part_a, r1);
  double beta        = sqrt(r1[0]);
  const double bnorm = beta;
  if (!(beta > 0.0) || !isfinite(beta)) {
    for (int j = threadIdx.x; j < d.cols; j += T) d.z[j] = 0.0;
    if (threadIdx.x == 0) outs[blockIdx.x] = lsqr_out{0, 0, beta, 0.0};
    return;
  }
  double us = 1.0 / beta;  // the normalised u is u * us
  // v = Op^T u / beta, alpha = |v|; x = w = 0 (w becomes v_1 in the first transpose product)
  t1[0] = 0.0;
  slice_products(d.slices_q, d.cols, d.q_slice, d.q_idx, d.q_val, u, [&](int j, double acc) {
    const double vj = acc * us;
    v[j]            = vj;
    x[j]            = 0.0;
    w[j]            = 0.0;
    t1[0] += vj * vj;
  });
  block_sums<1>(t1, part_b, r1);
  double alpha  = sqrt(r1[0]);
  double vs     = alpha > 0.0 ? 1.0 / alpha : 0.0;
  double rhobar = alpha, phibar = beta, anorm2 = 0.0, xnorm = 0.0;
  double c1 = 0.0, c2 = 0.0;  // pending update: x += c1 w; w = v - c2 w
  double rnorm = beta, arnorm = alpha * beta;
  int flag = 3, it = 0;
  if (!(alpha > 0.0)) {
    flag = 2;  // Op^T b = 0: z = 0 is the least-squares solution
  } else {
    for (it = 1; it <= d.max_iter; ++it) {
      // u <- Op v - alpha u  (normalised v = v * vs, normalised u = u * us)
      t1[0] = 0.0;
      slice_products(d.slices_p, d.rows, d.p_slice, d.p_idx, d.p_val, v, [&](int r, double acc) {
        const double un = acc * vs - alpha * (u[r] * us);
        u[r]            = un;
        t1[0] += un * un;
      });
      block_sums<1>(t1, part_a, r1);
      beta = sqrt(r1[0]);
      us   = beta > 0.0 ? 1.0 / beta : 0.0;
      anorm2 += alpha * alpha + beta * beta;
      // pending x / w update, then v <- Op^T u - beta v
      double t2[2] = {0.0, 0.0}, r2[2];
      slice_products(d.slices_q, d.cols, d.q_slice, d.q_idx, d.q_val, u, [&](int j, double acc) {
        const double vo = v[j] * vs;
        double wj       = w[j];
        const double xj = x[j] + c1 * wj;
        wj              = vo - c2 * wj;
        x[j]            = xj;
        w[j]            = wj;
        const double vn = acc * us - beta * vo;
        v[j]            = vn;
        t2[0] += vn * vn;
        t2[1] += xj * xj;
      });
      block_sums<2>(t2, part_b, r2);
      alpha = sqrt(r2[0]);
      vs    = alpha > 0.0 ? 1.0 / alpha : 0.0;
      xnorm = sqrt(r2[1]);
      // Plane rotation (no damping) and the new pending update.
      const double rho = sqrt(rhobar * rhobar + beta * beta);
      const double cs = rhobar / rho, sn = beta / rho;
      const double theta = sn * alpha;
      rhobar             = -cs * alpha;
      const double phi   = cs * phibar;
      phibar             = sn * phibar;
      c1                 = phi / rho;
      c2                 = theta / rho;
      rnorm              = phibar;
      arnorm             = alpha * fabs(sn * phi);
      const double anorm = sqrt(anorm2);
      if (rnorm <= d.tol * bnorm + d.tol * anorm * xnorm) {
        flag = 1;
        break;
      }
      if (arnorm <= d.tol * anorm * rnorm) {
        flag = 2;
        break;
      }
      if (!(alpha > 0.0) || !(beta > 0.0)) {  // exact breakdown: the Krylov space is exhausted
        flag = 1;
        break;
      }
    }
    if (it > d.max_iter) it = d.max_iter;
  }
  // The last pending x update, then the result.
  for (int j = threadIdx.x; j < d.cols; j += T) d.z[j] = x[j] + c1 * w[j];
  if (threadIdx.x == 0) outs[blockIdx.x] = lsqr_out{it, flag, rnorm, arnorm};
}

// Host-side packing of one problem: equilibration, transposition, row sorting, sliced ELL.
struct packed {
  int rows = 0, cols = 0;
  std::vector<double> dr, dc;          // equilibration: Op_s = diag(dr) Op diag(dc)
  std::vector<int> perm_p, perm_q;     // sorted position -> original row (P) / column (Q rows)
  std::vector<int64_t> p_slice, q_slice;
  std::vector<int> p_idx, q_idx;
  std::vector<double> p_val, q_val, b;
};

// Sliced ELL of a CSR matrix (rows sorted by length, descending) whose column indices are mapped
// through `colmap`.
void to_sell(int rows, const std::vector<int64_t>& off, const std::vector<int>& idx,
             const std::vector<double>& val, const std::vector<int>& colmap,
             std::vector<int>& perm, std::vector<int64_t>& slice, std::vector<int>& sidx,
             std::vector<double>& sval)
{
  perm.resize(rows);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) {
    return off[a + 1] - off[a] > off[b + 1] - off[b];
  });
  const int slices = (rows + kWarp - 1) / kWarp;
  slice.assign(slices + 1, 0);
  for (int s = 0; s < slices; ++s) {
    const int r0      = perm[s * kWarp];  // the longest row of the slice comes first
    const int64_t len = off[r0 + 1] - off[r0];
    slice[s + 1]      = slice[s] + len * kWarp;
  }
  sidx.assign(slice[slices], 0);
  sval.assign(slice[slices], 0.0);
  for (int s = 0; s < slices; ++s)
    for (int t = 0; t < kWarp && s * kWarp + t < rows; ++t) {
      const int r = perm[s * kWarp + t];
      int k       = 0;
      for (int64_t e = off[r]; e < off[r + 1]; ++e, ++k) {
        sidx[slice[s] + (int64_t)k * kWarp + t] = colmap[idx[e]];
        sval[slice[s] + (int64_t)k * kWarp + t] = val[e];
      }
    }
}

void pack(const lsqr_problem& p, packed& out)
{
  const int R = p.rows, Cc = p.cols;
  out.rows = R;
  out.cols = Cc;
  const int64_t nnz = p.off[R];
  // Two-sided equilibration: repeatedly divide rows and columns by the square roots of their
  // 2-norms (computed from the same scaled matrix), which brings both towards unit norm.
  out.dr.assign(R, 1.0);
  out.dc.assign(Cc, 1.0);
  std::vector<double> rn(R), cn(Cc);
  for (int pass = 0; pass < kEquilibrationPasses; ++pass) {
    std::fill(rn.begin(), rn.end(), 0.0);
    std::fill(cn.begin(), cn.end(), 0.0);
    for (int r = 0; r < R; ++r)
      for (int64_t e = p.off[r]; e < p.off[r + 1]; ++e) {
        const double a = p.val[e] * out.dr[r] * out.dc[p.idx[e]];
        rn[r] += a * a;
        cn[p.idx[e]] += a * a;
      }
    for (int r = 0; r < R; ++r)
      if (rn[r] > 0.0) out.dr[r] /= std::sqrt(std::sqrt(rn[r]));
    for (int j = 0; j < Cc; ++j)
      if (cn[j] > 0.0) out.dc[j] /= std::sqrt(std::sqrt(cn[j]));
  }
  // Scaled P in CSR, and its transpose Q.
  std::vector<double> sv(nnz);
  for (int r = 0; r < R; ++r)
    for (int64_t e = p.off[r]; e < p.off[r + 1]; ++e)
      sv[e] = p.val[e] * out.dr[r] * out.dc[p.idx[e]];
  std::vector<int64_t> qoff(Cc + 1, 0);
  for (int64_t e = 0; e < nnz; ++e) ++qoff[p.idx[e] + 1];
  for (int j = 0; j < Cc; ++j) qoff[j + 1] += qoff[j];
  std::vector<int> qidx(nnz);
  std::vector<double> qval(nnz);
  {
    std::vector<int64_t> pos(qoff.begin(), qoff.end() - 1);
    for (int r = 0; r < R; ++r)
      for (int64_t e = p.off[r]; e < p.off[r + 1]; ++e) {
        const int64_t q = pos[p.idx[e]]++;
        qidx[q]         = r;
        qval[q]         = sv[e];
      }
  }
  // Row orders first (P's columns refer to Q's sorted rows and the other way round).
  std::vector<int> idp(R), idq(Cc);
  std::iota(idp.begin(), idp.end(), 0);
  std::iota(idq.begin(), idq.end(), 0);
  std::vector<int64_t> tmp_slice;
  std::vector<int> tmp_idx;
  std::vector<double> tmp_val;
  out.perm_p.resize(R);
  out.perm_q.resize(Cc);
  std::iota(out.perm_p.begin(), out.perm_p.end(), 0);
  std::stable_sort(out.perm_p.begin(), out.perm_p.end(), [&](int a, int b) {
    return p.off[a + 1] - p.off[a] > p.off[b + 1] - p.off[b];
  });
  std::iota(out.perm_q.begin(), out.perm_q.end(), 0);
  std::stable_sort(out.perm_q.begin(), out.perm_q.end(), [&](int a, int b) {
    return qoff[a + 1] - qoff[a] > qoff[b + 1] - qoff[b];
  });
  std::vector<int> inv_p(R), inv_q(Cc);
  for (int i = 0; i < R; ++i) inv_p[out.perm_p[i]] = i;
  for (int j = 0; j < Cc; ++j) inv_q[out.perm_q[j]] = j;
  std::vector<int> check;
  to_sell(R, p.off, p.idx, sv, inv_q, check, out.p_slice, out.p_idx, out.p_val);
  to_sell(Cc, qoff, qidx, qval, inv_p, check, out.q_slice, out.q_idx, out.q_val);
  out.b.resize(R);
  for (int i = 0; i < R; ++i) out.b[i] = p.b[out.perm_p[i]] * out.dr[out.perm_p[i]];
}

template <typename F>
void parallel_for(int count, F&& f)
{
  const int nt = std::max(1, std::min<int>(count, (int)std::thread::hardware_concurrency()));
  if (nt <= 1) {
    for (int i = 0; i < count; ++i) f(i);
    return;
  }
  std::vector<std::thread> pool;
  std::atomic<int> next{0};
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&]() {
      for (int i; (i = next++) < count;) f(i);
    });
  for (auto& th : pool) th.join();
}

}  // namespace

std::vector<lsqr_result> lsqr_solve_batch(const std::vector<const lsqr_problem*>& ps,
                                          cudaStream_t s, double tol, int max_iter)
{
  const int count = (int)ps.size();
  std::vector<lsqr_result> res(count);
  std::vector<packed> pk(count);
  for (int i = 0; i < count; ++i) {
    const lsqr_problem& p = *ps[i];
    if ((int)p.off.size() != p.rows + 1 || (int)p.b.size() != p.rows || p.rows < 0 || p.cols < 0 ||
        (int64_t)p.idx.size() < p.off[p.rows] || (int64_t)p.val.size() < p.off[p.rows])
      throw std::invalid_argument("lsqr: malformed problem");
    for (int64_t e = 0; e < p.off[p.rows]; ++e)
      if (p.idx[e] < 0 || p.idx[e] >= p.cols) throw std::invalid_argument("lsqr: column out of range");
  }
  parallel_for(count, [&](int i) { pack(*ps[i], pk[i]); });

  // Systems with work go to the device, split by where their vectors fit.
  std::vector<int> smem_ids, glob_ids;
  size_t smem_bytes = 0, scratch_doubles = 0;
  for (int i = 0; i < count; ++i) {
    res[i].z.assign(ps[i]->cols, 0.0);
    if (pk[i].rows == 0 || pk[i].cols == 0) continue;
    const size_t need = ((size_t)pk[i].rows + 3 * (size_t)pk[i].cols) * sizeof(double);
    if (need <= kSmemBudget) {
      smem_ids.push_back(i);
      smem_bytes = std::max(smem_bytes, need);
    } else {
      glob_ids.push_back(i);
      scratch_doubles += (size_t)pk[i].rows + 3 * (size_t)pk[i].cols;
    }
  }
  if (smem_ids.empty() && glob_ids.empty()) return res;

  // One upload of every array: offsets, indices, values, right-hand sides; outputs z.
  size_t n_off = 0, n_idx = 0, n_val = 0, n_b = 0, n_z = 0;
  auto order = smem_ids;
  order.insert(order.end(), glob_ids.begin(), glob_ids.end());
  for (int i : order) {
    n_off += pk[i].p_slice.size() + pk[i].q_slice.size();
    n_idx += pk[i].p_idx.size() + pk[i].q_idx.size();
    n_val += pk[i].p_val.size() + pk[i].q_val.size();
    n_b += pk[i].rows;
    n_z += pk[i].cols;
  }
  std::vector<int64_t> h_off;
  std::vector<int> h_idx;
  std::vector<double> h_val, h_b;
  h_off.reserve(n_off);
  h_idx.reserve(n_idx);
  h_val.reserve(n_val + n_b);
  h_b.reserve(n_b);
  struct where {
    size_t p_off, q_off, p_idx, q_idx, p_val, q_val, b, z, scratch;
  };
  std::vector<where> at(count);
  size_t z_pos = 0, scratch_pos = 0;
  for (int i : order) {
    const packed& q = pk[i];
    where w{};
    w.p_off = h_off.size();
    h_off.insert(h_off.end(), q.p_slice.begin(), q.p_slice.end());
    w.q_off = h_off.size();
    h_off.insert(h_off.end(), q.q_slice.begin(), q.q_slice.end());
    w.p_idx = h_idx.size();
    h_idx.insert(h_idx.end(), q.p_idx.begin(), q.p_idx.end());
    w.q_idx = h_idx.size();
    h_idx.insert(h_idx.end(), q.q_idx.begin(), q.q_idx.end());
    w.p_val = h_val.size();
    h_val.insert(h_val.end(), q.p_val.begin(), q.p_val.end());
    w.q_val = h_val.size();
    h_val.insert(h_val.end(), q.q_val.begin(), q.q_val.end());
    w.b = h_b.size();
    h_b.insert(h_b.end(), q.b.begin(), q.b.end());
    w.z = z_pos;
    z_pos += q.cols;
    w.scratch = scratch_pos;
    if (std::find(glob_ids.begin(), glob_ids.end(), i) != glob_ids.end())
      scratch_pos += (size_t)q.rows + 3 * (size_t)q.cols;
    at[i] = w;
  }
  alloc_scope scope(s);
  dbuf<int64_t> d_off(std::max<size_t>(h_off.size(), 1));
  dbuf<int> d_idx(std::max<size_t>(h_idx.size(), 1));
  dbuf<double> d_val(std::max<size_t>(h_val.size(), 1)), d_b(std::max<size_t>(h_b.size(), 1));
  dbuf<double> d_z(std::max<size_t>(n_z, 1)), d_scratch(std::max<size_t>(scratch_doubles, 1));
  d_off.upload(h_off.data(), h_off.size(), s);
  d_idx.upload(h_idx.data(), h_idx.size(), s);
  d_val.upload(h_val.data(), h_val.size(), s);
  d_b.upload(h_b.data(), h_b.size(), s);
  const int default_iter = max_iter;
  std::vector<lsqr_desc> h_desc;
  for (int i : order) {
    const packed& q = pk[i];
    const where& w  = at[i];
    lsqr_desc d{};
    d.rows     = q.rows;
    d.cols     = q.cols;
    d.slices_p = (int)q.p_slice.size() - 1;
    d.slices_q = (int)q.q_slice.size() - 1;
    d.p_slice  = d_off.data() + w.p_off;
    d.q_slice  = d_off.data() + w.q_off;
    d.p_idx    = d_idx.data() + w.p_idx;
    d.q_idx    = d_idx.data() + w.q_idx;
    d.p_val    = d_val.data() + w.p_val;
    d.q_val    = d_val.data() + w.q_val;
    d.b        = d_b.data() + w.b;
    d.z        = d_z.data() + w.z;
    d.scratch  = d_scratch.data() + w.scratch;
    d.tol      = tol;
    d.max_iter = default_iter > 0 ? default_iter
                                  : (int)std::min<long long>(200000, 20LL * (q.rows + q.cols));
    h_desc.push_back(d);
  }
  dbuf<lsqr_desc> d_desc(h_desc.size());
  dbuf<lsqr_out> d_out(h_desc.size());
  d_desc.upload(h_desc.data(), h_desc.size(), s);
  const int n_smem = (int)smem_ids.size(), n_glob = (int)glob_ids.size();
  if (n_smem > 0) {
    allow_max_dynamic_smem((const void*)lsqr_kernel<true>);
    lsqr_kernel<true><<<n_smem, kLsqrThreads, smem_bytes, s>>>(d_desc.data(), d_out.data());
    B200_LAUNCH_CHECK();
  }
  if (n_glob > 0) {
    lsqr_kernel<false><<<n_glob, kLsqrThreads, 0, s>>>(d_desc.data() + n_smem,
                                                       d_out.data() + n_smem);
    B200_LAUNCH_CHECK();
  }
  std::vector<double> h_z(n_z);
  std::vector<lsqr_out> h_out(h_desc.size());
  d_z.download(h_z.data(), n_z, s);
  d_out.download(h_out.data(), h_out.size(), s);
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  for (size_t k = 0; k < order.size(); ++k) {
    const int i     = order[k];
    const packed& q = pk[i];
    lsqr_result& r  = res[i];
    for (int j = 0; j < q.cols; ++j) {
      const int c = q.perm_q[j];
      r.z[c]      = h_z[at[i].z + j] * q.dc[c];
    }
    r.iterations = h_out[k].iterations;
    r.flag       = h_out[k].flag;
    r.rnorm      = h_out[k].rnorm;
    r.arnorm     = h_out[k].arnorm;
  }
  return res;
}

}  // namespace cuopt_b200
