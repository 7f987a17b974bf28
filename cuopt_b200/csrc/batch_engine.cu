// Batched PDLP: many independent LPs solved together as one block-diagonal LP.
//
// Counterpart of the reference's batch solve (the Python BatchSolve through
// cuopt::cython::call_batch_solve, cpp/src/pdlp/utilities/cython_solve.cu:317-352, which runs one
// PDLP per problem on host threads) and of its batch climbers (cpp/src/pdlp/pdlp.cu:1447-1746).
// Here the instances are concatenated into one block-diagonal matrix and every PDHG sweep is one
// launch over all of them; each row reads the step sizes of its own instance.  Every instance
// keeps its own Stable3 state — scaling factors, step size (its own power iteration), primal
// weight, restart / PID state and termination — and follows the schedule of a single solve: that
// schedule depends only on the iteration count, which all instances share.  An instance that
// terminates is frozen: the sweeps skip its rows and no kernel writes its vectors again.
//
// Per-instance sums (norms, residuals, fixed-point errors) are formed deterministically: the
// epilogues write one value per row into a row buffer, and one block per instance adds its rows in
// a fixed order (the layout keeps every instance's rows contiguous inside the long-row and the
// sliced parts, see make_keys_kernel).
#include "device_layout.cuh"
#include "host_io.hpp"
#include "kernels.cuh"
#include "pdlp_engine.hpp"
#include "pdlp_schedule.hpp"
#include "plain_form.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <tuple>
#include <random>
#include <stdexcept>

namespace cuopt_b200 {

namespace {

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
dev_sell<T> bview(const dev_matrix& M, const T* v)
{
  return dev_sell<T>{M.rows, M.n_long, M.n_slices, M.long_off.data(), M.slice_off.data(),
                     M.idx.data(), v};
}

// ------------------------------------------------------------------------------------------------
// Device side

// Instance lookup shared by the batch epilogues.
struct inst_ctx {
  const int* inst;         // instance of every internal row of the swept matrix
  const int* active;       // per instance: still iterating
  const pdlp_scalars* sc;  // per instance step scalars
  // Rows r0..r1 lie in one class (long or sliced), where instances are sorted, so the instances
  // present are inst[r0]..inst[r1].
  __device__ __forceinline__ bool all_frozen(int r0, int r1) const
  {
    for (int b = inst[r0]; b <= inst[r1]; ++b)
      if (active[b]) return false;
    return true;
  }
};

template <typename TX, bool MAJOR, bool HALPERN, bool SAVE_ATY>
struct b_primal_epi {
  static constexpr int kRed = 0;
  const TX *x, *c, *lo, *up, *xa;
  TX *xbar, *xout, *xhat, *slack, *aty;
  inst_ctx ctx;
  int it_off;
  struct pre_t {
    TX x, c, lo, up, xa;
    int b;
  };
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int j) const
  {
    return pre_t{x[j], c[j], lo[j], up[j], HALPERN ? xa[j] : TX(0), ctx.inst[j]};
  }
  __device__ __forceinline__ void operator()(int j, double acc, const pre_t& p, red_t<0>&) const
  {
    if (!ctx.active[p.b]) return;
    primal_row_step<TX, MAJOR, HALPERN, SAVE_ATY>(j, acc, p, ctx.sc + p.b, it_off, xbar, xout,
                                                  xhat, slack, aty);
  }
};

// FPE: rowbuf[i] = (y_bar_i - y_i)^2.
template <typename TX, bool MAJOR, bool HALPERN, bool FPE>
struct b_dual_epi {
  static constexpr int kRed = 0;
  const TX *y, *lo, *up, *ya;
  TX *ybar, *yout, *yhat;
  double* rowbuf;
  inst_ctx ctx;
  int it_off;
  struct pre_t {
    TX y, lo, up, ya;
    int b;
  };
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int i) const
  {
    return pre_t{y[i], lo[i], up[i], HALPERN ? ya[i] : TX(0), ctx.inst[i]};
  }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t& p, red_t<0>&) const
  {
    if (!ctx.active[p.b]) return;
    const double d2 =
      dual_row_step<TX, MAJOR, HALPERN>(i, acc, p, ctx.sc + p.b, it_off, ybar, yout, yhat);
    if constexpr (FPE) rowbuf[i] = d2;
  }
};

// rowbuf[j] = (A^T y_bar - A^T y)_j (x_bar - x)_j ; rowbuf[stride + j] = (x_bar - x)_j^2.
template <typename TX>
struct b_fpe_epi {
  static constexpr int kRed = 0;
  const TX *aty, *xbar, *x;
  double* rowbuf;
  size_t stride;
  inst_ctx ctx;
  struct pre_t {
    TX aty, xbar, x;
    int b;
  };
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int j) const
  {
    return pre_t{aty[j], xbar[j], x[j], ctx.inst[j]};
  }
  __device__ __forceinline__ void operator()(int j, double acc, const pre_t& p, red_t<0>&) const
  {
    if (!ctx.active[p.b]) return;
    const double d  = acc - (double)p.aty;
    const double dx = (double)p.xbar - (double)p.x;
    rowbuf[j]          = d * dx;
    rowbuf[stride + j] = dx * dx;
  }
};

// Unscaled termination terms of row i of A: rp^2 and the dual-objective bound term.
struct b_term_primal_epi {
  static constexpr int kRed = 0;
  const double *lc, *uc, *y;
  double* rowbuf;
  size_t stride;
  inst_ctx ctx;
  struct pre_t {
    double l, u, y;
    int b;
  };
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int i) const
  {
    return pre_t{lc[i], uc[i], y[i], ctx.inst[i]};
  }
  __device__ __forceinline__ void operator()(int i, double ax, const pre_t& p, red_t<0>&) const
  {
    if (!ctx.active[p.b]) return;
    const double cl = fmax(p.l, fmin(ax, p.u));
    const double rp = ax - cl;
    rowbuf[i]          = rp * rp;
    rowbuf[stride + i] = fmax(p.y, 0.0) * finite_or_zero(p.l) + fmin(p.y, 0.0) * finite_or_zero(p.u);
  }
};

// Unscaled termination terms of row j of A^T: rd^2, c.x, s.x.
struct b_term_dual_epi {
  static constexpr int kRed = 0;
  const double *c, *x, *s;
  double* rowbuf;
  size_t stride;
  inst_ctx ctx;
  struct pre_t {
    double c, x, s;
    int b;
  };
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int j) const
  {
    return pre_t{c[j], x[j], s[j], ctx.inst[j]};
  }
  __device__ __forceinline__ void operator()(int j, double aty, const pre_t& p, red_t<0>&) const
  {
    if (!ctx.active[p.b]) return;
    const double rd        = (p.c - aty) - p.s;
    rowbuf[j]              = rd * rd;
    rowbuf[stride + j]     = p.c * p.x;
    rowbuf[2 * stride + j] = p.s * p.x;
  }
};

// Power iteration sweeps: out = A^T q (store) and z = A (A^T q) with rowbuf = q z.
template <typename TX>
struct b_store_epi {
  static constexpr int kRed = 0;
  TX* out;
  inst_ctx ctx;
  struct pre_t {};
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int) const { return pre_t{}; }
  __device__ __forceinline__ void operator()(int r, double acc, const pre_t&, red_t<0>&) const
  {
    out[r] = (TX)acc;
  }
};
struct b_power_z_epi {
  static constexpr int kRed = 0;
  double* z;
  const double* q;
  double* rowbuf;
  inst_ctx ctx;
  struct pre_t {
    double q;
    int b;
  };
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int i) const { return pre_t{q[i], ctx.inst[i]}; }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t& p, red_t<0>&) const
  {
    if (!ctx.active[p.b]) return;
    z[i]      = acc;
    rowbuf[i] = p.q * acc;
  }
};

// Rows of an instance are processed in chunks of at most kChunkRows (each inside one instance), so
// a large instance does not serialise a kernel on one block.
constexpr int kChunkRows = 2048;

// Per-instance sums of row-buffer planes, for instances of any size: block c sums the K planes over its
// chunk (instance chunks[c].x, rows [chunks[c].y, chunks[c].z)) into part[c K + q]; then one
// thread per instance adds its chunks in chunk order.
template <int K>
__global__ void __launch_bounds__(kBlock) chunk_reduce_kernel(const double* rowbuf, size_t stride,
                                                              const int4* chunks, const int* want,
                                                              double* part)
{
  const int4 ch = chunks[blockIdx.x];
  if (want && !want[ch.x]) return;
  __shared__ double sm[kBlock];
  for (int q = 0; q < K; ++q) {
    const double* v = rowbuf + (size_t)q * stride;
    ksum acc;
    for (int i = ch.y + threadIdx.x; i < ch.z; i += kBlock) acc.add(v[i]);
    sm[threadIdx.x] = acc.value();
    __syncthreads();
    for (int h = kBlock / 2; h > 0; h >>= 1) {
      if (threadIdx.x < h) sm[threadIdx.x] += sm[threadIdx.x + h];
      __syncthreads();
    }
    if (threadIdx.x == 0) part[(size_t)blockIdx.x * K + q] = sm[0];
    __syncthreads();
  }
}

template <int K>
__global__ void instance_reduce_kernel(const double* part, const int* chunk_off, int count,
                                       const int* want, double* out)
{
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x) {
    if (want && !want[b]) continue;
    for (int q = 0; q < K; ++q) {
      double t = 0.0;
      for (int c = chunk_off[b]; c < chunk_off[b + 1]; ++c) t += part[(size_t)c * K + q];
      out[(size_t)b * K + q] = t;
    }
  }
}

// Elementwise fills of the row buffer.
template <typename TA>
__global__ void sq_diff_kernel(const TA* a, const TA* b, int n, double* out)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double d = b ? (double)a[i] - (double)b[i] : (double)a[i];
    out[i]         = d * d;
  }
}
__global__ void bound_terms_kernel(const double* lo, const double* up, int n, double* out)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double l = lo[i], u = up[i];
    double s       = 0.0;
    if (isfinite(l) && l != u) s += l * l;
    if (isfinite(u)) s += u * u;
    out[i] = s;
  }
}

// Instance ranges in the internal order, where each instance's items are contiguous inside
// [0, n_long) and inside [n_long, count): r[b] = {long_lo, long_hi, short_lo, short_hi}.  Segment
// starts and ends are found where the instance id changes; an id out of [0, B) or a decrease
// inside a part (instances not contiguous) is counted in bad[0].  r must be zeroed first.
__global__ void instance_ranges_kernel(const int* inst, int count, int n_long, int B, int4* r,
                                       int* bad)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const int b = inst[i];
    if (b < 0 || b >= B) {
      atomicAdd(bad, 1);
      continue;
    }
    const bool is_long = i < n_long;
    const bool first   = i == 0 || i == n_long;
    const bool last    = i == count - 1 || i == n_long - 1;
    const int prev     = first ? -1 : inst[i - 1];
    const int next     = last ? -1 : inst[i + 1];
    if (!first && prev > b) atomicAdd(bad, 1);
    if (first || prev != b) {
      if (is_long)
        r[b].x = i;
      else
        r[b].z = i;
    }
    if (last || next != b) {
      if (is_long)
        r[b].y = i + 1;
      else
        r[b].w = i + 1;
    }
  }
}

__global__ void gather_int_kernel(const int* src, const int* perm, int count, int* dst)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    dst[i] = src[perm[i]];
}
__global__ void scale_by_inst_kernel(double* v, const int* inst, const double* f, int count)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    v[i] *= f[inst[i]];
}
// dst[perm[i]] = f[inst[i]] * src[i]
__global__ void scatter_by_inst_kernel(const double* src, const int* perm, const int* inst,
                                       const double* f, int count, double* dst)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x)
    dst[perm[i]] = (f ? f[inst[i]] : 1.0) * src[i];
}

// Bound / objective rescaling with each instance's beta and gamma.
template <typename TX>
__global__ void b_rescale_vectors_kernel(const double* cs, const double* ls, const double* us,
                                         const double* lcs, const double* ucs, const double* beta,
                                         const double* gamma, const int* cinst, const int* rinst,
                                         int n, int m, TX* c_out, TX* l_out, TX* u_out, TX* lc_out,
                                         TX* uc_out)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n) {
      const int b = cinst[i];
      c_out[i]    = (TX)(cs[i] * gamma[b]);
      l_out[i]    = (TX)(ls[i] * beta[b]);
      u_out[i]    = (TX)(us[i] * beta[b]);
    } else {
      const int r = i - n, b = rinst[r];
      lc_out[r]   = (TX)(lcs[r] * beta[b]);
      uc_out[r]   = (TX)(ucs[r] * beta[b]);
    }
  }
}

template <typename TX>
__global__ void b_unscale_kernel(const TX* xhat, const TX* yhat, const TX* slack, const double* dc,
                                 const double* dr, const double* beta, const double* gamma,
                                 const int* cinst, const int* rinst, const int* active, int n,
                                 int m, double* xu, double* yu, double* su)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n) {
      const int b = cinst[i];
      if (!active[b]) continue;
      const double ib = 1.0 / beta[b], ig = 1.0 / gamma[b];
      const double d  = dc[i];
      xu[i]           = ((double)xhat[i] * d) * ib;
      const double s  = (double)slack[i];
      su[i]           = (d != 0.0 ? s / d : s) * ig;
    } else {
      const int r = i - n, b = rinst[r];
      if (!active[b]) continue;
      yu[r] = ((double)yhat[r] * dr[r]) * (1.0 / gamma[b]);
    }
  }
}

template <typename TX>
__global__ void b_halpern_kernel(TX* x, const TX* xbar, const TX* xa, int n, TX* y, const TX* ybar,
                                 const TX* ya, int m, const int* cinst, const int* rinst,
                                 const int* active, const pdlp_scalars* sc)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n) {
      const int b = cinst[i];
      if (!active[b]) continue;
      const double w = halpern_weight(sc + b, 0);
      x[i]           = (TX)(w * (double)xbar[i] + (1.0 - w) * (double)xa[i]);
    } else {
      const int r = i - n, b = rinst[r];
      if (!active[b]) continue;
      const double w = halpern_weight(sc + b, 0);
      y[r]           = (TX)(w * (double)ybar[r] + (1.0 - w) * (double)ya[r]);
    }
  }
}

// Restart to the current average: x, x_anchor <- x_hat (and y) for flagged instances.
template <typename TX>
__global__ void b_restart_kernel(TX* x, TX* xa, const TX* xhat, int n, TX* y, TX* ya,
                                 const TX* yhat, int m, const int* cinst, const int* rinst,
                                 const int* flag)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n + m; i += gridDim.x * blockDim.x) {
    if (i < n) {
      if (!flag[cinst[i]]) continue;
      x[i]  = xhat[i];
      xa[i] = xhat[i];
    } else {
      const int r = i - n;
      if (!flag[rinst[r]]) continue;
      y[r]  = yhat[r];
      ya[r] = yhat[r];
    }
  }
}

// Warm start: a = b = c = v / d (v / d = v where d = 0) times the instance's factor f[inst].
template <typename TX>
__global__ void b_scale_initial_kernel(const double* v, const double* d, const int* inst,
                                       const double* f, int n, TX* a, TX* b, TX* c)
{
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double s = d[i] != 0.0 ? v[i] / d[i] : v[i];
    const TX w     = (TX)(s * f[inst[i]]);
    a[i]           = w;
    b[i]           = w;
    c[i]           = w;
  }
}

__global__ void b_advance_kernel(pdlp_scalars* sc, const int* active, int count, int steps)
{
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x)
    if (active[b]) sc[b].t0 += steps;
}

// Power iteration per instance (reference pdlp.cu:2620-2731), one block per instance.
struct b_power_state {
  double s2;
  double resid;
  int iters;
  int pad;
};

// Fixed-order block sum of per-thread values (compensated per thread, then a fixed tree).
__device__ __forceinline__ double block_sum(const ksum& acc, double* sm)
{
  sm[threadIdx.x] = acc.value();
  __syncthreads();
  for (int h = kBlock / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h) sm[threadIdx.x] += sm[threadIdx.x + h];
    __syncthreads();
  }
  const double v = sm[0];
  __syncthreads();
  return v;
}

// The power iteration's vector work runs on the same row chunks; chunk partial sums are combined
// per instance in chunk order (deterministic).

// Thread 0's fixed-order sum of the partials of instance b's chunks, shared with the block.
__device__ __forceinline__ double instance_total(const double* part, const int* chunk_off, int b,
                                                 double* slot)
{
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int c = chunk_off[b]; c < chunk_off[b + 1]; ++c) t += part[c];
    *slot = t;
  }
  __syncthreads();
  return *slot;
}

// part[c] = sum of z^2 over chunk c.
__global__ void __launch_bounds__(kBlock) b_chunk_sumsq_kernel(const int4* chunks, const int* pactive,
                                                               const double* z, double* part)
{
  const int4 ch = chunks[blockIdx.x];
  if (!pactive[ch.x]) return;
  __shared__ double sm[kBlock];
  ksum acc;
  for (int i = ch.y + threadIdx.x; i < ch.z; i += kBlock) acc.add(z[i] * z[i]);
  const double v = block_sum(acc, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}

// q = z / |z| over chunk c (|z| of its instance).
__global__ void __launch_bounds__(kBlock)
  b_chunk_normalize_kernel(const int4* chunks, const int* chunk_off, const int* pactive,
                           const double* part, const double* z, double* q)
{
  const int4 ch = chunks[blockIdx.x];
  if (!pactive[ch.x]) return;
  __shared__ double slot;
  const double nq = sqrt(instance_total(part, chunk_off, ch.x, &slot));
  for (int i = ch.y + threadIdx.x; i < ch.z; i += kBlock) q[i] = z[i] / nq;
}

// part[c] = sum of rowbuf (q_i z_i) over chunk c.
__global__ void __launch_bounds__(kBlock) b_chunk_sum_kernel(const int4* chunks, const int* pactive,
                                                             const double* v, double* part)
{
  const int4 ch = chunks[blockIdx.x];
  if (!pactive[ch.x]) return;
  __shared__ double sm[kBlock];
  ksum acc;
  for (int i = ch.y + threadIdx.x; i < ch.z; i += kBlock) acc.add(v[i]);
  const double t = block_sum(acc, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// The power iteration's step folds the next step's norm and normalisation into this step's
// chunk kernels (same values as the separate kernels above, two launches fewer per step):
// part[c] = sum of rowbuf (q_i z_i) over chunk c and part_z[c] = sum of z_i^2 over chunk c.
__global__ void __launch_bounds__(kBlock)
  b_chunk_sum_sumsq_kernel(const int4* chunks, const int* pactive, const double* v,
                           const double* z, double* part, double* part_z)
{
  const int4 ch = chunks[blockIdx.x];
  if (!pactive[ch.x]) return;
  __shared__ double sm[kBlock];
  ksum acc, acc_z;
  for (int i = ch.y + threadIdx.x; i < ch.z; i += kBlock) {
    acc.add(v[i]);
    acc_z.add(z[i] * z[i]);
  }
  const double t   = block_sum(acc, sm);
  const double t_z = block_sum(acc_z, sm);
  if (threadIdx.x == 0) {
    part[blockIdx.x]   = t;
    part_z[blockIdx.x] = t_z;
  }
}

// s2 = q . z of the instance;  part_r[c] = sum over chunk c of (z - s2 q)^2;  then q <- z / |z|,
// the next step's normalised vector.
__global__ void __launch_bounds__(kBlock)
  b_chunk_residual_next_kernel(const int4* chunks, const int* chunk_off, const int* pactive,
                               const double* part_s2, const double* part_z, const double* z,
                               double* q, double* part_r)
{
  const int4 ch = chunks[blockIdx.x];
  if (!pactive[ch.x]) return;
  __shared__ double slot, slot_z;
  __shared__ double sm[kBlock];
  const double s2 = instance_total(part_s2, chunk_off, ch.x, &slot);
  const double nq = sqrt(instance_total(part_z, chunk_off, ch.x, &slot_z));
  ksum acc;
  for (int i = ch.y + threadIdx.x; i < ch.z; i += kBlock) {
    const double v = q[i] * -s2 + z[i];
    acc.add(v * v);
    q[i] = z[i] / nq;
  }
  const double t = block_sum(acc, sm);
  if (threadIdx.x == 0) part_r[blockIdx.x] = t;
}

// Per instance: record sigma^2 and the residual, test convergence.
__global__ void b_power_check_kernel(const int* chunk_off, int count, const double* part_s2,
                                     const double* part_r, int* pactive, b_power_state* ps,
                                     double tol, int* remaining)
{
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x) {
    if (!pactive[b]) continue;
    double s2 = 0.0, r = 0.0;
    for (int c = chunk_off[b]; c < chunk_off[b + 1]; ++c) {
      s2 += part_s2[c];
      r += part_r[c];
    }
    ps[b].s2    = s2;
    ps[b].resid = sqrt(r);
    ps[b].iters += 1;
    if (ps[b].resid < tol) {
      pactive[b] = 0;
      atomicSub(remaining, 1);
    }
  }
}

// Golub-Kahan-Lanczos step size per instance (mixed precision), the single engine's
// lanczos_step_size run on every instance at once: u and v hold the unnormalised Lanczos vectors,
// st[b] their norms, and rowbuf the squares of the new vector for the per-instance norms.
struct b_gk_state {
  double beta;
  double alpha;
};

// Row j of A^T applied to u:  p_j = (A^T u)_j / beta - beta v_j / alpha  (written over v_j).
struct b_gk_primal_epi {
  static constexpr int kRed = 0;
  double* v;
  double* rowbuf;
  const b_gk_state* st;
  inst_ctx ctx;
  struct pre_t {
    double v;
    int b;
  };
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int j) const { return pre_t{v[j], ctx.inst[j]}; }
  __device__ __forceinline__ void operator()(int j, double acc, const pre_t& p, red_t<0>&) const
  {
    if (!ctx.active[p.b]) return;
    const double b = st[p.b].beta, a = st[p.b].alpha;
    const double pj = acc / b - (a > 0.0 ? b * (p.v / a) : 0.0);
    v[j]            = pj;
    rowbuf[j]       = pj * pj;
  }
};

// Row i of A applied to v:  q_i = (A v)_i / alpha - alpha u_i / beta  (written over u_i).
struct b_gk_dual_epi {
  static constexpr int kRed = 0;
  double* u;
  double* rowbuf;
  const b_gk_state* st;
  inst_ctx ctx;
  struct pre_t {
    double u;
    int b;
  };
  __device__ bool skip() const { return false; }
  __device__ bool skip_range(int r0, int r1) const { return ctx.all_frozen(r0, r1); }
  __device__ __forceinline__ pre_t load(int i) const { return pre_t{u[i], ctx.inst[i]}; }
  __device__ __forceinline__ void operator()(int i, double acc, const pre_t& p, red_t<0>&) const
  {
    if (!ctx.active[p.b]) return;
    const double a = st[p.b].alpha, b = st[p.b].beta;
    const double qi = acc / a - a * (p.u / b);
    u[i]            = qi;
    rowbuf[i]       = qi * qi;
  }
};

// Per iterating instance b, the norm of its new vector from the chunk sums: FIELD 0 sets alpha
// (hist[k * count + b]), FIELD 1 sets beta (hist[(k + 1) * count + b]).
template <int FIELD>
__global__ void b_gk_record_kernel(const int* chunk_off, int count, const double* part,
                                   const int* active, b_gk_state* st, double* hist, int k)
{
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x) {
    if (!active[b]) continue;
    double t = 0.0;
    for (int c = chunk_off[b]; c < chunk_off[b + 1]; ++c) t += part[c];
    const double v = sqrt(t);
    if (FIELD == 0) {
      st[b].alpha                     = v;
      hist[(size_t)k * count + b]     = v;
    } else {
      st[b].beta                      = v;
      hist[(size_t)(k + 1) * count + b] = v;
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Host side

struct inst_conv {
  double l2_primal = 0, l2_dual = 0, primal_obj = 0, dual_obj = 0, gap = 0, abs_obj = 0;
};

// Timing decisions of batch solves, remembered for the life of the process as those of single
// solves are: per batch shape (rows, columns, non-zeros, instances), device, iterate precision and
// the parameter that restricts the decision, and for the form of the plain iterations per set of
// active instances (a hash of their indices; 0 when all are active).  A later solve of the same
// batch reuses them instead of timing again.
using batch_key = std::tuple<int, int, int64_t, int, int, int, int, uint64_t>;
struct batch_form_choice {
  int form;
  double us[2];  // graphs, persistent kernel: microseconds per iteration when it was chosen
};
struct batch_shape_choice {
  int wpb_primal, wpb_dual;
  double ms[2][3];
};
std::mutex& batch_tune_mutex()
{
  static std::mutex mu;
  return mu;
}
std::map<batch_key, batch_form_choice>& batch_form_cache()
{
  static std::map<batch_key, batch_form_choice> c;
  return c;
}
std::map<batch_key, batch_shape_choice>& batch_shape_cache()
{
  static std::map<batch_key, batch_shape_choice> c;
  return c;
}
// FNV-1a hash of the indices of the active instances (0 when every instance is active).
uint64_t active_set_hash(const std::vector<int>& act)
{
  if (std::all_of(act.begin(), act.end(), [](int a) { return a != 0; })) return 0;
  uint64_t h = 1469598103934665603ull;
  for (size_t b = 0; b < act.size(); ++b)
    if (act[b]) {
      h ^= (uint64_t)b + 1;
      h *= 1099511628211ull;
    }
  return h == 0 ? 1 : h;
}

template <typename TX>
class batch_engine {
 public:
  batch_engine(const batch_device_input& in, const pdlp_params& p, cudaStream_t s)
    : in_(in), p_(p), s_(s), B_(in.count)
  {
    int dev = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
    B200_CUDA_CHECK(cudaMallocHost(&hbuf_, sizeof(double) * 8 * (size_t)std::max(B_, 1)));
    B200_CUDA_CHECK(cudaMallocHost(&hstatus_, sizeof(int)));
  }
  ~batch_engine()
  {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    cudaFreeHost(hbuf_);
    cudaFreeHost(hstatus_);
  }

  std::vector<pdlp_result> run(double* x_out, double* y_out, double* rc_out)
  {
    alloc_scope scope(s_);
    t_start_ = now_s();
    results_.assign(B_, pdlp_result{});
    setup();
    tune_sweep_shape();
    init_plain_form(B_);
    t_loop_ = now_s();
    loop();
    trace("batch: loop");
    write_outputs(x_out, y_out, rc_out);
    const double t = now_s();
    for (int b = 0; b < B_; ++b) {
      results_[b].setup_time      = t_loop_ - t_start_;
      results_[b].loop_time       = results_[b].solve_time - (t_loop_ - t_start_);
      results_[b].kernel_launches = launches_;
      results_[b].power_iterations = power_iters_[b];
      results_[b].plain_form          = first_form_;
      results_[b].persistent_blocks   = first_blocks_;
      results_[b].us_plain_graphs     = first_us_[0];
      results_[b].us_plain_persistent = first_us_[1];
      results_[b].wpb_primal          = wpb_primal_;
      results_[b].wpb_dual            = wpb_dual_;
      std::memcpy(results_[b].wpb_ms, wpb_ms_, sizeof(wpb_ms_));
    }
    (void)t;
    return results_;
  }

 private:
  // ---------------------------------------------------------------- setup
  void setup()
  {
    const int m = in_.m, n = in_.n;
    layout_params lp;
    lp.row_inst = in_.row_inst;
    lp.col_inst = in_.col_inst;
    trace("batch: start");
    build_device_layout(m, n, in_.row_off, in_.col_idx, in_.val, s_, L_, lp);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    trace("batch: layout");
    vgrid_ = sms_ * 4;
    const int g = std::max({sell_grid(bview(L_.A, L_.A.val.data())),
                            sell_grid(bview(L_.AT, L_.AT.val.data())), vgrid_});
    partials_.resize((size_t)g * 4);
    stride_ = (size_t)std::max(m, n);
    rowbuf_.resize(3 * stride_);
    segout_.resize((size_t)B_ * 8);

    // Instance of every internal row / column, and each instance's ranges.
    rinst_.resize(m);
    cinst_.resize(n);
    gather_int_kernel<<<vgrid_, kBlock, 0, s_>>>(in_.row_inst, L_.row_new2old.data(), m,
                                                 rinst_.data());
    gather_int_kernel<<<vgrid_, kBlock, 0, s_>>>(in_.col_inst, L_.col_new2old.data(), n,
                                                 cinst_.data());
    B200_LAUNCH_CHECK();
    rranges_ = ranges_of(rinst_, m, L_.A.n_long);
    cranges_ = ranges_of(cinst_, n, L_.AT.n_long);
    trace("batch: instance ranges");
    rr_d_.resize(B_);
    cr_d_.resize(B_);
    rr_d_.upload(rranges_.data(), B_, s_);
    cr_d_.upload(cranges_.data(), B_, s_);
    build_chunks(rranges_, rows_);
    build_chunks(cranges_, cols_);

    // Per-instance sign (maximisation) and objective scale / offset.
    std::vector<double> sgn(B_);
    obj_scale_.resize(B_);
    obj_offset_.resize(B_);
    for (int b = 0; b < B_; ++b) {
      const bool mx  = in_.maximize[b] != 0;
      sgn[b]         = mx ? -1.0 : 1.0;
      obj_scale_[b]  = mx ? -1.0 : 1.0;
      obj_offset_[b] = mx ? -in_.obj_offset[b] : in_.obj_offset[b];
    }
    sgn_d_.resize(B_);
    sgn_d_.upload(sgn.data(), B_, s_);

    c64_.resize(n);
    l64_.resize(n);
    u64_.resize(n);
    lc64_.resize(m);
    uc64_.resize(m);
    permute_gather(in_.c, L_.col_new2old.data(), n, 1.0, c64_.data(), s_);
    scale_by_inst_kernel<<<vgrid_, kBlock, 0, s_>>>(c64_.data(), cinst_.data(), sgn_d_.data(), n);
    permute_gather(in_.var_lo, L_.col_new2old.data(), n, 1.0, l64_.data(), s_);
    permute_gather(in_.var_up, L_.col_new2old.data(), n, 1.0, u64_.data(), s_);
    permute_gather(in_.con_lo, L_.row_new2old.data(), m, 1.0, lc64_.data(), s_);
    permute_gather(in_.con_up, L_.row_new2old.data(), m, 1.0, uc64_.data(), s_);

    // Ruiz (10 passes) then Pock-Chambolle (alpha = 1); row / column operations, so the batch
    // scales every instance exactly as a single solve would (reference initial_scaling.cu:152-365).
    const auto A64 = bview(L_.A, L_.A.val.data()), AT64 = bview(L_.AT, L_.AT.val.data());
    dr_.resize(m);
    dc_.resize(n);
    fill(dr_.data(), m, 1.0);
    fill(dc_.data(), n, 1.0);
    dbuf<double> rtmp(m), ctmp(n);
    for (int it = 0; it < kRuizIterations; ++it) {
      row_scaled_abs_kernel<0, false><<<sell_grid(A64), kBlock, 0, s_>>>(A64, dr_.data(),
                                                                        dc_.data(), 0.0,
                                                                        rtmp.data());
      row_scaled_abs_kernel<0, true><<<sell_grid(AT64), kBlock, 0, s_>>>(AT64, dr_.data(),
                                                                        dc_.data(), 0.0,
                                                                        ctmp.data());
      apply_root_scaling_kernel<<<vgrid_, kBlock, 0, s_>>>(dr_.data(), rtmp.data(), m);
      apply_root_scaling_kernel<<<vgrid_, kBlock, 0, s_>>>(dc_.data(), ctmp.data(), n);
    }
    row_scaled_abs_kernel<1, false><<<sell_grid(A64), kBlock, 0, s_>>>(A64, dr_.data(), dc_.data(),
                                                                      kPcAlpha, rtmp.data());
    row_scaled_abs_kernel<1, true><<<sell_grid(AT64), kBlock, 0, s_>>>(
      AT64, dr_.data(), dc_.data(), 2.0 - kPcAlpha, ctmp.data());
    apply_root_scaling_kernel<<<vgrid_, kBlock, 0, s_>>>(dr_.data(), rtmp.data(), m);
    apply_root_scaling_kernel<<<vgrid_, kBlock, 0, s_>>>(dc_.data(), ctmp.data(), n);
    B200_LAUNCH_CHECK();
    As_.resize(L_.A.stored());
    ATs_.resize(L_.AT.stored());
    scale_values_kernel<TX, false><<<sell_grid(A64), kBlock, 0, s_>>>(A64, dr_.data(), dc_.data(),
                                                                     As_.data());
    scale_values_kernel<TX, true><<<sell_grid(AT64), kBlock, 0, s_>>>(AT64, dr_.data(),
                                                                     dc_.data(), ATs_.data());
    B200_LAUNCH_CHECK();

    // All instances active from here on (the power iteration has its own flags).
    active_h_.assign(B_, 1);
    active_d_.resize(B_);
    active_d_.upload(active_h_.data(), B_, s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    trace("batch: ranges + scaling");
    prepare_vectors();
    trace("batch: vectors");
    // Step size from the largest singular value of each scaled instance: the power iteration
    // (reference pdlp.cu:2620-2731), or Golub-Kahan-Lanczos in mixed precision, as single solves.
    if ((int)in_.initial_step.size() == B_) {
      eta_ = in_.initial_step;
      power_iters_.assign(B_, 0);
    } else if (p_.precision == 1)
      lanczos_step_size();
    else
      power_iteration();
    trace("batch: step size");

    xu_.resize(n);
    su_.resize(n);
    yu_.resize(m);
    xu_.zero(s_);
    su_.zero(s_);
    yu_.zero(s_);
    sc_d_.resize(B_);
    if ((int)in_.initial_weight.size() == B_)
      omega_ = in_.initial_weight;
    else
      omega_.assign(B_, 1.0);
    best_omega_ = omega_;
    restarts_.assign(B_, 0);
    for (auto* b : {&x_, &xhat_, &slack_, &xbar_, &xa_, &aty_}) {
      b->resize(n);
      b->zero(s_);
    }
    for (auto* b : {&y_, &yhat_, &ybar_, &ya_}) {
      b->resize(m);
      b->zero(s_);
    }
    // Warm start: iterate, anchor and x_hat from the initial solution in the scaled space (the
    // single engine's load_initial_solution, per instance).
    if (in_.initial_primal) {
      dbuf<double> v(n);
      permute_gather(in_.initial_primal, L_.col_new2old.data(), n, 1.0, v.data(), s_);
      b_scale_initial_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(v.data(), dc_.data(), cinst_.data(),
                                                            beta_d_.data(), n, x_.data(),
                                                            xhat_.data(), xa_.data());
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    }
    if (in_.initial_dual) {
      dbuf<double> v(m);
      permute_gather(in_.initial_dual, L_.row_new2old.data(), m, 1.0, v.data(), s_);
      b_scale_initial_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(v.data(), dr_.data(), rinst_.data(),
                                                            gamma_d_.data(), m, y_.data(),
                                                            yhat_.data(), ya_.data());
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    }
    clamp_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(x_.data(), ls_.data(), us_.data(), n);
    launches_ += 1;
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  // Ranges {long_lo, long_hi, short_lo, short_hi} of every instance in an internal order whose
  // instance ids are sorted inside [0, n_long) and inside [n_long, count).
  std::vector<int4> ranges_of(const dbuf<int>& inst, int count, int n_long)
  {
    dbuf<int4> r(B_);
    dbuf<int> bad(1);
    r.zero(s_);
    bad.zero(s_);
    if (count > 0)
      instance_ranges_kernel<<<vgrid_, kBlock, 0, s_>>>(inst.data(), count, n_long, B_, r.data(),
                                                        bad.data());
    B200_LAUNCH_CHECK();
    std::vector<int4> h(B_);
    int hbad = 0;
    r.download(h.data(), B_, s_);
    bad.download(&hbad, 1, s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    if (hbad) throw std::runtime_error("batch layout: instance ids out of range or not contiguous");
    return h;
  }

  void fill(double* p, int n, double v)
  {
    fill_kernel<<<vgrid_, kBlock, 0, s_>>>(p, n, v);
    ++launches_;
    B200_LAUNCH_CHECK();
  }

  // Per-instance sums of K planes of the row buffer over rows (ROWS) or columns; result in
  // segout_ + offset, optionally only for active instances.
  // Row chunks of every instance (rows of A, or of A^T for the columns), see kChunkRows.
  struct chunk_table {
    dbuf<int4> chunks;
    dbuf<int> offsets;
    int count = 0;
  };
  void build_chunks(const std::vector<int4>& ranges, chunk_table& t)
  {
    std::vector<int4> chunks;
    std::vector<int> off(B_ + 1, 0);
    for (int b = 0; b < B_; ++b) {
      off[b]       = (int)chunks.size();
      const int4 r = ranges[b];
      for (int lo = r.x; lo < r.y; lo += kChunkRows)
        chunks.push_back(int4{b, lo, std::min(lo + kChunkRows, r.y), 0});
      for (int lo = r.z; lo < r.w; lo += kChunkRows)
        chunks.push_back(int4{b, lo, std::min(lo + kChunkRows, r.w), 0});
    }
    off[B_] = (int)chunks.size();
    t.count = (int)chunks.size();
    t.chunks.resize(std::max(t.count, 1));
    t.offsets.resize(B_ + 1);
    if (t.count > 0) t.chunks.upload(chunks.data(), t.count, s_);
    t.offsets.upload(off.data(), B_ + 1, s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  // Per-instance sums of K planes of the row buffer over rows (ROWS) or columns; result in
  // segout_ + offset, optionally only for active instances.
  template <int K>
  void seg_reduce(bool rows, size_t offset, bool only_active)
  {
    const chunk_table& t = rows ? rows_ : cols_;
    const int* want      = only_active ? active_d_.data() : nullptr;
    if (chunk_part_.size() < (size_t)std::max(rows_.count, cols_.count) * 3)
      chunk_part_.resize((size_t)std::max({rows_.count, cols_.count, 1}) * 3);
    if (t.count > 0)
      chunk_reduce_kernel<K><<<t.count, kBlock, 0, s_>>>(rowbuf_.data(), stride_, t.chunks.data(),
                                                         want, chunk_part_.data());
    instance_reduce_kernel<K><<<ceil_div(B_, kBlock), kBlock, 0, s_>>>(
      chunk_part_.data(), t.offsets.data(), B_, want, segout_.data() + offset);
    launches_ += 2;
  }
  void fetch(size_t offset, size_t count, double* dst)
  {
    B200_CUDA_CHECK(cudaMemcpyAsync(dst, segout_.data() + offset, count * sizeof(double),
                                    cudaMemcpyDeviceToHost, s_));
    if (persist_used_)
      B200_CUDA_CHECK(cudaMemcpyAsync(hstatus_, &pctl_.data()->status, sizeof(int),
                                      cudaMemcpyDeviceToHost, s_));
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    if (persist_used_) {
      persist_used_ = false;
      if (*hstatus_ != 0)
        throw cuda_error(*hstatus_ == kBarrierTimedOut
                           ? "persistent batch iterations: a grid barrier passed its deadline"
                           : "persistent batch iterations: a grid barrier passed its poll limit");
    }
    collect_form_timing();
  }

  void prepare_vectors()
  {
    const int m = in_.m, n = in_.n;
    std::vector<double> h(4 * (size_t)B_);
    sq_diff_kernel<double><<<vgrid_, kBlock, 0, s_>>>(c64_.data(), nullptr, n, rowbuf_.data());
    seg_reduce<1>(false, 0, false);
    bound_terms_kernel<<<vgrid_, kBlock, 0, s_>>>(lc64_.data(), uc64_.data(), m, rowbuf_.data());
    seg_reduce<1>(true, B_, false);
    dbuf<double> cs(n), ls(n), us(n), lcs(m), ucs(m);
    scale_vectors_kernel<<<vgrid_, kBlock, 0, s_>>>(c64_.data(), l64_.data(), u64_.data(),
                                                    lc64_.data(), uc64_.data(), dc_.data(),
                                                    dr_.data(), n, m, cs.data(), ls.data(),
                                                    us.data(), lcs.data(), ucs.data());
    sq_diff_kernel<double><<<vgrid_, kBlock, 0, s_>>>(cs.data(), nullptr, n, rowbuf_.data());
    seg_reduce<1>(false, 2 * (size_t)B_, false);
    bound_terms_kernel<<<vgrid_, kBlock, 0, s_>>>(lcs.data(), ucs.data(), m, rowbuf_.data());
    seg_reduce<1>(true, 3 * (size_t)B_, false);
    launches_ += 5;
    B200_LAUNCH_CHECK();
    fetch(0, 4 * (size_t)B_, h.data());
    c_norm_.resize(B_);
    b_norm_.resize(B_);
    std::vector<double> beta(B_), gamma(B_);
    for (int b = 0; b < B_; ++b) {
      c_norm_[b] = std::sqrt(h[b]);
      b_norm_[b] = std::sqrt(h[B_ + b]);
      gamma[b]   = 1.0 / (std::sqrt(h[2 * B_ + b]) + 1.0);
      beta[b]    = 1.0 / (std::sqrt(h[3 * B_ + b]) + 1.0);
    }
    beta_d_.resize(B_);
    gamma_d_.resize(B_);
    beta_d_.upload(beta.data(), B_, s_);
    gamma_d_.upload(gamma.data(), B_, s_);
    beta_  = beta;
    gamma_ = gamma;
    cs_.resize(n);
    ls_.resize(n);
    us_.resize(n);
    lcs_.resize(m);
    ucs_.resize(m);
    b_rescale_vectors_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(
      cs.data(), ls.data(), us.data(), lcs.data(), ucs.data(), beta_d_.data(), gamma_d_.data(),
      cinst_.data(), rinst_.data(), n, m, cs_.data(), ls_.data(), us_.data(), lcs_.data(),
      ucs_.data());
    ++launches_;
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  // Power iteration of every instance (graph chunks of 32 iterations; converged instances freeze).
  void power_iteration()
  {
    const int m = in_.m, n = in_.n;
    // Every instance starts from the first m_b values of the std::mt19937(1) normal sequence.
    std::vector<double> z0(m);
    int max_rows = 0;
    for (int b = 0; b < B_; ++b) max_rows = std::max(max_rows, in_.row_start[b + 1] - in_.row_start[b]);
    const auto seq = power_start_sequence(max_rows);
    for (int b = 0; b < B_; ++b)
      std::copy(seq->begin(), seq->begin() + (in_.row_start[b + 1] - in_.row_start[b]),
                z0.begin() + in_.row_start[b]);
    dbuf<double> dz(m), dq(m), datq(n);
    dq.upload(z0.data(), m, s_);
    permute_gather(dq.data(), L_.row_new2old.data(), m, 1.0, dz.data(), s_);
    dbuf<b_power_state> ps(B_);
    ps.zero(s_);
    dbuf<int> pact(B_), remaining(1);
    std::vector<int> pact_h(B_, 1);
    pact.upload(pact_h.data(), B_, s_);
    remaining.upload(&B_, 1, s_);
    const inst_ctx rctx{rinst_.data(), pact.data(), nullptr};
    const inst_ctx cctx{cinst_.data(), pact.data(), nullptr};
    const int nchunks = rows_.count;
    dbuf<double> part_z(std::max(nchunks, 1)), part_s2(std::max(nchunks, 1)),
      part_r(std::max(nchunks, 1));
    const int4* dchunks_p   = rows_.chunks.data();
    const int* dchunk_off_p = rows_.offsets.data();
    // q = z0 / |z0| once; every step then ends with the next step's q (z / |z|).
    b_chunk_sumsq_kernel<<<nchunks, kBlock, 0, s_>>>(dchunks_p, pact.data(), dz.data(),
                                                     part_z.data());
    b_chunk_normalize_kernel<<<nchunks, kBlock, 0, s_>>>(dchunks_p, dchunk_off_p, pact.data(),
                                                         part_z.data(), dz.data(), dq.data());
    launches_ += 2;
    B200_LAUNCH_CHECK();
    auto one_iteration = [&]() {
      const auto As  = wview<TX>(true, As_.data());
      const auto ATs = wview<TX>(false, ATs_.data());
      sell_map_kernel<TX, double, b_store_epi<double>><<<sell_grid(ATs), kBlock, 0, s_>>>(
        ATs, dq.data(), b_store_epi<double>{datq.data(), cctx}, partials_.data());
      sell_map_kernel<TX, double, b_power_z_epi><<<sell_grid(As), kBlock, 0, s_>>>(
        As, datq.data(), b_power_z_epi{dz.data(), dq.data(), rowbuf_.data(), rctx},
        partials_.data());
      b_chunk_sum_sumsq_kernel<<<nchunks, kBlock, 0, s_>>>(dchunks_p, pact.data(),
                                                           rowbuf_.data(), dz.data(),
                                                           part_s2.data(), part_z.data());
      b_chunk_residual_next_kernel<<<nchunks, kBlock, 0, s_>>>(
        dchunks_p, dchunk_off_p, pact.data(), part_s2.data(), part_z.data(), dz.data(),
        dq.data(), part_r.data());
      b_power_check_kernel<<<ceil_div(B_, kBlock), kBlock, 0, s_>>>(
        dchunk_off_p, B_, part_s2.data(), part_r.data(), pact.data(), ps.data(), kPowerTol,
        remaining.data());
    };
    // Chunks of 32 iterations are captured into a graph.  When the instances still iterating are
    // at most half of those the sweeps were last restricted to, the work lists shrink to them and
    // the chunk is captured again.
    cudaGraphExec_t exec = nullptr;
    auto capture = [&]() {
      if (exec) cudaGraphExecDestroy(exec);
      cudaGraph_t graph;
      B200_CUDA_CHECK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
      for (int i = 0; i < 32; ++i) one_iteration();
      B200_CUDA_CHECK(cudaStreamEndCapture(s_, &graph));
      B200_CUDA_CHECK(cudaGraphInstantiate(&exec, graph, 0));
      cudaGraphDestroy(graph);
    };
    capture();
    int left = B_, listed = B_;
    for (int done_iters = 0; done_iters < kPowerMaxIters; done_iters += 32) {
      if (kPowerMaxIters - done_iters < 32) {
        for (int i = 0; i < kPowerMaxIters - done_iters; ++i) one_iteration();
      } else {
        B200_CUDA_CHECK(cudaGraphLaunch(exec, s_));
      }
      launches_ += 5.0 * std::min(32, kPowerMaxIters - done_iters);
      remaining.download(&left, 1, s_);
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
      if (left == 0) break;
      if (2 * left <= listed) {
        pact.download(pact_h.data(), B_, s_);
        B200_CUDA_CHECK(cudaStreamSynchronize(s_));
        rebuild_work(pact_h);
        listed = left;
        capture();
        char what[96];
        std::snprintf(what, sizeof what, "batch: power to %d its, %d instances left",
                      done_iters + 32, left);
        trace(what);
      }
    }
    cudaGraphExecDestroy(exec);
    clear_work();
    std::vector<b_power_state> h(B_);
    ps.download(h.data(), B_, s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    eta_.resize(B_);
    power_iters_.resize(B_);
    for (int b = 0; b < B_; ++b) {
      eta_[b]         = kStepScaling / std::sqrt(h[b].s2);
      power_iters_[b] = h[b].iters;
    }
  }

  // Golub-Kahan-Lanczos on every instance (the single engine's lanczos_step_size, per instance):
  // chunks of kLanczosChunk steps; after each chunk an instance whose sigma_max^2 estimate moved by
  // at most kLanczosTol (relative), or whose recurrence broke down, stops, and the sweeps shrink
  // to the instances still iterating once they are at most half of those listed.
  void lanczos_step_size()
  {
    const int m = in_.m, n = in_.n;
    const int ld = kLanczosMaxSteps + 2;  // history rows (steps), each B_ wide
    // Every instance starts from the first m_b values of the std::mt19937(1) normal sequence.
    std::vector<double> z0(m);
    int max_rows = 0;
    for (int b = 0; b < B_; ++b) max_rows = std::max(max_rows, in_.row_start[b + 1] - in_.row_start[b]);
    const auto seq = power_start_sequence(max_rows);
    for (int b = 0; b < B_; ++b)
      std::copy(seq->begin(), seq->begin() + (in_.row_start[b + 1] - in_.row_start[b]),
                z0.begin() + in_.row_start[b]);
    dbuf<double> u(m), v(n), tmp(m), alphas((size_t)B_ * ld), betas((size_t)B_ * ld);
    dbuf<b_gk_state> st(B_);
    tmp.upload(z0.data(), m, s_);
    permute_gather(tmp.data(), L_.row_new2old.data(), m, 1.0, u.data(), s_);
    v.zero(s_);
    st.zero(s_);
    dbuf<int> pact(B_);
    std::vector<int> pact_h(B_, 1);
    pact.upload(pact_h.data(), B_, s_);
    const inst_ctx rctx{rinst_.data(), pact.data(), nullptr};
    const inst_ctx cctx{cinst_.data(), pact.data(), nullptr};
    dbuf<double> part_r(std::max(rows_.count, 1)), part_c(std::max(cols_.count, 1));
    // beta_0 = |z0| per instance (betas[b * ld + 0])
    b_chunk_sumsq_kernel<<<rows_.count, kBlock, 0, s_>>>(rows_.chunks.data(), pact.data(),
                                                        u.data(), part_r.data());
    b_gk_record_kernel<1><<<ceil_div(B_, kBlock), kBlock, 0, s_>>>(
      rows_.offsets.data(), B_, part_r.data(), pact.data(), st.data(), betas.data(), -1);
    launches_ += 2;
    B200_LAUNCH_CHECK();
    auto step = [&](int k) {
      const auto As  = wview<TX>(true, As_.data());
      const auto ATs = wview<TX>(false, ATs_.data());
      sell_map_kernel<TX, double, b_gk_primal_epi><<<sell_grid(ATs), kBlock, 0, s_>>>(
        ATs, u.data(), b_gk_primal_epi{v.data(), rowbuf_.data(), st.data(), cctx},
        partials_.data());
      b_chunk_sum_kernel<<<cols_.count, kBlock, 0, s_>>>(cols_.chunks.data(), pact.data(),
                                                         rowbuf_.data(), part_c.data());
      b_gk_record_kernel<0><<<ceil_div(B_, kBlock), kBlock, 0, s_>>>(
        cols_.offsets.data(), B_, part_c.data(), pact.data(), st.data(), alphas.data(), k);
      sell_map_kernel<TX, double, b_gk_dual_epi><<<sell_grid(As), kBlock, 0, s_>>>(
        As, v.data(), b_gk_dual_epi{u.data(), rowbuf_.data(), st.data(), rctx},
        partials_.data());
      b_chunk_sum_kernel<<<rows_.count, kBlock, 0, s_>>>(rows_.chunks.data(), pact.data(),
                                                         rowbuf_.data(), part_r.data());
      b_gk_record_kernel<1><<<ceil_div(B_, kBlock), kBlock, 0, s_>>>(
        rows_.offsets.data(), B_, part_r.data(), pact.data(), st.data(), betas.data(), k);
    };
    std::vector<double> ha((size_t)B_ * ld), hb((size_t)B_ * ld), prev(B_, -1.0), sigma2(B_, 0.0);
    std::vector<char> done(B_, 0);
    std::vector<int> used_steps(B_, 0);
    eta_.assign(B_, 0.0);
    power_iters_.assign(B_, 0);
    int left = B_, listed = B_, k = 0;
    while (left > 0 && k < kLanczosMaxSteps) {
      const int c = std::min(kLanczosChunk, kLanczosMaxSteps - k);
      for (int i = 0; i < c; ++i) step(k + i);
      launches_ += 6.0 * c;
      B200_LAUNCH_CHECK();
      k += c;
      alphas.download(ha.data(), (size_t)k * B_, s_);
      betas.download(hb.data(), (size_t)(k + 1) * B_, s_);
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
      // Each instance's estimate (a Sturm bisection per instance, the host's share of the step)
      // is independent of the others: instances are split over host threads, each writing only
      // its own entries, so the results do not depend on the split.
      parallel_ranges(B_, [&](int b0, int b1) {
        std::vector<double> a(ld), bb(ld);
        for (int b = b0; b < b1; ++b) {
          if (!pact_h[b]) continue;
          // betas[0] holds |z0|; the recurrence coefficients are betas[1..].
          for (int j = 0; j < k; ++j) a[j] = ha[(size_t)j * B_ + b];
          for (int j = 0; j <= k; ++j) bb[j] = hb[(size_t)j * B_ + b];
          bool breakdown = false;
          int used       = k;
          for (int j = 0; j < k; ++j)
            if (!(a[j] > 0.0) || !(bb[j + 1] > 0.0) || !std::isfinite(a[j]) ||
                !std::isfinite(bb[j + 1])) {
              used      = j + 1;
              breakdown = true;
              break;
            }
          sigma2[b]     = largest_bidiagonal_sigma2(a.data(), bb.data() + 1, used);
          done[b]       = breakdown || k >= kLanczosMaxSteps ||
                    (prev[b] > 0.0 && std::fabs(sigma2[b] - prev[b]) <= kLanczosTol * sigma2[b]);
          used_steps[b] = used;
          prev[b]       = sigma2[b];
        }
      });
      for (int b = 0; b < B_; ++b)
        if (pact_h[b] && done[b]) {
          pact_h[b]       = 0;
          power_iters_[b] = used_steps[b];
          --left;
        }
      if (left == 0) break;
      pact.upload(pact_h.data(), B_, s_);
      if (2 * left <= listed) {
        rebuild_work(pact_h);
        listed = left;
        char what[96];
        std::snprintf(what, sizeof what, "batch: lanczos to %d steps, %d instances left", k,
                      left);
        trace(what);
      }
    }
    clear_work();
    for (int b = 0; b < B_; ++b) {
      if (pact_h[b]) power_iters_[b] = k;  // step limit reached
      eta_[b] = kStepScaling / std::sqrt(sigma2[b]);
    }
  }

  // ---------------------------------------------------------------- work lists
  // Sweeps over A (rows = constraints) and A^T (rows = variables), restricted to the listed long
  // rows and slices once some instances have finished.
  template <typename T>
  dev_sell<T> wview(bool of_A, const T* vals) const
  {
    dev_sell<T> v = bview<T>(of_A ? L_.A : L_.AT, vals);
    if (lists_on_) {
      const work_list& w = of_A ? wa_ : wt_;
      v.long_list        = w.longs.data();
      v.slice_list       = w.slices.data();
      v.work_long        = w.n_long;
      v.work_slices      = w.n_slices;
    }
    return v;
  }

  struct work_list {
    dbuf<int> longs, slices;
    int n_long = 0, n_slices = 0;
  };

  void build_list(const std::vector<int4>& ranges, int n_long_rows, const std::vector<int>& act,
                  work_list& w)
  {
    std::vector<int> longs, slices;
    for (int b = 0; b < B_; ++b) {
      if (!act[b]) continue;
      const int4 r = ranges[b];
      for (int i = r.x; i < r.y; ++i) longs.push_back(i);
      if (r.z < r.w) {
        const int first = (r.z - n_long_rows) / kWarp, last = (r.w - 1 - n_long_rows) / kWarp;
        for (int q = first; q <= last; ++q)
          if (slices.empty() || slices.back() < q) slices.push_back(q);
      }
    }
    w.n_long   = (int)longs.size();
    w.n_slices = (int)slices.size();
    w.longs.resize(std::max<size_t>(longs.size(), 1));
    w.slices.resize(std::max<size_t>(slices.size(), 1));
    if (!longs.empty()) w.longs.upload(longs.data(), longs.size(), s_);
    if (!slices.empty()) w.slices.upload(slices.data(), slices.size(), s_);
  }

  // Restricts the sweeps to the instances flagged in `act`; cached graphs are dropped because
  // they hold the previous lists.
  void rebuild_work(const std::vector<int>& act)
  {
    build_list(rranges_, L_.A.n_long, act, wa_);
    build_list(cranges_, L_.AT.n_long, act, wt_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    lists_on_ = true;
    drop_graphs();
    init_plain_form((int)std::count(act.begin(), act.end(), 1), active_set_hash(act));
  }
  void clear_work()
  {
    lists_on_ = false;
    drop_graphs();
    init_plain_form(B_);
  }
  void drop_graphs()
  {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
  }

  // ---------------------------------------------------------------- iterations
  inst_ctx ctx_rows() const { return inst_ctx{rinst_.data(), active_d_.data(), sc_d_.data()}; }
  inst_ctx ctx_cols() const { return inst_ctx{cinst_.data(), active_d_.data(), sc_d_.data()}; }

  // The plain sweeps run with the tuned number of warps per block (tune_sweep_shape).
  template <bool MAJOR, bool HALPERN, bool SAVE_ATY>
  void launch_primal(int it_off, int wpb = 0)
  {
    const auto A = wview<TX>(false, ATs_.data());
    b_primal_epi<TX, MAJOR, HALPERN, SAVE_ATY> e{x_.data(),    cs_.data(),   ls_.data(),
                                                 us_.data(),   xa_.data(),   xbar_.data(),
                                                 x_.data(),    xhat_.data(), slack_.data(),
                                                 aty_.data(),  ctx_cols(),   it_off};
    if constexpr (!MAJOR && HALPERN && !SAVE_ATY)
      launch_sell_wpb(wpb ? wpb : wpb_primal_, A, y_.data(), e, partials_.data(), s_);
    else
      sell_map_kernel<TX, TX, decltype(e)><<<sell_grid(A), kBlock, 0, s_>>>(A, y_.data(), e,
                                                                           partials_.data());
    ++launches_;
  }
  template <bool MAJOR, bool HALPERN, bool FPE>
  void launch_dual(int it_off, int wpb = 0)
  {
    const auto A = wview<TX>(true, As_.data());
    b_dual_epi<TX, MAJOR, HALPERN, FPE> e{y_.data(),     lcs_.data(),  ucs_.data(),
                                          ya_.data(),    ybar_.data(), y_.data(),
                                          yhat_.data(),  rowbuf_.data(), ctx_rows(), it_off};
    if constexpr (!MAJOR && HALPERN && !FPE)
      launch_sell_wpb(wpb ? wpb : wpb_dual_, A, xbar_.data(), e, partials_.data(), s_);
    else
      sell_map_kernel<TX, TX, decltype(e)><<<sell_grid(A), kBlock, 0, s_>>>(A, xbar_.data(), e,
                                                                           partials_.data());
    ++launches_;
  }

  // Block shape of the plain sweeps over all instances (pdlp_sweep_warps_per_block = 0): 4, 8 and
  // 16 warps per block, a warm-up launch and about 1 ms of launches each; another shape replaces 8
  // warps when it is at least 3 % faster.  The iterates the timed sweeps move are restored (x, y) or
  // cleared (x_bar, y_bar) afterwards.
  void tune_sweep_shape()
  {
    wpb_primal_ = wpb_dual_ = p_.sweep_wpb ? p_.sweep_wpb : kWarpsPerBlock;
    if (p_.sweep_wpb) return;
    const batch_key key = tune_key(0, 0);
    {
      std::lock_guard<std::mutex> lock(batch_tune_mutex());
      auto it = batch_shape_cache().find(key);
      if (it != batch_shape_cache().end()) {
        wpb_primal_ = it->second.wpb_primal;
        wpb_dual_   = it->second.wpb_dual;
        std::memcpy(wpb_ms_, it->second.ms, sizeof(wpb_ms_));
        return;
      }
    }
    const int m = in_.m, n = in_.n;
    upload_scalars(std::vector<long>(B_, 0));
    dbuf<TX> x0(n), y0(m);
    B200_CUDA_CHECK(cudaMemcpyAsync(x0.data(), x_.data(), n * sizeof(TX),
                                    cudaMemcpyDeviceToDevice, s_));
    B200_CUDA_CHECK(cudaMemcpyAsync(y0.data(), y_.data(), m * sizeof(TX),
                                    cudaMemcpyDeviceToDevice, s_));
    cudaEvent_t e0, e1;
    B200_CUDA_CHECK(cudaEventCreate(&e0));
    B200_CUDA_CHECK(cudaEventCreate(&e1));
    // One warm-up launch, then enough launches for about a millisecond of timed work (at least 3).
    auto time_of = [&](auto&& launch) {
      B200_CUDA_CHECK(cudaEventRecord(e0, s_));
      launch();
      B200_CUDA_CHECK(cudaEventRecord(e1, s_));
      B200_CUDA_CHECK(cudaEventSynchronize(e1));
      float ms = 0.f;
      B200_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      const int reps = std::max(3, std::min(200, (int)std::ceil(1.0 / std::max(ms, 1e-3f))));
      B200_CUDA_CHECK(cudaEventRecord(e0, s_));
      for (int i = 0; i < reps; ++i) launch();
      B200_CUDA_CHECK(cudaEventRecord(e1, s_));
      B200_CUDA_CHECK(cudaEventSynchronize(e1));
      B200_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      return (double)ms / reps;
    };
    static constexpr int kShapes[3] = {4, 8, 16};
    for (int q = 0; q < 3; ++q) {
      wpb_ms_[0][q] = time_of([&] { launch_primal<false, true, false>(0, kShapes[q]); });
      wpb_ms_[1][q] = time_of([&] { launch_dual<false, true, false>(0, kShapes[q]); });
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // Another shape replaces the default 8 warps only when it is at least 3 % faster.
    auto best = [&](const double* t) {
      int b = 1;
      for (int q = 0; q < 3; ++q)
        if (t[q] > 0 && t[q] < 0.97 * t[1] && t[q] < t[b]) b = q;
      return kShapes[b];
    };
    wpb_primal_ = best(wpb_ms_[0]);
    wpb_dual_   = best(wpb_ms_[1]);
    {
      std::lock_guard<std::mutex> lock(batch_tune_mutex());
      batch_shape_choice c{wpb_primal_, wpb_dual_, {}};
      std::memcpy(c.ms, wpb_ms_, sizeof(wpb_ms_));
      batch_shape_cache()[key] = c;
    }
    B200_CUDA_CHECK(cudaMemcpyAsync(x_.data(), x0.data(), n * sizeof(TX),
                                    cudaMemcpyDeviceToDevice, s_));
    B200_CUDA_CHECK(cudaMemcpyAsync(y_.data(), y0.data(), m * sizeof(TX),
                                    cudaMemcpyDeviceToDevice, s_));
    xbar_.zero(s_);
    ybar_.zero(s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    if (std::getenv("CUOPT_B200_TRACE"))
      std::fprintf(stderr,
                   "[cuopt_b200] batch sweep block shape: primal %.4f/%.4f/%.4f ms -> %d warps; "
                   "dual %.4f/%.4f/%.4f ms -> %d warps (4/8/16 warps per block)\n",
                   wpb_ms_[0][0], wpb_ms_[0][1], wpb_ms_[0][2], wpb_primal_, wpb_ms_[1][0],
                   wpb_ms_[1][1], wpb_ms_[1][2], wpb_dual_);
  }
  void advance(int steps)
  {
    b_advance_kernel<<<ceil_div(B_, kBlock), kBlock, 0, s_>>>(sc_d_.data(), active_d_.data(), B_,
                                                             steps);
    ++launches_;
  }
  void plain_iterations(int L)
  {
    for (int i = 0; i < L; ++i) {
      launch_primal<false, true, false>(i);
      launch_dual<false, true, false>(i);
    }
    advance(L);
  }
  // ---------------------------------------------------------------- persistent plain iterations
  // The same choice as for single solves (plain_form.hpp), made again for every work list: the
  // sweeps shrink as instances finish, and the cost of kernel boundaries grows relative to them.
  using persist_pe = b_primal_epi<TX, false, true, false>;
  using persist_de = b_dual_epi<TX, false, true, false>;
  static const void* persistent_fn()
  {
    return (const void*)persistent_plain_kernel<TX, persist_pe, persist_de, advance_active>;
  }
  batch_key tune_key(int param, uint64_t set_hash) const
  {
    int dev = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    return batch_key{in_.m, in_.n, L_.nnz, B_, dev, (int)sizeof(TX), param, set_hash};
  }
  void init_plain_form(int n_active, uint64_t set_hash = 0)
  {
    int dev = 0, coop = 0, per_sm = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    B200_CUDA_CHECK(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_fn(), kBlock, 0));
    const int need = std::max(sell_grid(wview<TX>(false, ATs_.data())),
                              sell_grid(wview<TX>(true, As_.data())));
    persist_grid_  = std::min(need, per_sm * sms_);
    if (pctl_.size() == 0) {
      pctl_.resize(1);
      pctl_.zero(s_);
    }
    form_active_ = n_active;
    cycle_open_  = false;
    ++form_epochs_;
    const bool avail[plain_form_tuner::kForms] = {true, coop && persist_grid_ > 0, false};
    form_key_   = tune_key(p_.persistent, set_hash);
    int known   = -1;
    known_us_[0] = known_us_[1] = 0.0;
    if (p_.persistent < 0) {
      std::lock_guard<std::mutex> lock(batch_tune_mutex());
      auto it = batch_form_cache().find(form_key_);
      if (it != batch_form_cache().end()) {
        known        = it->second.form;
        known_us_[0] = it->second.us[0];
        known_us_[1] = it->second.us[1];
      }
    }
    form_.reset(p_.persistent, known, avail);
    if (n_active == B_ && form_.decided()) {  // forced, remembered, or the only form available
      first_form_   = form_.chosen();
      first_blocks_ = persist_grid_;
      first_us_[0]  = known_us_[0];
      first_us_[1]  = known_us_[1];
    }
  }
  void trace_form()
  {
    if (form_active_ == B_ && first_form_ < 0) {
      first_form_    = form_.chosen();
      first_us_[0]   = form_.us_per_iteration(0);
      first_us_[1]   = form_.us_per_iteration(1);
      first_blocks_  = persist_grid_;
    }
    if (std::getenv("CUOPT_B200_TRACE"))
      std::fprintf(stderr,
                   "[cuopt_b200] batch plain iterations (%d instances): graphs %.2f us, "
                   "persistent (%d blocks) %.2f us per iteration -> %s\n",
                   form_active_, form_.us_per_iteration(0), persist_grid_,
                   form_.us_per_iteration(1), form_.chosen() ? "persistent" : "graphs");
  }
  void collect_form_timing()
  {
    const bool before = form_.decided();
    form_.collect();
    if (!before && form_.decided()) {
      trace_form();
      std::lock_guard<std::mutex> lock(batch_tune_mutex());
      batch_form_cache()[form_key_] =
        batch_form_choice{form_.chosen(), {form_.us_per_iteration(0), form_.us_per_iteration(1)}};
    }
  }
  // Returns true for the first launch of the engine (which may include loading the kernel).
  bool launch_persistent(int L)
  {
    const auto AT = wview<TX>(false, ATs_.data()), A = wview<TX>(true, As_.data());
    persist_pe pe{x_.data(),   cs_.data(),   ls_.data(),    us_.data(),  xa_.data(),
                  xbar_.data(), x_.data(),   xhat_.data(),  slack_.data(), aty_.data(),
                  ctx_cols(),  0};
    persist_de de{y_.data(),    lcs_.data(),  ucs_.data(),    ya_.data(), ybar_.data(),
                  y_.data(),    yhat_.data(), rowbuf_.data(), ctx_rows(), 0};
    advance_active adv{sc_d_.data(), active_d_.data(), B_};
    int gp = sell_grid(AT), gd = sell_grid(A);
    const TX* y    = y_.data();
    const TX* xb   = xbar_.data();
    persist_ctl* c = pctl_.data();
    unsigned long long budget = kPersistBudgetNs;
    B200_CUDA_CHECK(cudaMemsetAsync(&c->arrivals, 0, sizeof(unsigned), s_));
    void* args[] = {(void*)&AT, (void*)&A, (void*)&y, (void*)&xb, (void*)&pe, (void*)&de,
                    (void*)&adv, (void*)&L, (void*)&gp, (void*)&gd, (void*)&c, (void*)&budget};
    B200_CUDA_CHECK(cudaLaunchCooperativeKernel(persistent_fn(), dim3(persist_grid_),
                                                dim3(kBlock), args, 0, s_));
    ++launches_;
    persist_used_ = true;
    return persist_launches_++ == 0;
  }

  // A timing cycle runs from the first plain run after a termination check to the next check:
  // all its plain runs use one form, and its events bracket everything the GPU does in between
  // (major steps, fixed-point errors and every launch boundary), so the forms are compared on
  // what they cost the loop.
  void run_plain(long R, long k)
  {
    if (!cycle_open_) {
      cycle_form_     = form_.next();
      cycle_k0_       = k;
      cycle_one_time_ = false;
      cycle_open_     = true;
      form_.begin(s_);
    }
    cycle_one_time_ |= cycle_form_ == 1 ? launch_persistent((int)R) : run_graphs(R);
  }
  void close_cycle(long k)
  {
    if (!cycle_open_) return;
    cycle_open_ = false;
    form_.end(s_, cycle_form_, k - cycle_k0_, cycle_one_time_);
  }

  // Returns true when a graph had to be captured and instantiated first.
  bool run_graphs(long R)
  {
    bool built = false;
    for (int L = 128; L >= 1; L >>= 1) {
      while (R >= L) {
        auto it = graphs_.find(L);
        if (it == graphs_.end()) {
          cudaGraph_t g;
          cudaGraphExec_t e;
          B200_CUDA_CHECK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
          const double before = launches_;
          plain_iterations(L);
          launches_ = before;
          B200_CUDA_CHECK(cudaStreamEndCapture(s_, &g));
          B200_CUDA_CHECK(cudaGraphInstantiate(&e, g, 0));
          cudaGraphDestroy(g);
          it = graphs_.emplace(L, e).first;
          built = true;
        }
        B200_CUDA_CHECK(cudaGraphLaunch(it->second, s_));
        launches_ += 2.0 * L + 1.0;
        R -= L;
      }
    }
    return built;
  }

  void upload_scalars(const std::vector<long>& since)
  {
    std::vector<pdlp_scalars> h(B_);
    for (int b = 0; b < B_; ++b)
      h[b] = pdlp_scalars{eta_[b] / omega_[b], eta_[b] * omega_[b], eta_[b], omega_[b],
                          (long long)since[b]};
    sc_d_.upload(h.data(), B_, s_);
    active_d_.upload(active_h_.data(), B_, s_);
  }

  // Unscaled residuals / objectives of every active instance (x_hat, y_hat, slack of the last
  // major step), like the single-LP evaluation.
  std::vector<inst_conv> evaluate()
  {
    const int m = in_.m, n = in_.n;
    b_unscale_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(
      xhat_.data(), yhat_.data(), slack_.data(), dc_.data(), dr_.data(), beta_d_.data(),
      gamma_d_.data(), cinst_.data(), rinst_.data(), active_d_.data(), n, m, xu_.data(), yu_.data(),
      su_.data());
    const auto A = wview<double>(true, L_.A.val.data()), AT = wview<double>(false, L_.AT.val.data());
    sell_map_kernel<double, double, b_term_primal_epi><<<sell_grid(A), kBlock, 0, s_>>>(
      A, xu_.data(),
      b_term_primal_epi{lc64_.data(), uc64_.data(), yu_.data(), rowbuf_.data(), stride_,
                        ctx_rows()},
      partials_.data());
    seg_reduce<2>(true, 0, true);
    sell_map_kernel<double, double, b_term_dual_epi><<<sell_grid(AT), kBlock, 0, s_>>>(
      AT, yu_.data(),
      b_term_dual_epi{c64_.data(), xu_.data(), su_.data(), rowbuf_.data(), stride_, ctx_cols()},
      partials_.data());
    seg_reduce<3>(false, 2 * (size_t)B_, true);
    launches_ += 3;
    B200_LAUNCH_CHECK();
    fetch(0, 5 * (size_t)B_, hbuf_);
    std::vector<inst_conv> cv(B_);
    for (int b = 0; b < B_; ++b) {
      if (!active_h_[b]) continue;
      const double* pr = hbuf_ + 2 * b;
      const double* du = hbuf_ + 2 * B_ + 3 * b;
      inst_conv& c     = cv[b];
      c.l2_primal      = std::sqrt(pr[0]);
      c.l2_dual        = std::sqrt(du[0]);
      c.primal_obj     = du[1];
      c.dual_obj       = du[2] + pr[1];
      if (obj_scale_[b] != 1.0 || obj_offset_[b] != 0.0) {
        c.primal_obj = obj_scale_[b] * (c.primal_obj + obj_offset_[b]);
        c.dual_obj   = obj_scale_[b] * (c.dual_obj + obj_offset_[b]);
      }
      c.gap     = std::fabs(c.primal_obj - c.dual_obj);
      c.abs_obj = std::fabs(c.primal_obj) + std::fabs(c.dual_obj);
    }
    return cv;
  }

  void finish(int b, int status, const inst_conv& c, long k)
  {
    pdlp_result& r   = results_[b];
    r.status         = status;
    r.iterations     = k;
    r.primal_obj     = c.primal_obj;
    r.dual_obj       = c.dual_obj;
    r.l2_primal      = c.l2_primal;
    r.l2_dual        = c.l2_dual;
    r.rel_primal     = c.l2_primal / (1.0 + b_norm_[b]);
    r.rel_dual       = c.l2_dual / (1.0 + c_norm_[b]);
    r.gap            = c.gap;
    r.rel_gap        = c.gap / (1.0 + c.abs_obj);
    r.step_size      = eta_[b];
    r.primal_weight  = omega_[b];
    r.restarts       = restarts_[b];
    r.solve_time     = now_s() - t_start_;
    active_h_[b]     = 0;
  }

  // Same schedule and per-instance decisions as engine::loop of the single-LP solver.
  void loop()
  {
    const int m = in_.m, n = in_.n;
    const double qnan = std::numeric_limits<double>::quiet_NaN();
    const double inf  = std::numeric_limits<double>::infinity();
    std::vector<double> fpe(B_, qnan), fpe0(B_, qnan), last_trial(B_, inf);
    std::vector<double> pid_sum(B_, 0.0), pid_last(B_, 0.0), best_gap(B_, inf);
    std::vector<long> since(B_, 0);
    std::vector<int> restarted(B_, 0);
    // Stall test of mixed precision (per instance; see kStallWindow).
    std::vector<double> stall_ref(B_, std::numeric_limits<double>::infinity());
    std::vector<long> stall_k(B_, 0);
    int n_active = B_, listed = B_;
    upload_scalars(since);

    for (long k = 0;;) {
      const bool major = (k % kMajor == 0 && k > 0) || k <= 0;
      const bool cond  = (k % conditional_major(k)) == 0;
      std::fill(restarted.begin(), restarted.end(), 0);
      bool any_restart = false;
      if (major || cond) {
        close_cycle(k);
        const std::vector<inst_conv> cv = evaluate();
        const bool out_of_time = now_s() - t_start_ >= p_.time_limit;
        for (int b = 0; b < B_; ++b) {
          if (!active_h_[b]) continue;
          const inst_conv& c   = cv[b];
          const bool primal_ok = c.l2_primal <= p_.abs_primal + p_.rel_primal * b_norm_[b];
          const bool optimal   = c.l2_dual <= p_.abs_dual + p_.rel_dual * c_norm_[b] &&
                               primal_ok && c.gap <= p_.abs_gap + p_.rel_gap * c.abs_obj;
          if (k > 1 && optimal)
            finish(b, kOptimal, c, k);
          else if (out_of_time)
            finish(b, kTimeLimit, c, k);
          else if (k >= p_.iteration_limit)
            finish(b, kIterationLimit, c, k);
          else if (!std::isfinite(c.l2_primal) || !std::isfinite(c.l2_dual))
            finish(b, kNumericalError, c, k);
          else if (std::is_same_v<TX, float>) {
            const double q = termination_distance(
              c.l2_primal, p_.abs_primal + p_.rel_primal * b_norm_[b], c.l2_dual,
              p_.abs_dual + p_.rel_dual * c_norm_[b], c.gap, p_.abs_gap + p_.rel_gap * c.abs_obj);
            if (q <= 0.5 * stall_ref[b]) {
              stall_ref[b] = q;
              stall_k[b]   = k;
            } else if (k - stall_k[b] >= kStallWindow)
              finish(b, kStalled, c, k);
          }
        }
        n_active = (int)std::count(active_h_.begin(), active_h_.end(), 1);
        if (n_active == 0) break;
        if (2 * n_active <= listed) {
          rebuild_work(active_h_);
          listed = n_active;
          char what[96];
          std::snprintf(what, sizeof what, "batch: loop to %ld its, %d instances left", k,
                        n_active);
          trace(what);
        }

        if (major) {
          // Restart distances of every active instance.
          sq_diff_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(xa_.data(), xhat_.data(), n,
                                                        rowbuf_.data());
          active_d_.upload(active_h_.data(), B_, s_);
          seg_reduce<1>(false, 0, true);
          sq_diff_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(ya_.data(), yhat_.data(), m,
                                                        rowbuf_.data());
          seg_reduce<1>(true, B_, true);
          launches_ += 2;
          fetch(0, 2 * (size_t)B_, hbuf_);
          for (int b = 0; b < B_; ++b) {
            if (!active_h_[b]) continue;
            // should_cupdlpx_restart (reference pdlp_restart_strategy.cu:689-754)
            bool restart = false;
            if (k == kMajor)
              restart = true;
            else if (k > kMajor) {
              if (fpe[b] <= kSufficientReduction * fpe0[b])
                restart = true;
              else if (fpe[b] <= kNecessaryReduction * fpe0[b] && fpe[b] > last_trial[b])
                restart = true;
              else if ((double)since[b] >= kArtificialRestart * (double)k)
                restart = true;
            }
            last_trial[b] = fpe[b];
            if (!restart) continue;
            // cupdlpx_restart + PID primal weight (reference pdlp_restart_strategy.cu:758-986)
            const inst_conv& c      = cv[b];
            const double rel_dual   = c.l2_dual / (1.0 + c_norm_[b]);
            const double rel_primal = c.l2_primal / (1.0 + b_norm_[b]);
            const double lp = std::sqrt(hbuf_[b]), ld = std::sqrt(hbuf_[B_ + b]);
            const double ratio = rel_primal == 0.0 ? inf : rel_dual / rel_primal;
            if (lp > 1e-16 && ld > 1e-16 && lp < 1e12 && ld < 1e12 && ratio > 1e-8 &&
                ratio < 1e8) {
              const double err  = std::log(ld) - std::log(lp) - std::log(omega_[b]);
              pid_sum[b]        = pid_sum[b] * kISmooth + err;
              const double derr = err - pid_last[b];
              omega_[b]   = std::exp(kKp * err + kKi * pid_sum[b] + kKd * derr) * omega_[b];
              pid_last[b] = err;
            } else {
              omega_[b]    = best_omega_[b];
              pid_sum[b]   = 0.0;
              pid_last[b]  = 0.0;
            }
            const double rgap = std::fabs(std::log10(ratio));
            if (rgap < best_gap[b]) {
              best_gap[b]    = rgap;
              best_omega_[b] = omega_[b];
            }
            since[b]      = 0;
            last_trial[b] = inf;
            restarted[b]  = 1;
            any_restart   = true;
            ++restarts_[b];
          }
          if (any_restart) {
            restart_flags_.resize(B_);
            restart_flags_.upload(restarted.data(), B_, s_);
            b_restart_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(
              x_.data(), xa_.data(), xhat_.data(), n, y_.data(), ya_.data(), yhat_.data(), m,
              cinst_.data(), rinst_.data(), restart_flags_.data());
            ++launches_;
          }
        }
        upload_scalars(since);
        B200_LAUNCH_CHECK();
      }

      const bool mstep   = is_major_step(k);
      const bool fpe_all = ((k + 1) % kMajor == 0);
      if (!mstep && !fpe_all && !any_restart) {
        long R = 1;
        while (R < 255) {
          const long kk = k + R;
          if (is_check(kk) || is_major_step(kk) || ((kk + 1) % kMajor == 0)) break;
          ++R;
        }
        run_plain(R, k);
        k += R;
        for (int b = 0; b < B_; ++b)
          if (active_h_[b]) since[b] += R;
        continue;
      }

      if (fpe_all || any_restart) {
        // Every active instance takes the fixed-point-error form of the step (the same update
        // with the Halpern step applied separately); only instances that need the error use it.
        if (mstep) {
          launch_primal<true, false, true>(0);
          launch_dual<true, false, true>(0);
        } else {
          launch_primal<false, false, true>(0);
          launch_dual<false, false, true>(0);
        }
        seg_reduce<1>(true, 0, true);
        const auto AT = wview<TX>(false, ATs_.data());
        sell_map_kernel<TX, TX, b_fpe_epi<TX>><<<sell_grid(AT), kBlock, 0, s_>>>(
          AT, ybar_.data(),
          b_fpe_epi<TX>{aty_.data(), xbar_.data(), x_.data(), rowbuf_.data(), stride_, ctx_cols()},
          partials_.data());
        seg_reduce<2>(false, B_, true);
        b_halpern_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(x_.data(), xbar_.data(), xa_.data(), n,
                                                        y_.data(), ybar_.data(), ya_.data(), m,
                                                        cinst_.data(), rinst_.data(),
                                                        active_d_.data(), sc_d_.data());
        advance(1);
        launches_ += 2;
        B200_LAUNCH_CHECK();
        fetch(0, 3 * (size_t)B_, hbuf_);
        for (int b = 0; b < B_; ++b) {
          if (!active_h_[b] || !(fpe_all || restarted[b])) continue;
          const double ndy = hbuf_[b], inter = hbuf_[B_ + 2 * b], ndx = hbuf_[B_ + 2 * b + 1];
          const double movement = ndx * omega_[b] + ndy / omega_[b];
          fpe[b]                = std::sqrt(movement + 2.0 * inter * eta_[b]);
          if (restarted[b]) fpe0[b] = fpe[b];
        }
      } else {
        launch_primal<true, true, false>(0);
        launch_dual<true, true, false>(0);
        advance(1);
        B200_LAUNCH_CHECK();
      }
      ++k;
      for (int b = 0; b < B_; ++b)
        if (active_h_[b]) ++since[b];
    }
  }

  void write_outputs(double* x_out, double* y_out, double* rc_out)
  {
    const int m = in_.m, n = in_.n;
    if (x_out)
      scatter_by_inst_kernel<<<vgrid_, kBlock, 0, s_>>>(xu_.data(), L_.col_new2old.data(),
                                                        cinst_.data(), nullptr, n, x_out);
    if (rc_out)
      scatter_by_inst_kernel<<<vgrid_, kBlock, 0, s_>>>(su_.data(), L_.col_new2old.data(),
                                                        cinst_.data(), sgn_d_.data(), n, rc_out);
    if (y_out)
      scatter_by_inst_kernel<<<vgrid_, kBlock, 0, s_>>>(yu_.data(), L_.row_new2old.data(),
                                                        rinst_.data(), sgn_d_.data(), m, y_out);
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  // ---------------------------------------------------------------- state
  const batch_device_input& in_;
  const pdlp_params& p_;
  cudaStream_t s_;
  int B_;
  int sms_ = 148, vgrid_ = 592;
  double* hbuf_ = nullptr;
  double t_start_ = 0, t_loop_ = 0;
  double launches_ = 0;
  size_t stride_ = 0;

  device_layout L_;
  dbuf<TX> As_, ATs_;
  dbuf<int> rinst_, cinst_, active_d_, restart_flags_;
  dbuf<int4> rr_d_, cr_d_;
  std::vector<int4> rranges_, cranges_;
  dbuf<double> c64_, l64_, u64_, lc64_, uc64_, dr_, dc_, sgn_d_, beta_d_, gamma_d_;
  dbuf<TX> cs_, ls_, us_, lcs_, ucs_;
  dbuf<TX> x_, xhat_, slack_, xbar_, xa_, aty_, y_, yhat_, ybar_, ya_;
  dbuf<double> xu_, yu_, su_, rowbuf_, segout_, partials_;
  dbuf<pdlp_scalars> sc_d_;

  std::vector<double> obj_scale_, obj_offset_, c_norm_, b_norm_, beta_, gamma_, eta_, omega_,
    best_omega_;
  std::vector<int> restarts_, power_iters_, active_h_;
  std::vector<pdlp_result> results_;
  std::map<int, cudaGraphExec_t> graphs_;
  work_list wa_, wt_;
  bool lists_on_ = false;
  chunk_table rows_, cols_;
  dbuf<double> chunk_part_;
  // Persistent plain iterations: control block, grid, the choice of form for the current work
  // list, and the choice made while every instance ran (reported in the results).
  dbuf<persist_ctl> pctl_;
  int* hstatus_      = nullptr;
  bool cycle_open_ = false, cycle_one_time_ = false;
  int cycle_form_  = 0;
  long cycle_k0_   = 0;
  int persist_grid_  = 0;
  bool persist_used_ = false;
  long persist_launches_ = 0;
  plain_form_tuner form_;
  int form_active_ = 0, form_epochs_ = 0;
  int first_form_ = -1, first_blocks_ = 0;
  double first_us_[2] = {0, 0};
  batch_key form_key_{};           // the current work list's form decision in batch_form_cache
  double known_us_[2] = {0, 0};    // its timings, when it was remembered from an earlier solve
  // Warps per block of the plain sweeps and the timings they were chosen by.
  int wpb_primal_ = kWarpsPerBlock, wpb_dual_ = kWarpsPerBlock;
  double wpb_ms_[2][3] = {{0, 0, 0}, {0, 0, 0}};
};


}  // namespace

std::vector<pdlp_result> pdlp_batch_solve_device(const batch_device_input& in,
                                                 const pdlp_params& p, cudaStream_t stream,
                                                 double* x_out, double* y_out, double* rc_out)
{
  if (in.count <= 0 || in.count > 65535)
    throw std::invalid_argument("batch size must be in [1, 65535]");
  configure_pool_once();
  joined_stream js(stream);
  if (p.precision == 1) {
    batch_engine<float> e(in, p, js.own);
    return e.run(x_out, y_out, rc_out);
  }
  batch_engine<double> e(in, p, js.own);
  return e.run(x_out, y_out, rc_out);
}

}  // namespace cuopt_b200
