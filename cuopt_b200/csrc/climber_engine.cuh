// Same-matrix batch ("climbers"): B copies of one LP that differ only in the bounds of one variable
// each — the strong-branching batch of the reference (batch_pdlp_solve, cpp/src/pdlp/solve.cu:
// 884-919, run_batch_pdlp :740-882; climbers and new_bounds in pdlp.cu:1447-1746).
//
// Included by pdlp_engine.cu after engine<TX>: a climber_engine takes the layout, the scaling and
// the step size of an engine<double> that was set up on the base LP (variable bounds change none of
// them) and iterates all climbers together.  Vectors are stored climber-interleaved (element j of
// climber b at j * ld + b), so a sweep reads the matrix once for a group of kGroup climbers and
// each gather fetches kGroup contiguous values of one column: whole sectors instead of one 8-byte
// value per sector request.  Every climber keeps its own Stable3 state (restarts, primal weight,
// termination) and follows the iterates of a single solve of its LP.

constexpr int kGroup = 8;  // climbers per sweep launch

// A climber's override of one variable's bounds (internal column, scaled bounds).
struct climber_bound {
  int col;
  double l, u;
};

__device__ __forceinline__ void gather_group(const double* __restrict__ p, double (&v)[kGroup])
{
  const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int h = 0; h < kGroup / 2; ++h) {
    const double2 t = q[h];
    v[2 * h]        = t.x;
    v[2 * h + 1]    = t.y;
  }
}

// acc[b] = sum_k A[r,k] g[idx[r,k] * ld + g0 + b] for the kGroup climbers of a group, then
// epi(r, acc, pre, red).  One launch covers the n_groups groups listed in `groups`: block
// q * n_groups + i sweeps matrix block q for group groups[i] (its g0 replaces the epilogue's), so
// the blocks that read one stretch of the matrix run side by side and share it through L2.  The
// block sums of group g go to partials + g * pstride.
template <class Epi>
__global__ void __launch_bounds__(kBlock) mm_sweep_kernel(const dev_sell<double> A,
                                                          const double* __restrict__ g, int ld,
                                                          const int* __restrict__ groups,
                                                          int n_groups, Epi epi, double* partials,
                                                          size_t pstride)
{
  constexpr int K = Epi::kRed;
  const int grp = groups[blockIdx.x % n_groups];
  const int xb  = (int)(blockIdx.x / n_groups);
  const int g0  = grp * kGroup;
  epi.ctx.g0    = g0;
  red_t<K> red;
#pragma unroll
  for (int q = 0; q < (K > 0 ? K : 1); ++q) red.v[q] = 0.0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int lb   = long_blocks(A.n_long);
  double acc[kGroup];
#pragma unroll
  for (int b = 0; b < kGroup; ++b) acc[b] = 0.0;
  if (xb < lb) {
    const int row = xb * kWarpsPerBlock + warp;
    if (row < A.n_long) {
      const auto pre = epi.load(row);
      for (int64_t k = A.long_off[row] + lane; k < A.long_off[row + 1]; k += kWarp) {
        const double v = ld_stream(A.val + k);
        double gv[kGroup];
        gather_group(g + (size_t)ld_stream(A.idx + k) * ld + g0, gv);
#pragma unroll
        for (int b = 0; b < kGroup; ++b) acc[b] += v * gv[b];
      }
#pragma unroll
      for (int b = 0; b < kGroup; ++b) acc[b] = warp_sum(acc[b]);
      if (lane == 0) epi(row, acc, pre, red);
    }
  } else {
    const int s = (xb - lb) * kWarpsPerBlock + warp;
    if (s < A.n_slices) {
      const int row      = A.n_long + s * kWarp + lane;
      const bool valid   = row < A.rows;
      const auto pre     = epi.load(valid ? row : A.rows - 1);
      const int64_t base = A.slice_off[s];
      const int nchunk   = (int)((A.slice_off[s + 1] - base) >> 7);
      const double* v    = A.val + base + lane * kChunk;
      const int* ix      = A.idx + base + lane * kChunk;
      for (int q = 0; q < nchunk; ++q) {
        const int4 i4 = load_idx_chunk(ix);
        double v4[4];
        load_chunk(v, v4);
        const int id[4] = {i4.x, i4.y, i4.z, i4.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          double gv[kGroup];
          gather_group(g + (size_t)id[e] * ld + g0, gv);
#pragma unroll
          for (int b = 0; b < kGroup; ++b) acc[b] += v4[e] * gv[b];
        }
        v += kWarp * kChunk;
        ix += kWarp * kChunk;
      }
      if (valid) epi(row, acc, pre, red);
    }
  }
  block_reduce_store<K>(red, partials + (size_t)grp * pstride, xb);
}

// out[g * stride + q] = the ordered sum of group g's block sums, one block per listed group.
template <int K>
__global__ void __launch_bounds__(kBlock) mm_finalize_kernel(const double* partials, size_t pstride,
                                                             int nblocks, const int* groups,
                                                             double* out, int stride)
{
  const int grp = groups[blockIdx.x];
  ordered_block_sum<K>(partials + (size_t)grp * pstride, nblocks, out + (size_t)grp * stride);
}

// Per-climber state shared by the climber epilogues.
struct mm_ctx {
  int ld, g0;
  const pdlp_scalars* sc;
  const int* active;
  __device__ __forceinline__ size_t at(int row, int b) const { return (size_t)row * ld + g0 + b; }
};

struct mm_x {  // primal values of one climber for primal_row_step
  double x, c, lo, up, xa;
};
struct mm_y {  // dual values of one climber for dual_row_step
  double y, lo, up, ya;
};

template <bool MAJOR, bool HALPERN, bool SAVE_ATY>
struct mm_primal_epi {
  static constexpr int kRed = 0;
  const double *x, *xa, *c, *lo, *up;
  double *xbar, *xout, *xhat, *slack, *aty;
  const climber_bound* ovr;
  mm_ctx ctx;
  int it_off;
  struct pre_t {
    double c, lo, up, x[kGroup], xa[kGroup];
  };
  __device__ __forceinline__ pre_t load(int j) const
  {
    pre_t p;
    p.c  = c[j];
    p.lo = lo[j];
    p.up = up[j];
    gather_group(x + ctx.at(j, 0), p.x);
    if (HALPERN) gather_group(xa + ctx.at(j, 0), p.xa);
    return p;
  }
  __device__ __forceinline__ void operator()(int j, const double (&acc)[kGroup], const pre_t& p,
                                             red_t<0>&) const
  {
#pragma unroll
    for (int b = 0; b < kGroup; ++b) {
      const int gb = ctx.g0 + b;
      if (!ctx.active[gb]) continue;
      const climber_bound o = ovr[gb];
      const mm_x v{p.x[b], p.c, o.col == j ? o.l : p.lo, o.col == j ? o.u : p.up,
                   HALPERN ? p.xa[b] : 0.0};
      const size_t e = ctx.at(j, b);
      primal_row_step<double, MAJOR, HALPERN, SAVE_ATY>(0, acc[b], v, ctx.sc + gb, it_off,
                                                        xbar + e, xout + e, xhat + e, slack + e,
                                                        aty + e);
    }
  }
};

// FPE: red[b] += (y_bar - y)^2 of climber b.
template <bool MAJOR, bool HALPERN, bool FPE>
struct mm_dual_epi {
  static constexpr int kRed = FPE ? kGroup : 0;
  const double *y, *ya, *lo, *up;
  double *ybar, *yout, *yhat;
  mm_ctx ctx;
  int it_off;
  struct pre_t {
    double lo, up, y[kGroup], ya[kGroup];
  };
  __device__ __forceinline__ pre_t load(int i) const
  {
    pre_t p;
    p.lo = lo[i];
    p.up = up[i];
    gather_group(y + ctx.at(i, 0), p.y);
    if (HALPERN) gather_group(ya + ctx.at(i, 0), p.ya);
    return p;
  }
  __device__ __forceinline__ void operator()(int i, const double (&acc)[kGroup], const pre_t& p,
                                             red_t<kRed>& r) const
  {
#pragma unroll
    for (int b = 0; b < kGroup; ++b) {
      const int gb = ctx.g0 + b;
      if (!ctx.active[gb]) continue;
      const mm_y v{p.y[b], p.lo, p.up, HALPERN ? p.ya[b] : 0.0};
      const size_t e = ctx.at(i, b);
      const double d2 =
        dual_row_step<double, MAJOR, HALPERN>(0, acc[b], v, ctx.sc + gb, it_off, ybar + e,
                                              yout + e, yhat + e);
      if constexpr (FPE) r.v[b] += d2;
    }
  }
};

// red[b] += (A^T y_bar - A^T y)_j (x_bar - x)_j ; red[kGroup + b] += (x_bar - x)_j^2.
struct mm_fpe_epi {
  static constexpr int kRed = 2 * kGroup;
  const double *aty, *xbar, *x;
  mm_ctx ctx;
  struct pre_t {
    double aty[kGroup], xbar[kGroup], x[kGroup];
  };
  __device__ __forceinline__ pre_t load(int j) const
  {
    pre_t p;
    gather_group(aty + ctx.at(j, 0), p.aty);
    gather_group(xbar + ctx.at(j, 0), p.xbar);
    gather_group(x + ctx.at(j, 0), p.x);
    return p;
  }
  __device__ __forceinline__ void operator()(int, const double (&acc)[kGroup], const pre_t& p,
                                             red_t<kRed>& r) const
  {
#pragma unroll
    for (int b = 0; b < kGroup; ++b) {
      const double d  = acc[b] - p.aty[b];
      const double dx = p.xbar[b] - p.x[b];
      r.v[b] += d * dx;
      r.v[kGroup + b] += dx * dx;
    }
  }
};

// Unscaled termination terms (FP64 matrix): row i of A -> rp^2, dual bound term.
struct mm_term_primal_epi {
  static constexpr int kRed = 2 * kGroup;
  const double *lc, *uc, *y;
  mm_ctx ctx;
  struct pre_t {
    double l, u, y[kGroup];
  };
  __device__ __forceinline__ pre_t load(int i) const
  {
    pre_t p;
    p.l = lc[i];
    p.u = uc[i];
    gather_group(y + ctx.at(i, 0), p.y);
    return p;
  }
  __device__ __forceinline__ void operator()(int, const double (&ax)[kGroup], const pre_t& p,
                                             red_t<kRed>& r) const
  {
#pragma unroll
    for (int b = 0; b < kGroup; ++b) {
      const double rp = ax[b] - fmax(p.l, fmin(ax[b], p.u));
      r.v[b] += rp * rp;
      r.v[kGroup + b] += fmax(p.y[b], 0.0) * finite_or_zero(p.l) + fmin(p.y[b], 0.0) * finite_or_zero(p.u);
    }
  }
};

// Row j of A^T -> rd^2, c.x, s.x.
struct mm_term_dual_epi {
  static constexpr int kRed = 3 * kGroup;
  const double *c, *x, *s;
  mm_ctx ctx;
  struct pre_t {
    double c, x[kGroup], s[kGroup];
  };
  __device__ __forceinline__ pre_t load(int j) const
  {
    pre_t p;
    p.c = c[j];
    gather_group(x + ctx.at(j, 0), p.x);
    gather_group(s + ctx.at(j, 0), p.s);
    return p;
  }
  __device__ __forceinline__ void operator()(int, const double (&aty)[kGroup], const pre_t& p,
                                             red_t<kRed>& r) const
  {
#pragma unroll
    for (int b = 0; b < kGroup; ++b) {
      const double rd = (p.c - aty[b]) - p.s[b];
      r.v[b] += rd * rd;
      r.v[kGroup + b] += p.c * p.x[b];
      r.v[2 * kGroup + b] += p.s[b] * p.x[b];
    }
  }
};

// Element-wise kernels over climber-interleaved vectors (element e = row * ld + climber).
__global__ void mm_halpern_kernel(double* x, const double* xbar, const double* xa, size_t nx,
                                  double* y, const double* ybar, const double* ya, size_t ny,
                                  int ld, const int* active, const pdlp_scalars* sc)
{
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nx + ny;
       e += (size_t)gridDim.x * blockDim.x) {
    const bool is_x = e < nx;
    const size_t k  = is_x ? e : e - nx;
    const int b     = (int)(k % ld);
    if (!active[b]) continue;
    const double w = halpern_weight(sc + b, 0);
    if (is_x)
      x[k] = w * xbar[k] + (1.0 - w) * xa[k];
    else
      y[k] = w * ybar[k] + (1.0 - w) * ya[k];
  }
}

__global__ void mm_unscale_kernel(const double* xhat, const double* yhat, const double* slack,
                                  const double* dc, const double* dr, double inv_beta,
                                  double inv_gamma, int n, int m, int ld, const int* active,
                                  double* xu, double* yu, double* su)
{
  const size_t nx = (size_t)n * ld, ny = (size_t)m * ld;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nx + ny;
       e += (size_t)gridDim.x * blockDim.x) {
    if (e < nx) {
      const int b = (int)(e % ld), j = (int)(e / ld);
      if (!active[b]) continue;
      const double d = dc[j];
      xu[e]          = (xhat[e] * d) * inv_beta;
      su[e]          = (d != 0.0 ? slack[e] / d : slack[e]) * inv_gamma;
    } else {
      const size_t k = e - nx;
      const int b = (int)(k % ld), i = (int)(k / ld);
      if (!active[b]) continue;
      yu[k] = (yhat[k] * dr[i]) * inv_gamma;
    }
  }
}

__global__ void mm_restart_kernel(double* x, double* xa, const double* xhat, size_t nx, double* y,
                                  double* ya, const double* yhat, size_t ny, int ld,
                                  const int* flag)
{
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < nx + ny;
       e += (size_t)gridDim.x * blockDim.x) {
    const bool is_x = e < nx;
    const size_t k  = is_x ? e : e - nx;
    if (!flag[k % ld]) continue;
    if (is_x) {
      x[k]  = xhat[k];
      xa[k] = xhat[k];
    } else {
      y[k]  = yhat[k];
      ya[k] = yhat[k];
    }
  }
}

__global__ void mm_advance_kernel(pdlp_scalars* sc, const int* active, int count, int steps)
{
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x)
    if (active[b]) sc[b].t0 += steps;
}

// Per-block partial sums of (a - b)^2 over `rows` rows for the kGroup climbers of every listed
// group (blocks laid out as in mm_sweep_kernel).
__global__ void __launch_bounds__(kBlock) mm_sqdiff_kernel(const double* a, const double* b,
                                                           int rows, int ld, const int* groups,
                                                           int n_groups, double* partials,
                                                           size_t pstride)
{
  const int grp = groups[blockIdx.x % n_groups];
  const int xb = (int)(blockIdx.x / n_groups), nxb = (int)(gridDim.x / n_groups);
  const int g0 = grp * kGroup;
  red_t<kGroup> r;
#pragma unroll
  for (int q = 0; q < kGroup; ++q) r.v[q] = 0.0;
  for (int i = xb * kBlock + threadIdx.x; i < rows; i += nxb * kBlock) {
    double va[kGroup], vb[kGroup];
    gather_group(a + (size_t)i * ld + g0, va);
    gather_group(b + (size_t)i * ld + g0, vb);
#pragma unroll
    for (int q = 0; q < kGroup; ++q) r.v[q] += (va[q] - vb[q]) * (va[q] - vb[q]);
  }
  block_reduce_store<kGroup>(r, partials + (size_t)grp * pstride, xb);
}

// x = clamp(x, l, u) with the climbers' overrides (project_initial_primal).
__global__ void mm_initial_primal_kernel(double* x, const double* l, const double* u, int n, int ld,
                                         const climber_bound* ovr)
{
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)n * ld;
       e += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(e % ld), j = (int)(e / ld);
    const climber_bound o = ovr[b];
    const double lo = o.col == j ? o.l : l[j], hi = o.col == j ? o.u : u[j];
    x[e]            = fmin(fmax(x[e], lo), hi);
  }
}

// a = b = c = src broadcast to every climber (element e = row * ld + climber).
__global__ void mm_broadcast_kernel(const double* src, int rows, int ld, double* a, double* b,
                                    double* c)
{
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < (size_t)rows * ld;
       e += (size_t)gridDim.x * blockDim.x) {
    const double v = src[e / ld];
    a[e]           = v;
    b[e]           = v;
    c[e]           = v;
  }
}

class climber_engine {
 public:
  // base: an engine<double> whose setup ran on the LP; var / lo / up: per climber the user-order
  // variable and its new (unscaled) bounds.
  climber_engine(engine<double>& base, const pdlp_params& p, const std::vector<int>& var,
                 const std::vector<double>& lo, const std::vector<double>& up)
    : e_(base), p_(p), s_(base.s_), B_((int)var.size())
  {
    ld_     = std::max(kGroup, (B_ + kGroup - 1) / kGroup * kGroup);
    groups_ = ld_ / kGroup;
    B200_CUDA_CHECK(cudaMallocHost(&hbuf_, sizeof(double) * 6 * (size_t)ld_ + 64));
    var_ = var;
    lo_  = lo;
    up_  = up;
  }
  ~climber_engine()
  {
    drop_graphs();
    cudaFreeHost(hbuf_);
  }

  std::vector<pdlp_result> run(double* x_out, double* y_out, double* rc_out)
  {
    alloc_scope scope(s_);
    t_start_ = e_.t_start_;
    results_.assign(B_, pdlp_result{});
    setup();
    t_loop_ = now_s();
    loop();
    write_outputs(x_out, y_out, rc_out);
    for (int b = 0; b < B_; ++b) {
      results_[b].setup_time       = t_loop_ - t_start_;
      results_[b].loop_time        = results_[b].solve_time - (t_loop_ - t_start_);
      results_[b].power_iterations = e_.power_iters_;
      results_[b].kernel_launches  = launches_ + e_.launches_;
    }
    return results_;
  }

 private:
  void setup()
  {
    const int m = e_.in_.m, n = e_.in_.n;
    const size_t nx = (size_t)n * ld_, ny = (size_t)m * ld_;
    // Overrides in the internal numbering and the scaled space (scale_vectors_kernel +
    // rescale_vectors_kernel of the base engine).
    std::vector<int> old2new(n);
    e_.L_.col_old2new.download(old2new.data(), n, s_);
    std::vector<double> dcol(n);
    e_.dc_.download(dcol.data(), n, s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    std::vector<climber_bound> ov(ld_, climber_bound{-1, 0.0, 0.0});
    for (int b = 0; b < B_; ++b) {
      if (var_[b] < 0 || var_[b] >= n)
        throw std::invalid_argument("climber variable index out of range");
      const int j    = old2new[var_[b]];
      const double d = dcol[j];
      ov[b]          = climber_bound{j, d == 0.0 ? 0.0 : lo_[b] / d * e_.beta_,
                            d == 0.0 ? 0.0 : up_[b] / d * e_.beta_};
      if (!(up_[b] >= lo_[b])) crossing_.push_back(b);
    }
    ovr_.resize(ld_);
    ovr_.upload(ov.data(), ld_, s_);
    active_h_.assign(ld_, 0);
    for (int b = 0; b < B_; ++b) active_h_[b] = 1;
    for (int b : crossing_) active_h_[b] = 0;  // crossing bounds: Infeasible without iterating
    active_d_.resize(ld_);
    active_d_.upload(active_h_.data(), ld_, s_);
    groups_d_.resize(groups_);
    refresh_groups();
    for (auto* v : {&x_, &xhat_, &slack_, &xbar_, &xa_, &aty_, &xu_, &su_}) {
      v->resize(nx);
      v->zero(s_);
    }
    for (auto* v : {&y_, &yhat_, &ybar_, &ya_, &yu_}) {
      v->resize(ny);
      v->zero(s_);
    }
    // A warm start (the caller's initial solution, scaled by the base engine into x_hat and y_hat
    // of the base) starts every climber at the same point, as the reference's batch does with
    // its initial solution; the primal is then projected onto each climber's bounds.
    if (e_.in_.initial_primal) {
      mm_broadcast_kernel<<<e_.vgrid_, kBlock, 0, s_>>>(e_.xhat_.data(), n, ld_, x_.data(),
                                                        xhat_.data(), xa_.data());
      ++launches_;
    }
    if (e_.in_.initial_dual) {
      mm_broadcast_kernel<<<e_.vgrid_, kBlock, 0, s_>>>(e_.yhat_.data(), m, ld_, y_.data(),
                                                        yhat_.data(), ya_.data());
      ++launches_;
    }
    mm_initial_primal_kernel<<<e_.vgrid_, kBlock, 0, s_>>>(x_.data(), e_.ls_.data(),
                                                           e_.us_.data(), n, ld_, ovr_.data());
    ++launches_;
    sc_d_.resize(ld_);
    omega_.assign(ld_, e_.omega_);
    best_omega_.assign(ld_, e_.best_omega_);
    restarts_.assign(ld_, 0);
    const int g =
      std::max({sell_grid(view64(e_.L_.A)), sell_grid(view64(e_.L_.AT)), e_.vgrid_});
    pstride_ = (size_t)g * 3 * kGroup;
    partials_.resize(pstride_ * groups_);
    dres_.resize((size_t)6 * ld_);
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  bool group_active(int g) const
  {
    for (int b = g * kGroup; b < (g + 1) * kGroup; ++b)
      if (active_h_[b]) return true;
    return false;
  }
  // The list of groups with an active climber, on the device for the sweeps (captured graphs see
  // it by address: they are dropped whenever it changes).
  void refresh_groups()
  {
    groups_h_.clear();
    for (int g = 0; g < groups_; ++g)
      if (group_active(g)) groups_h_.push_back(g);
    if (!groups_h_.empty()) groups_d_.upload(groups_h_.data(), groups_h_.size(), s_);
  }
  int n_act() const { return (int)groups_h_.size(); }
  // g0 is set per block by the kernels.
  mm_ctx ctx() const { return mm_ctx{ld_, 0, sc_d_.data(), active_d_.data()}; }
  template <class Epi>
  void sweep(const dev_sell<double>& A, const double* g, const Epi& ep)
  {
    if (n_act() == 0) return;
    mm_sweep_kernel<<<sell_grid(A) * n_act(), kBlock, 0, s_>>>(
      A, g, ld_, groups_d_.data(), n_act(), ep, partials_.data(), pstride_);
    ++launches_;
  }

  template <bool MAJOR, bool HALPERN, bool SAVE_ATY>
  void launch_primal(int it_off)
  {
    const auto A = view_of<double>(e_.L_.AT, e_.ATs_.data());
    sweep(A, y_.data(),
          mm_primal_epi<MAJOR, HALPERN, SAVE_ATY>{
            x_.data(), xa_.data(), e_.cs_.data(), e_.ls_.data(), e_.us_.data(), xbar_.data(),
            x_.data(), xhat_.data(), slack_.data(), aty_.data(), ovr_.data(), ctx(), it_off});
  }
  template <bool MAJOR, bool HALPERN, bool FPE>
  void launch_dual(int it_off)
  {
    const auto A = view_of<double>(e_.L_.A, e_.As_.data());
    sweep(A, xbar_.data(),
          mm_dual_epi<MAJOR, HALPERN, FPE>{y_.data(), ya_.data(), e_.lcs_.data(), e_.ucs_.data(),
                                           ybar_.data(), y_.data(), yhat_.data(), ctx(), it_off});
  }
  void advance(int steps)
  {
    mm_advance_kernel<<<ceil_div(ld_, kBlock), kBlock, 0, s_>>>(sc_d_.data(), active_d_.data(),
                                                               ld_, steps);
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
  void run_plain(long R)
  {
    for (int L = 128; L >= 1; L >>= 1) {
      while (R >= L) {
        auto it = graphs_.find(L);
        if (it == graphs_.end()) {
          cudaGraph_t gr;
          cudaGraphExec_t ex;
          B200_CUDA_CHECK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
          const double before = launches_;
          plain_iterations(L);
          launches_ = before;
          B200_CUDA_CHECK(cudaStreamEndCapture(s_, &gr));
          B200_CUDA_CHECK(cudaGraphInstantiate(&ex, gr, 0));
          cudaGraphDestroy(gr);
          it = graphs_.emplace(L, ex).first;
        }
        B200_CUDA_CHECK(cudaGraphLaunch(it->second, s_));
        launches_ += 2.0 * L + 1.0;
        R -= L;
      }
    }
  }
  void drop_graphs()
  {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
    graphs_.clear();
  }

  void upload_state(const std::vector<long>& since)
  {
    std::vector<pdlp_scalars> h(ld_);
    const double eta = e_.eta_;
    for (int b = 0; b < ld_; ++b)
      h[b] = pdlp_scalars{eta / omega_[b], eta * omega_[b], eta, omega_[b], (long long)since[b]};
    sc_d_.upload(h.data(), ld_, s_);
    active_d_.upload(active_h_.data(), ld_, s_);
  }

  // Sums the K values per block of every listed group g from the partials into
  // dres_ + off + g * stride.
  template <int K>
  void finalize(int nblocks, size_t off, int stride)
  {
    if (n_act() == 0) return;
    mm_finalize_kernel<K><<<n_act(), kBlock, 0, s_>>>(partials_.data(), pstride_, nblocks,
                                                      groups_d_.data(), dres_.data() + off, stride);
    ++launches_;
  }
  // Sums of (a - b)^2 per climber over `rows` rows into dres_ + off + climber.
  void sqdiff(const double* a, const double* b, int rows, size_t off)
  {
    if (n_act() == 0) return;
    mm_sqdiff_kernel<<<e_.vgrid_ * n_act(), kBlock, 0, s_>>>(a, b, rows, ld_, groups_d_.data(),
                                                            n_act(), partials_.data(), pstride_);
    ++launches_;
    finalize<kGroup>(e_.vgrid_, off, kGroup);
  }
  void fetch(size_t count)
  {
    B200_CUDA_CHECK(
      cudaMemcpyAsync(hbuf_, dres_.data(), count * sizeof(double), cudaMemcpyDeviceToHost, s_));
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  // Residuals and objectives of every active climber (unscaled x_hat, y_hat, slack).
  std::vector<conv_info> evaluate()
  {
    const int m = e_.in_.m, n = e_.in_.n;
    mm_unscale_kernel<<<e_.vgrid_, kBlock, 0, s_>>>(
      xhat_.data(), yhat_.data(), slack_.data(), e_.dc_.data(), e_.dr_.data(), 1.0 / e_.beta_,
      1.0 / e_.gamma_, n, m, ld_, active_d_.data(), xu_.data(), yu_.data(), su_.data());
    ++launches_;
    const auto A = view64(e_.L_.A), AT = view64(e_.L_.AT);
    std::vector<conv_info> cv(ld_);
    sweep(A, xu_.data(), mm_term_primal_epi{e_.lc64_.data(), e_.uc64_.data(), yu_.data(), ctx()});
    finalize<2 * kGroup>(sell_grid(A), 0, 5 * kGroup);
    sweep(AT, yu_.data(), mm_term_dual_epi{e_.c64_.data(), xu_.data(), su_.data(), ctx()});
    finalize<3 * kGroup>(sell_grid(AT), 2 * kGroup, 5 * kGroup);
    B200_LAUNCH_CHECK();
    fetch(5 * (size_t)ld_);
    for (int g : groups_h_) {
      const double* h = hbuf_ + (size_t)g * 5 * kGroup;
      for (int q = 0; q < kGroup; ++q) {
        const int b = g * kGroup + q;
        if (!active_h_[b]) continue;
        conv_info& c = cv[b];
        c.l2_primal  = std::sqrt(h[q]);
        c.l2_dual    = std::sqrt(h[2 * kGroup + q]);
        c.primal_obj = h[3 * kGroup + q];
        c.dual_obj   = h[4 * kGroup + q] + h[kGroup + q];
        if (e_.obj_scale_ != 1.0 || e_.obj_offset_ != 0.0) {
          c.primal_obj = e_.obj_scale_ * (c.primal_obj + e_.obj_offset_);
          c.dual_obj   = e_.obj_scale_ * (c.dual_obj + e_.obj_offset_);
        }
        c.gap     = std::fabs(c.primal_obj - c.dual_obj);
        c.abs_obj = std::fabs(c.primal_obj) + std::fabs(c.dual_obj);
      }
    }
    return cv;
  }

  void finish(int b, int status, const conv_info& c, long k)
  {
    pdlp_result& r  = results_[b];
    r.status        = status;
    r.iterations    = k;
    r.primal_obj    = c.primal_obj;
    r.dual_obj      = c.dual_obj;
    r.l2_primal     = c.l2_primal;
    r.l2_dual       = c.l2_dual;
    r.rel_primal    = c.l2_primal / (1.0 + e_.b_norm_);
    r.rel_dual      = c.l2_dual / (1.0 + e_.c_norm_);
    r.gap           = c.gap;
    r.rel_gap       = c.gap / (1.0 + c.abs_obj);
    r.step_size     = e_.eta_;
    r.primal_weight = omega_[b];
    r.restarts      = restarts_[b];
    r.solve_time    = now_s() - t_start_;
    active_h_[b]    = 0;
  }

  // The schedule and per-climber decisions of engine::loop.
  void loop()
  {
    const int m = e_.in_.m, n = e_.in_.n;
    const size_t nx = (size_t)n * ld_, ny = (size_t)m * ld_;
    const double qnan = std::numeric_limits<double>::quiet_NaN();
    const double inf  = std::numeric_limits<double>::infinity();
    const double eta  = e_.eta_;
    std::vector<double> fpe(ld_, qnan), fpe0(ld_, qnan), last_trial(ld_, inf);
    std::vector<double> pid_sum(ld_, 0.0), pid_last(ld_, 0.0), best_gap(ld_, inf);
    std::vector<long> since(ld_, 0);
    std::vector<int> restarted(ld_, 0);
    for (int b : crossing_) {
      results_[b].status     = kPrimalInfeasible;
      results_[b].solve_time = now_s() - t_start_;
    }
    upload_state(since);
    std::vector<int> groups_seen(groups_);
    for (int g = 0; g < groups_; ++g) groups_seen[g] = group_active(g);

    for (long k = 0;;) {
      const bool major = (k % kMajor == 0 && k > 0) || k <= 0;
      const bool cond  = (k % conditional_major(k)) == 0;
      std::fill(restarted.begin(), restarted.end(), 0);
      bool any_restart = false;
      if (major || cond) {
        const std::vector<conv_info> cv = evaluate();
        const bool out_of_time = now_s() - t_start_ >= p_.time_limit;
        for (int b = 0; b < B_; ++b) {
          if (!active_h_[b]) continue;
          const conv_info& c   = cv[b];
          const bool primal_ok = c.l2_primal <= p_.abs_primal + p_.rel_primal * e_.b_norm_;
          const bool optimal   = c.l2_dual <= p_.abs_dual + p_.rel_dual * e_.c_norm_ &&
                               primal_ok && c.gap <= p_.abs_gap + p_.rel_gap * c.abs_obj;
          if (k > 1 && optimal)
            finish(b, kOptimal, c, k);
          else if (out_of_time)
            finish(b, kTimeLimit, c, k);
          else if (k >= p_.iteration_limit)
            finish(b, kIterationLimit, c, k);
          else if (!std::isfinite(c.l2_primal) || !std::isfinite(c.l2_dual))
            finish(b, kNumericalError, c, k);
        }
        if (std::count(active_h_.begin(), active_h_.end(), 1) == 0) break;
        bool groups_changed = false;
        for (int g = 0; g < groups_; ++g)
          if (groups_seen[g] && !group_active(g)) {
            groups_seen[g] = 0;
            groups_changed = true;
          }
        if (groups_changed) {
          drop_graphs();
          refresh_groups();
        }
        active_d_.upload(active_h_.data(), ld_, s_);

        if (major) {
          sqdiff(xa_.data(), xhat_.data(), n, 0);
          sqdiff(ya_.data(), yhat_.data(), m, (size_t)ld_);
          B200_LAUNCH_CHECK();
          fetch(2 * (size_t)ld_);
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
            const conv_info& c      = cv[b];
            const double rel_dual   = c.l2_dual / (1.0 + e_.c_norm_);
            const double rel_primal = c.l2_primal / (1.0 + e_.b_norm_);
            const double lp = std::sqrt(hbuf_[b]), ld = std::sqrt(hbuf_[ld_ + b]);
            const double ratio = rel_primal == 0.0 ? inf : rel_dual / rel_primal;
            if (lp > 1e-16 && ld > 1e-16 && lp < 1e12 && ld < 1e12 && ratio > 1e-8 &&
                ratio < 1e8) {
              const double err  = std::log(ld) - std::log(lp) - std::log(omega_[b]);
              pid_sum[b]        = pid_sum[b] * kISmooth + err;
              const double derr = err - pid_last[b];
              omega_[b]   = std::exp(kKp * err + kKi * pid_sum[b] + kKd * derr) * omega_[b];
              pid_last[b] = err;
            } else {
              omega_[b]   = best_omega_[b];
              pid_sum[b]  = 0.0;
              pid_last[b] = 0.0;
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
            flags_.resize(ld_);
            flags_.upload(restarted.data(), ld_, s_);
            mm_restart_kernel<<<e_.vgrid_, kBlock, 0, s_>>>(x_.data(), xa_.data(), xhat_.data(),
                                                            nx, y_.data(), ya_.data(),
                                                            yhat_.data(), ny, ld_, flags_.data());
            ++launches_;
          }
        }
        upload_state(since);
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
        run_plain(R);
        k += R;
        for (int b = 0; b < B_; ++b)
          if (active_h_[b]) since[b] += R;
        continue;
      }

      if (fpe_all || any_restart) {
        const auto A = view_of<double>(e_.L_.A, e_.As_.data());
        const auto AT = view_of<double>(e_.L_.AT, e_.ATs_.data());
        if (mstep) {
          launch_primal<true, false, true>(0);
          launch_dual<true, false, true>(0);
        } else {
          launch_primal<false, false, true>(0);
          launch_dual<false, false, true>(0);
        }
        finalize<kGroup>(sell_grid(A), 0, kGroup);
        sweep(AT, ybar_.data(), mm_fpe_epi{aty_.data(), xbar_.data(), x_.data(), ctx()});
        finalize<2 * kGroup>(sell_grid(AT), (size_t)ld_, 2 * kGroup);
        mm_halpern_kernel<<<e_.vgrid_, kBlock, 0, s_>>>(x_.data(), xbar_.data(), xa_.data(), nx,
                                                        y_.data(), ybar_.data(), ya_.data(), ny,
                                                        ld_, active_d_.data(), sc_d_.data());
        ++launches_;
        advance(1);
        B200_LAUNCH_CHECK();
        fetch(3 * (size_t)ld_);
        for (int b = 0; b < B_; ++b) {
          if (!active_h_[b] || !(fpe_all || restarted[b])) continue;
          const int g = b / kGroup, q = b % kGroup;
          const double ndy   = hbuf_[b];
          const double inter = hbuf_[ld_ + 2 * g * kGroup + q];
          const double ndx   = hbuf_[ld_ + 2 * g * kGroup + kGroup + q];
          const double movement = ndx * omega_[b] + ndy / omega_[b];
          fpe[b]                = std::sqrt(movement + 2.0 * inter * eta);
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

  // Climber-interleaved unscaled solutions to the user's order, climber-major (B x n, B x m).
  void write_outputs(double* x_out, double* y_out, double* rc_out)
  {
    const int m = e_.in_.m, n = e_.in_.n;
    const double sgn = e_.in_.maximize ? -1.0 : 1.0;
    std::vector<int> c2o(n), r2o(m);
    e_.L_.col_new2old.download(c2o.data(), n, s_);
    e_.L_.row_new2old.download(r2o.data(), m, s_);
    std::vector<double> hx((size_t)n * ld_), hs((size_t)n * ld_), hy((size_t)m * ld_);
    xu_.download(hx.data(), hx.size(), s_);
    su_.download(hs.data(), hs.size(), s_);
    yu_.download(hy.data(), hy.size(), s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    for (int b = 0; b < B_; ++b) {
      for (int j = 0; j < n; ++j) {
        if (x_out) x_out[(size_t)b * n + c2o[j]] = hx[(size_t)j * ld_ + b];
        if (rc_out) rc_out[(size_t)b * n + c2o[j]] = sgn * hs[(size_t)j * ld_ + b];
      }
      if (y_out)
        for (int i = 0; i < m; ++i) y_out[(size_t)b * m + r2o[i]] = sgn * hy[(size_t)i * ld_ + b];
    }
  }

  engine<double>& e_;
  const pdlp_params& p_;
  cudaStream_t s_;
  int B_, ld_ = kGroup, groups_ = 1;
  double* hbuf_ = nullptr;
  double t_start_ = 0, t_loop_ = 0, launches_ = 0;
  std::vector<int> var_, crossing_;
  std::vector<double> lo_, up_;
  std::vector<int> active_h_, restarts_;
  std::vector<double> omega_, best_omega_;
  std::vector<pdlp_result> results_;
  dbuf<climber_bound> ovr_;
  dbuf<int> active_d_, flags_, groups_d_;
  std::vector<int> groups_h_;
  size_t pstride_ = 0;
  dbuf<pdlp_scalars> sc_d_;
  dbuf<double> x_, xhat_, slack_, xbar_, xa_, aty_, y_, yhat_, ybar_, ya_, xu_, yu_, su_;
  dbuf<double> partials_, dres_;
  std::map<int, cudaGraphExec_t> graphs_;
};
