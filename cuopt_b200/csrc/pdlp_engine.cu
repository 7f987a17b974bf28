// PDLP (Stable3: restarted reflected Halpern PDHG with cuPDLPx restarts) on sm_100a.
//
// Host driver counterpart of the reference's pdlp_solver_t::run_solver
// (cpp/src/pdlp/pdlp.cu:2013-2457).  The host keeps the scalar state that the reference keeps on
// the host (restart decision, PID primal weight, fixed-point errors); all vector and matrix work
// is in the kernels of kernels.cuh.  Iterations that need neither a termination test, a "major"
// step nor a fixed-point error are replayed from cached CUDA graphs of 2^k iterations, or run by one
// persistent cooperative launch, whichever form timed faster on the solve's first runs.
#include "device_layout.cuh"
#include "host_io.hpp"
#include "kernels.cuh"
#include "pdlp_engine.hpp"
#include "pdlp_schedule.hpp"
#include "plain_form.hpp"
#include "tile_sweep.cuh"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <tuple>

namespace cuopt_b200 {

namespace {

double now_s()
{
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
dev_sell<T> view_of(const dev_matrix& M, const T* v)
{
  return dev_sell<T>{M.rows, M.n_long, M.n_slices, M.long_off.data(), M.slice_off.data(),
                     M.idx.data(), v};
}
inline dev_sell<double> view64(const dev_matrix& M) { return view_of<double>(M, M.val.data()); }

struct conv_info {
  double l2_primal, l2_dual, primal_obj, dual_obj, gap, abs_obj;
  double linf_primal = 0, linf_dual = 0;  // per-constraint forms, when asked for
};

// Iteration count and restart / PID state of the main loop (host side).
struct loop_state {
  long k = 0, since = 0;
  double fpe        = std::numeric_limits<double>::quiet_NaN();
  double fpe0       = std::numeric_limits<double>::quiet_NaN();
  double last_trial = std::numeric_limits<double>::infinity();
  double pid_sum = 0.0, pid_last = 0.0;
  double best_gap = std::numeric_limits<double>::infinity();
  bool fresh      = true;  // no iteration run yet: the loop starts by zeroing the step counter
  // Infeasibility test statistics (zero until first computed, then kept between computations).
  double primal_ray_obj = 0.0, max_primal_ray_inf = 0.0;
  double dual_ray_obj = 0.0, max_dual_ray_inf = 0.0;
  // Stall test of mixed precision: reference distance and the iteration it was reached.
  double stall_ref = std::numeric_limits<double>::infinity();
  long stall_k     = 0;
};

class climber_engine;

// Autotuning decisions of the mixed-precision sweeps, per problem shape (m, n, nnz) and device,
// for the life of the process: (tiled primal sweep, tiled dual sweep).
using tune_key = std::tuple<int, int, int64_t, int>;
std::map<tune_key, std::pair<bool, bool>>& tune_cache()
{
  static std::map<tune_key, std::pair<bool, bool>> c;
  return c;
}
std::mutex& tune_mutex()
{
  static std::mutex mu;
  return mu;
}
// Form of the plain iterations (0 CUDA graphs, 1 persistent kernel) chosen by timing, per problem
// shape (m, n, nnz), device and iterate precision (bytes), for the life of the process.
// The timings it was chosen by are kept with it (microseconds per plain iteration).
using form_key = std::tuple<int, int, int64_t, int, int>;
struct form_choice {
  int form;
  double us[3];  // graphs, persistent kernel, cluster
};
std::map<form_key, form_choice>& form_cache()
{
  static std::map<form_key, form_choice> c;
  return c;
}
// Warps per block of the plain sweeps chosen by timing, with the timings (ms per launch with 4, 8
// and 16 warps per block; primal sweep, then dual sweep), per shape, device and precision.
struct shape_choice {
  int wpb_primal, wpb_dual;
  double ms[2][3];
};
std::map<form_key, shape_choice>& shape_cache()
{
  static std::map<form_key, shape_choice> c;
  return c;
}

template <typename TX>
class engine {
  template <typename>
  friend class engine;
  friend class climber_engine;

 public:
  engine(const lp_device_input& in, const pdlp_params& p, cudaStream_t s)
    : in_(in), p_(p), s_(s)
  {
    int dev = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
    configure_pool_once();
    hres_ = pinned_scratch();
  }
  ~engine()
  {
    for (auto& kv : graphs_) cudaGraphExecDestroy(kv.second);
  }

  // Setup only (layout, scaling, step size): the base of a climber batch.
  void prepare()
  {
    alloc_scope scope(s_);
    t_start_ = now_s();
    setup();
  }

  pdlp_result run(double* x_out, double* y_out, double* rc_out)
  {
    alloc_scope scope(s_);
    x_out_   = x_out;
    y_out_   = y_out;
    rc_out_  = rc_out;
    t_start_ = now_s();
    pdlp_result r;
    setup();
    r.power_iterations = power_iters_;
    if (!(std::isfinite(eta_) && eta_ > 0)) {
      r.status    = kNumericalError;
      r.step_size = eta_;
      finish_times(r);
      return r;
    }
    t_loop_ = now_s();
    loop(r);
    write_outputs();
    finish_times(r);
    return r;
  }

  // FP64 continuation of a mixed-precision solve (used on engine<double>): takes over the layout,
  // the scaling, the step size, the primal weight, the iterates, the Halpern anchor and the
  // schedule / restart state of `mixed`, and resumes its iteration in FP64 at the check where it
  // stopped, until the tolerances of this engine's parameters hold on the original LP.  Iteration
  // counts, restarts and times continue those of the first solve.
  template <typename TM>
  pdlp_result continue_from(engine<TM>& mixed, double* x_out, double* y_out, double* rc_out)
  {
    alloc_scope scope(s_);
    x_out_  = x_out;
    y_out_  = y_out;
    rc_out_ = rc_out;
    adopt(mixed);
    pdlp_result r;
    loop(r);
    r.power_iterations  = power_iters_;
    r.refinement_passes = 1;
    write_outputs();
    finish_times(r);
    return r;
  }

 private:
  // ------------------------------------------------------------------ setup
  void setup()
  {
    const int m = in_.m, n = in_.n;
    trace("engine: start");
    build_device_layout(m, n, in_.row_off, in_.col_idx, in_.val, s_, L_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    trace("engine: layout");
    vgrid_ = sms_ * 4;
    const int g = std::max({sell_grid(view64(L_.A)), sell_grid(view64(L_.AT)), vgrid_});
    partials_.resize((size_t)g * 4);
    dres_.resize(64);

    // Unscaled vectors in internal order; objective negated for maximisation
    // (reference problem_helpers.cuh:132-151).
    const double sgn = in_.maximize ? -1.0 : 1.0;
    obj_scale_       = in_.maximize ? -1.0 : 1.0;
    obj_offset_      = in_.maximize ? -in_.obj_offset : in_.obj_offset;
    c64_.resize(n);
    l64_.resize(n);
    u64_.resize(n);
    lc64_.resize(m);
    uc64_.resize(m);
    permute_gather(in_.c, L_.col_new2old.data(), n, sgn, c64_.data(), s_);
    permute_gather(in_.var_lo, L_.col_new2old.data(), n, 1.0, l64_.data(), s_);
    permute_gather(in_.var_up, L_.col_new2old.data(), n, 1.0, u64_.data(), s_);
    permute_gather(in_.con_lo, L_.row_new2old.data(), m, 1.0, lc64_.data(), s_);
    permute_gather(in_.con_up, L_.row_new2old.data(), m, 1.0, uc64_.data(), s_);

    // Ruiz (10 passes) then Pock-Chambolle (alpha = 1) (reference initial_scaling.cu:152-365).
    dr_.resize(m);
    dc_.resize(n);
    fill(dr_.data(), m, 1.0);
    fill(dc_.data(), n, 1.0);
    dbuf<double> rtmp(m), ctmp(n);
    for (int it = 0; it < kRuizIterations; ++it) {
      row_scaled_abs_kernel<0, false><<<sell_grid(view64(L_.A)), kBlock, 0, s_>>>(
        view64(L_.A), dr_.data(), dc_.data(), 0.0, rtmp.data());
      row_scaled_abs_kernel<0, true><<<sell_grid(view64(L_.AT)), kBlock, 0, s_>>>(
        view64(L_.AT), dr_.data(), dc_.data(), 0.0, ctmp.data());
      apply_root_scaling_kernel<<<vgrid_, kBlock, 0, s_>>>(dr_.data(), rtmp.data(), m);
      apply_root_scaling_kernel<<<vgrid_, kBlock, 0, s_>>>(dc_.data(), ctmp.data(), n);
    }
    row_scaled_abs_kernel<1, false><<<sell_grid(view64(L_.A)), kBlock, 0, s_>>>(
      view64(L_.A), dr_.data(), dc_.data(), kPcAlpha, rtmp.data());
    row_scaled_abs_kernel<1, true><<<sell_grid(view64(L_.AT)), kBlock, 0, s_>>>(
      view64(L_.AT), dr_.data(), dc_.data(), 2.0 - kPcAlpha, ctmp.data());
    apply_root_scaling_kernel<<<vgrid_, kBlock, 0, s_>>>(dr_.data(), rtmp.data(), m);
    apply_root_scaling_kernel<<<vgrid_, kBlock, 0, s_>>>(dc_.data(), ctmp.data(), n);
    B200_LAUNCH_CHECK();

    // Scaled matrix values in the iterate precision.
    As_.resize(L_.A.stored());
    ATs_.resize(L_.AT.stored());
    scale_values_kernel<TX, false><<<sell_grid(view64(L_.A)), kBlock, 0, s_>>>(
      view64(L_.A), dr_.data(), dc_.data(), As_.data());
    scale_values_kernel<TX, true><<<sell_grid(view64(L_.AT)), kBlock, 0, s_>>>(
      view64(L_.AT), dr_.data(), dc_.data(), ATs_.data());

    prepare_vectors();
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    trace("engine: scaling");
    // Step size from the largest singular value of the scaled A (reference pdlp.cu:2620-2731),
    // unless the caller gives it (pdlp.cu:2036-2059).
    if (std::isfinite(p_.initial_step_size))
      eta_ = p_.initial_step_size;
    else if (p_.precision == 1)
      lanczos_step_size();
    else
      power_iteration();
    trace("engine: power iteration");

    xu_.resize(n);
    su_.resize(n);
    yu_.resize(m);
    scalars_.resize(1);
    reset_iterates(true);
    if constexpr (std::is_same_v<TX, float>) {
      if (tune_tiles()) reset_iterates(true);  // the timed sweeps moved the iterates
      trace("engine: sweep autotuning");
    }
    if (tune_sweep_shape()) reset_iterates(true);
    init_plain_form();
  }

  // Takes the precision-independent state of another engine over (see continue_from).
  template <typename TM>
  void adopt(engine<TM>& o)
  {
    const int m = in_.m, n = in_.n;
    t_start_     = o.t_start_;
    t_loop_      = o.t_loop_;
    sms_         = o.sms_;
    vgrid_       = o.vgrid_;
    L_           = std::move(o.L_);
    c64_         = std::move(o.c64_);
    l64_         = std::move(o.l64_);
    u64_         = std::move(o.u64_);
    lc64_        = std::move(o.lc64_);
    uc64_        = std::move(o.uc64_);
    dr_          = std::move(o.dr_);
    dc_          = std::move(o.dc_);
    partials_    = std::move(o.partials_);
    dres_        = std::move(o.dres_);
    scalars_     = std::move(o.scalars_);
    xu_          = std::move(o.xu_);
    yu_          = std::move(o.yu_);
    su_          = std::move(o.su_);
    obj_scale_   = o.obj_scale_;
    obj_offset_  = o.obj_offset_;
    eta_         = o.eta_;
    omega_       = o.omega_;
    best_omega_  = o.best_omega_;
    power_iters_ = o.power_iters_;
    restarts_    = o.restarts_;
    launches_    = o.launches_;
    sched_       = o.sched_;
    // Scaled matrices and vectors in FP64, from the unscaled data and the shared scaling.
    As_.resize(L_.A.stored());
    ATs_.resize(L_.AT.stored());
    scale_values_kernel<TX, false><<<sell_grid(view64(L_.A)), kBlock, 0, s_>>>(
      view64(L_.A), dr_.data(), dc_.data(), As_.data());
    scale_values_kernel<TX, true><<<sell_grid(view64(L_.AT)), kBlock, 0, s_>>>(
      view64(L_.AT), dr_.data(), dc_.data(), ATs_.data());
    launches_ += 2;
    prepare_vectors();
    // Iterates, anchors and the last averaged iterate, converted to FP64.
    for (auto* b : {&x_, &xhat_, &slack_, &xbar_, &xa_, &aty_}) {
      b->resize(n);
      b->zero(s_);
    }
    for (auto* b : {&y_, &yhat_, &ybar_, &ya_}) {
      b->resize(m);
      b->zero(s_);
    }
    copy_convert_kernel<TM, TX><<<vgrid_, kBlock, 0, s_>>>(x_.data(), o.x_.data(), n);
    copy_convert_kernel<TM, TX><<<vgrid_, kBlock, 0, s_>>>(xa_.data(), o.xa_.data(), n);
    copy_convert_kernel<TM, TX><<<vgrid_, kBlock, 0, s_>>>(xhat_.data(), o.xhat_.data(), n);
    copy_convert_kernel<TM, TX><<<vgrid_, kBlock, 0, s_>>>(slack_.data(), o.slack_.data(), n);
    copy_convert_kernel<TM, TX><<<vgrid_, kBlock, 0, s_>>>(y_.data(), o.y_.data(), m);
    copy_convert_kernel<TM, TX><<<vgrid_, kBlock, 0, s_>>>(ya_.data(), o.ya_.data(), m);
    copy_convert_kernel<TM, TX><<<vgrid_, kBlock, 0, s_>>>(yhat_.data(), o.yhat_.data(), m);
    launches_ += 7;
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    init_plain_form();
  }

  // Norms of the unscaled vectors and their scaled copies in the iterate precision (bound /
  // objective rescaling recomputed, reference initial_scaling.cu:95-149, 417-569).  Called at setup
  // and by an FP64 continuation that takes the scaling of a mixed-precision solve over.
  void prepare_vectors()
  {
    const int m = in_.m, n = in_.n;
    // Constant norms of the unscaled problem (reference convergence_information.cu:92-106).
    c_norm_ = std::sqrt(reduce<0>(c64_.data(), (const double*)nullptr, n));
    b_norm_ = std::sqrt(reduce<2>(lc64_.data(), uc64_.data(), m));
    dbuf<double> cs(n), ls(n), us(n), lcs(m), ucs(m);
    scale_vectors_kernel<<<vgrid_, kBlock, 0, s_>>>(c64_.data(), l64_.data(), u64_.data(),
                                                    lc64_.data(), uc64_.data(), dc_.data(),
                                                    dr_.data(), n, m, cs.data(), ls.data(),
                                                    us.data(), lcs.data(), ucs.data());
    beta_  = 1.0 / (std::sqrt(reduce<2>(lcs.data(), ucs.data(), m)) + 1.0);
    gamma_ = 1.0 / (std::sqrt(reduce<0>(cs.data(), (const double*)nullptr, n)) + 1.0);
    cs_.resize(n);
    ls_.resize(n);
    us_.resize(n);
    lcs_.resize(m);
    ucs_.resize(m);
    rescale_vectors_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(
      cs.data(), ls.data(), us.data(), lcs.data(), ucs.data(), beta_, gamma_, n, m, cs_.data(),
      ls_.data(), us_.data(), lcs_.data(), ucs_.data());
    launches_ += 2;
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  // Zeroed iterates (plus the caller's initial solution on the first solve), projected primal.
  void reset_iterates(bool with_initial)
  {
    const int m = in_.m, n = in_.n;
    // bound_objective_rescaling => primal weight 1 (pdlp.cu:2799-2810); a given initial weight
    // replaces it and the PID controller's best weight (pdlp.cu:2061-2083).
    omega_      = with_initial && std::isfinite(p_.initial_primal_weight) ? p_.initial_primal_weight
                                                                          : 1.0;
    best_omega_ = omega_;
    restarts_   = 0;
    // Four elements of zero padding: the tiled sweeps copy the gathered vectors in 16-byte units.
    for (auto* b : {&x_, &xhat_, &slack_, &xbar_, &xa_, &aty_}) {
      b->resize((size_t)n + 4);
      b->zero(s_);
    }
    for (auto* b : {&y_, &yhat_, &ybar_, &ya_}) {
      b->resize((size_t)m + 4);
      b->zero(s_);
    }
    if (with_initial && (in_.initial_primal || in_.initial_dual)) load_initial_solution();
    // project_initial_primal (reference pdlp.cu:2237-2262): only the current primal iterate.
    clamp_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(x_.data(), ls_.data(), us_.data(), n);
    ++launches_;
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  // Initial iterates: copied to x, x_hat and the anchor, then scaled
  // (reference pdlp.cu:1109-1245, compute_initial_primal_weight_before_scaling branch).
  void load_initial_solution()
  {
    const int m = in_.m, n = in_.n;
    if (in_.initial_primal) {
      dbuf<double> v(n);
      permute_gather(in_.initial_primal, L_.col_new2old.data(), n, 1.0, v.data(), s_);
      scale_initial_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(v.data(), dc_.data(), beta_, n,
                                                          x_.data(), xhat_.data(), xa_.data());
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    }
    if (in_.initial_dual) {
      dbuf<double> v(m);
      permute_gather(in_.initial_dual, L_.row_new2old.data(), m, 1.0, v.data(), s_);
      scale_initial_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(v.data(), dr_.data(), gamma_, m,
                                                          y_.data(), yhat_.data(), ya_.data());
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    }
    B200_LAUNCH_CHECK();
  }

  void fill(double* p, int n, double v)
  {
    fill_kernel<<<vgrid_, kBlock, 0, s_>>>(p, n, v);
    ++launches_;
    B200_LAUNCH_CHECK();
  }

  // Sum reduction of a vector expression (see vec_reduce_kernel) returned to the host.
  template <int MODE, typename TA>
  double reduce(const TA* a, const TA* b, int n)
  {
    vec_reduce_kernel<MODE, TA><<<vgrid_, kBlock, 0, s_>>>(a, b, n, partials_.data(), nullptr);
    finalize_sum_kernel<1><<<1, kBlock, 0, s_>>>(partials_.data(), vgrid_, dres_.data());
    launches_ += 2;
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(cudaMemcpyAsync(hres_, dres_.data(), sizeof(double), cudaMemcpyDeviceToHost, s_));
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    return hres_[0];
  }

  void power_iteration()
  {
    const int m = in_.m, n = in_.n;
    // Start vector: std::mt19937(1) normals in the user's constraint order (pdlp.cu:2632-2638).
    const auto seq          = power_start_sequence(m);
    const std::vector<double>& z0 = *seq;
    dbuf<double> dz(m), dq(m), datq(n);
    dbuf<power_state> ps(1);
    ps.zero(s_);
    dq.upload(z0.data(), m, s_);
    permute_gather(dq.data(), L_.row_new2old.data(), m, 1.0, dz.data(), s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    dbuf<TX> q_tx, atq_tx;
    const auto As  = view_of<TX>(L_.A, As_.data());
    const auto ATs = view_of<TX>(L_.AT, ATs_.data());
    const int ga = sell_grid(As), gt = sell_grid(ATs);
    // Block partials: |z|^2 and q . z in the first half of partials_ (the second overwrites the
    // first once it is consumed), the residual's in the second half.
    double* part   = partials_.data();
    double* part_r = partials_.data() + partials_.size() / 2;
    // The vector steps run on a grid sized to the m entries (at most vgrid_ blocks): small LPs
    // launch a few blocks instead of vgrid_ mostly idle ones.
    const int pg = std::max(1, std::min(vgrid_, ceil_div(m, kBlock)));
    if (cluster_power(As, ATs, dz.data(), ps.data(), pg, ga, gt)) return;
    auto one_iteration = [&]() {
      vec_reduce_kernel<0, double><<<pg, kBlock, 0, s_>>>(dz.data(), nullptr, m, part,
                                                          &ps.data()->done);
      power_normalize_sum_kernel<<<pg, kBlock, 0, s_>>>(dz.data(), dq.data(), m, part, pg,
                                                        ps.data());
      sell_map_kernel<TX, double, store_epi<double>><<<gt, kBlock, 0, s_>>>(
        ATs, dq.data(), store_epi<double>{datq.data(), &ps.data()->done}, part);
      sell_map_kernel<TX, double, power_z_epi><<<ga, kBlock, 0, s_>>>(
        As, datq.data(), power_z_epi{dz.data(), dq.data(), &ps.data()->done}, part);
      power_residual_sum_kernel<<<pg, kBlock, 0, s_>>>(dq.data(), dz.data(), m, part, ga,
                                                       ps.data(), part_r);
      power_check_sum_kernel<<<1, kBlock, 0, s_>>>(ps.data(), part, ga, part_r, pg, kPowerTol);
    };
    // Chunks of 32 iterations are captured once into a graph and replayed until convergence.
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    B200_CUDA_CHECK(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
    for (int i = 0; i < 32; ++i) one_iteration();
    B200_CUDA_CHECK(cudaStreamEndCapture(s_, &graph));
    B200_CUDA_CHECK(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    power_state h{};
    for (int done_iters = 0; done_iters < kPowerMaxIters; done_iters += 32) {
      if (kPowerMaxIters - done_iters < 32) {
        for (int i = 0; i < kPowerMaxIters - done_iters; ++i) one_iteration();
      } else {
        B200_CUDA_CHECK(cudaGraphLaunch(exec, s_));
      }
      launches_ += 6.0 * std::min(32, kPowerMaxIters - done_iters);
      B200_CUDA_CHECK(cudaMemcpyAsync(&h, ps.data(), sizeof(h), cudaMemcpyDeviceToHost, s_));
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
      if (h.done) break;
    }
    cudaGraphExecDestroy(exec);
    power_iters_ = h.iters;
    eta_         = kStepScaling / std::sqrt(h.s2);
  }

  // Small LPs (at most kClusterPowerNnz non-zeros and kClusterPowerMaxRows rows, z, q and A^T q
  // within one block's shared memory, and unless CUDA graphs are asked for with
  // pdlp_persistent_iterations = 0): the whole power iteration in one launch of
  // cluster_power_kernel, which forms every sum as the multi-kernel form does (same step size bit
  // for bit) with two cluster barriers per step in place of six kernel boundaries.  Returns false
  // where it does not apply.
  static constexpr int64_t kClusterPowerNnz = 262144;
  bool cluster_power(const dev_sell<TX>& As, const dev_sell<TX>& ATs, const double* z0,
                     power_state* ps, int pg, int ga, int gt)
  {
    if (p_.persistent == 0 || L_.nnz > kClusterPowerNnz || in_.m > kClusterPowerMaxRows ||
        pg > kClusterPowerMaxBlocks || ga > kClusterPowerMaxBlocks)
      return false;
    int dev = 0, optin = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t vec_smem = cluster_power_smem(in_.m, in_.n, pg, ga);
    const size_t limit = max_dynamic_smem((const void*)cluster_power_kernel<TX>);
    if (vec_smem > limit) return false;
    // Shared memory a block needs to hold its own virtual blocks of both sweeps (cluster size c).
    auto ranges = [&](const dev_matrix& M) {
      std::vector<int64_t> lo(M.n_long + 1), so(M.n_slices + 1);
      B200_CUDA_CHECK(cudaMemcpyAsync(lo.data(), M.long_off.data(), lo.size() * sizeof(int64_t),
                                      cudaMemcpyDeviceToHost, s_));
      B200_CUDA_CHECK(cudaMemcpyAsync(so.data(), M.slice_off.data(),
                                      so.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, s_));
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
      std::vector<int64_t> count;  // elements of each virtual block
      const int lb = long_blocks(M.n_long);
      for (int vb = 0; vb < lb; ++vb)
        count.push_back(lo[std::min((vb + 1) * kWarpsPerBlock, M.n_long)] - lo[vb * kWarpsPerBlock]);
      for (int s0 = 0; s0 < M.n_slices; s0 += kWarpsPerBlock)
        count.push_back(so[std::min(s0 + kWarpsPerBlock, M.n_slices)] - so[s0]);
      return count;
    };
    const std::vector<int64_t> cnt_t = ranges(L_.AT), cnt_a = ranges(L_.A);
    auto copy_smem = [&](int c) -> size_t {
      size_t worst = 0;
      for (int r = 0; r < c; ++r) {
        size_t bytes = 0;
        int own      = 0;
        for (const auto* cnt : {&cnt_t, &cnt_a}) {
          int k = 0;
          for (size_t vb = r; vb < cnt->size(); vb += c, ++k)
            bytes += (((*cnt)[vb] * sizeof(TX) + 15) & ~size_t(15)) +
                     (((*cnt)[vb] * sizeof(int) + 15) & ~size_t(15));
          own = std::max(own, k);
        }
        if (own > kClusterPowerMaxOwn) return SIZE_MAX;
        worst = std::max(worst, bytes);
      }
      return worst;
    };
    const void* fn = (const void*)cluster_power_kernel<TX>;
    int blocks = 0, cache = 0;
    size_t smem = vec_smem;
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    // 16 blocks where the device allows clusters of that size, else the portable 8; the matrix
    // copy where it fits beside the vectors.
    for (int c : {16, 8}) {
      if (c > 8)
        if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
            cudaSuccess) {
          (void)cudaGetLastError();
          continue;
        }
      const size_t mat = copy_smem(c);
      cache            = mat != SIZE_MAX && vec_smem + mat <= limit;
      smem             = vec_smem + (cache ? mat : 0);
      allow_max_dynamic_smem(fn);
      cfg                      = cudaLaunchConfig_t{};
      cfg.gridDim              = dim3(c);
      cfg.blockDim             = dim3(kBlock);
      cfg.dynamicSmemBytes     = smem;
      cfg.stream               = s_;
      attr[0].id               = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = c;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs                = attr;
      cfg.numAttrs             = 1;
      int clusters             = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, fn, &cfg) == cudaSuccess && clusters > 0) {
        blocks = c;
        break;
      }
      (void)cudaGetLastError();
    }
    if (blocks == 0) return false;
    B200_CUDA_CHECK(cudaLaunchKernelEx(&cfg, cluster_power_kernel<TX>, ATs, As, z0, in_.m, in_.n,
                                       pg, gt, ga, ps, kPowerTol, kPowerMaxIters, cache));
    ++launches_;
    power_state h{};
    B200_CUDA_CHECK(cudaMemcpyAsync(&h, ps, sizeof(h), cudaMemcpyDeviceToHost, s_));
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    power_iters_    = h.iters;
    eta_            = kStepScaling / std::sqrt(h.s2);
    cluster_blocks_ = blocks;
    if (std::getenv("CUOPT_B200_TRACE"))
      std::fprintf(stderr, "[cuopt_b200] cluster power iteration: %d blocks, %zu bytes of shared "
                           "memory each, matrix copy %s\n",
                   blocks, smem, cache ? "on" : "off");
    return true;
  }

  // Largest singular value of the scaled A by Golub-Kahan-Lanczos bidiagonalisation, used in
  // mixed precision (where the iterates are not expected to match the FP64 reference path): the
  // estimate sigma_max(B_k) of the bidiagonal B_k rises to sigma_max(A) within tens of matrix
  // pairs, where the reference's power iteration (kept for FP64) takes hundreds.  Same start vector
  // as the power iteration; stops when the estimate changes by less than 1e-10 relative.
  void lanczos_step_size()
  {
    const int m = in_.m, n = in_.n;
    const auto seq          = power_start_sequence(m);
    const std::vector<double>& z0 = *seq;
    constexpr int kChunk = kLanczosChunk, kMaxSteps = kLanczosMaxSteps;
    dbuf<double> u(m), v(n), tmp(m), alphas(kMaxSteps + 1), betas(kMaxSteps + 2);
    dbuf<gk_state> st(1);
    tmp.upload(z0.data(), m, s_);
    permute_gather(tmp.data(), L_.row_new2old.data(), m, 1.0, u.data(), s_);
    v.zero(s_);
    st.zero(s_);
    double beta0 = 0.0;
    {
      vec_reduce_kernel<0, double><<<vgrid_, kBlock, 0, s_>>>(u.data(), nullptr, m,
                                                              partials_.data(), nullptr);
      finalize_sum_kernel<1><<<1, kBlock, 0, s_>>>(partials_.data(), vgrid_, dres_.data());
      gk_record_kernel<1><<<1, 1, 0, s_>>>(st.data(), dres_.data(), betas.data(), -1);
      launches_ += 3;
      B200_LAUNCH_CHECK();
      betas.download(&beta0, 1, s_);
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    }
    const auto As = view_of<TX>(L_.A, As_.data()), ATs = view_of<TX>(L_.AT, ATs_.data());
    auto step = [&](int k) {
      sell_map_kernel<TX, double, gk_primal_epi><<<sell_grid(ATs), kBlock, 0, s_>>>(
        ATs, u.data(), gk_primal_epi{v.data(), st.data()}, partials_.data());
      finalize_sum_kernel<1><<<1, kBlock, 0, s_>>>(partials_.data(), sell_grid(ATs),
                                                   dres_.data());
      gk_record_kernel<0><<<1, 1, 0, s_>>>(st.data(), dres_.data(), alphas.data(), k);
      sell_map_kernel<TX, double, gk_dual_epi><<<sell_grid(As), kBlock, 0, s_>>>(
        As, v.data(), gk_dual_epi{u.data(), st.data()}, partials_.data());
      finalize_sum_kernel<1><<<1, kBlock, 0, s_>>>(partials_.data(), sell_grid(As),
                                                   dres_.data() + 1);
      gk_record_kernel<1><<<1, 1, 0, s_>>>(st.data(), dres_.data() + 1, betas.data(), k);
    };
    std::vector<double> ha(kMaxSteps + 1), hb(kMaxSteps + 2);
    double sigma2 = 0.0, prev = -1.0;
    int k = 0;
    while (k < kMaxSteps) {
      const int c = std::min(kChunk, kMaxSteps - k);
      for (int i = 0; i < c; ++i) step(k + i);
      launches_ += 6.0 * c;
      B200_LAUNCH_CHECK();
      k += c;
      alphas.download(ha.data(), k, s_);
      betas.download(hb.data(), k + 1, s_);
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
      // betas[0] holds |z0| (written at index -1 + 1); the recurrence coefficients are betas[1..].
      bool breakdown = false;
      int used = k;
      for (int j = 0; j < k; ++j)
        if (!(ha[j] > 0.0) || !(hb[j + 1] > 0.0) || !std::isfinite(ha[j]) || !std::isfinite(hb[j + 1])) {
          used      = j + 1;
          breakdown = true;
          break;
        }
      sigma2 = largest_bidiagonal_sigma2(ha.data(), hb.data() + 1, used);
      if (breakdown || (prev > 0.0 && std::fabs(sigma2 - prev) <= kLanczosTol * sigma2)) {
        k = used;
        break;
      }
      prev = sigma2;
    }
    (void)beta0;
    power_iters_ = k;
    eta_         = kStepScaling / std::sqrt(sigma2);
  }

  // ------------------------------------------------------------------ iteration kernels
  dev_sell<TX> As_view() const { return view_of<TX>(L_.A, As_.data()); }
  dev_sell<TX> ATs_view() const { return view_of<TX>(L_.AT, ATs_.data()); }

  // The plain sweeps (not major, Halpern step fused, no fixed-point error) run with the tuned
  // number of warps per block; the others with kWarpsPerBlock.
  template <bool MAJOR, bool HALPERN, bool SAVE_ATY>
  void launch_primal(int it_off, int wpb = 0)
  {
    const auto A = ATs_view();
    primal_epi<TX, MAJOR, HALPERN, SAVE_ATY> e{x_.data(),    cs_.data(),    ls_.data(),
                                               us_.data(),   xa_.data(),    xbar_.data(),
                                               x_.data(),    xhat_.data(),  slack_.data(),
                                               aty_.data(),  scalars_.data(), it_off};
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
    const auto A = As_view();
    dual_epi<TX, MAJOR, HALPERN, FPE> e{y_.data(),    lcs_.data(), ucs_.data(),     ya_.data(),
                                        ybar_.data(), y_.data(),   yhat_.data(),    scalars_.data(),
                                        it_off};
    if constexpr (!MAJOR && HALPERN && !FPE)
      launch_sell_wpb(wpb ? wpb : wpb_dual_, A, xbar_.data(), e, partials_.data(), s_);
    else
      sell_map_kernel<TX, TX, decltype(e)><<<sell_grid(A), kBlock, 0, s_>>>(A, xbar_.data(), e,
                                                                           partials_.data());
    ++launches_;
  }

  // Block shape of the plain sliced-ELL sweeps (pdlp_sweep_warps_per_block = 0): each sweep is
  // timed with 4, 8 and 16 warps per block (a warm-up launch, then about 1 ms of launches, CUDA
  // events on the solve's stream); another shape replaces 8 warps when it is at least 3 % faster.
  // The shape only groups the same warps differently, so the iterates do not depend on it.
  // Decisions are remembered per problem shape, device and precision.  Returns true when sweeps
  // were launched (the caller then resets the iterates).
  bool tune_sweep_shape()
  {
    for (auto& t : wpb_ms_) t[0] = t[1] = t[2] = 0.0;
    wpb_primal_ = wpb_dual_ = p_.sweep_wpb ? p_.sweep_wpb : kWarpsPerBlock;
    if (p_.sweep_wpb) return false;
    int dev = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    const form_key key{in_.m, in_.n, L_.nnz, dev, (int)sizeof(TX)};
    {
      std::lock_guard<std::mutex> lock(tune_mutex());
      auto it = shape_cache().find(key);
      if (it != shape_cache().end()) {
        wpb_primal_ = it->second.wpb_primal;
        wpb_dual_   = it->second.wpb_dual;
        std::memcpy(wpb_ms_, it->second.ms, sizeof(wpb_ms_));
        return false;
      }
    }
    set_scalars(0);
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
      const int w = kShapes[q];
      if (!(tile_primal_)) wpb_ms_[0][q] = time_of([&] { launch_primal<false, true, false>(0, w); });
      if (!(tile_dual_)) wpb_ms_[1][q] = time_of([&] { launch_dual<false, true, false>(0, w); });
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
      std::lock_guard<std::mutex> lock(tune_mutex());
      shape_choice c{wpb_primal_, wpb_dual_, {}};
      std::memcpy(c.ms, wpb_ms_, sizeof(wpb_ms_));
      shape_cache()[key] = c;
    }
    if (std::getenv("CUOPT_B200_TRACE"))
      std::fprintf(stderr,
                   "[cuopt_b200] sweep block shape: primal %.4f/%.4f/%.4f ms -> %d warps; dual "
                   "%.4f/%.4f/%.4f ms -> %d warps (4/8/16 warps per block)\n",
                   wpb_ms_[0][0], wpb_ms_[0][1], wpb_ms_[0][2], wpb_primal_, wpb_ms_[1][0],
                   wpb_ms_[1][1], wpb_ms_[1][2], wpb_dual_);
    return true;
  }

  // Tiled forms of the plain (non-major, Halpern) sweeps: the tile kernel's partial sums, then the
  // epilogue row pass with the same functor as the sliced-ELL sweep.
  void launch_primal_tiled(int it_off)
  {
    const tile_view T = view_of(tAT_);
    tile_sweep_kernel<<<T.row_blocks * T.groups, kTileThreads, tAT_.smem_bytes(), s_>>>(
      T, y_.data(), tpart_.data(), terr_.data());
    primal_epi<TX, false, true, false> e{x_.data(),   cs_.data(),   ls_.data(),   us_.data(),
                                         xa_.data(),  xbar_.data(), x_.data(),    xhat_.data(),
                                         slack_.data(), aty_.data(), scalars_.data(), it_off};
    tile_epilogue_kernel<decltype(e)><<<epi_grid(in_.n), kBlock, 0, s_>>>(
      in_.n, T.groups, tpart_.data(), e, partials_.data());
    launches_ += 2;
  }
  void launch_dual_tiled(int it_off)
  {
    const tile_view T = view_of(tA_);
    tile_sweep_kernel<<<T.row_blocks * T.groups, kTileThreads, tA_.smem_bytes(), s_>>>(
      T, xbar_.data(), tpart_.data(), terr_.data());
    dual_epi<TX, false, true, false> e{y_.data(),    lcs_.data(), ucs_.data(),     ya_.data(),
                                       ybar_.data(), y_.data(),   yhat_.data(),    scalars_.data(),
                                       it_off};
    tile_epilogue_kernel<decltype(e)><<<epi_grid(in_.m), kBlock, 0, s_>>>(
      in_.m, T.groups, tpart_.data(), e, partials_.data());
    launches_ += 2;
  }
  int epi_grid(int rows) const { return std::max(1, std::min(ceil_div(rows, kBlock), vgrid_)); }

  // Autotuning of the mixed-precision sweeps (pdlp_tiled_sweeps = -1): builds the tiled copies of
  // A and A^T where they apply, times each plain sweep both ways (one warm-up and three timed
  // launches each, CUDA events on the solve's stream) and keeps the faster form per sweep.  With
  // pdlp_tiled_sweeps = 1 the tiled form is used wherever it was built, with 0 never.  Returns true
  // when sweeps were launched (the caller then resets the iterates).
  bool tune_tiles()
  {
    tile_primal_ = tile_dual_ = false;
    if (p_.tiled_sweeps == 0) return false;
    int dev = 0, optin = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t limit = (size_t)optin - 64;  // the two mbarriers of the static shared memory
    // A shape tuned before in this process reuses its decision: only the tiled copies it chose
    // are built, and nothing is timed.
    const tune_key key{in_.m, in_.n, L_.nnz, dev};
    bool want_a = true, want_t = true, cached = false;
    if (p_.tiled_sweeps == -1) {
      std::lock_guard<std::mutex> lock(tune_mutex());
      auto it = tune_cache().find(key);
      if (it != tune_cache().end()) {
        cached = true;
        want_t = it->second.first;
        want_a = it->second.second;
      }
    }
    if (cached && !want_a && !want_t) return false;
    // Worth trying only when a row block's panel copies stay within a few matrix reads.
    auto worth = [&](const tile_matrix& t, int64_t nnz) {
      return p_.tiled_sweeps == 1 || t.staging_bytes() <= 4.0 * (double)nnz * 8.0;
    };
    const int64_t nnz = L_.nnz;
    bool have_a = want_a && build_tile_matrix(L_.A, As_.data(), sms_, limit, s_, tA_) &&
                  worth(tA_, nnz);
    bool have_t = want_t && build_tile_matrix(L_.AT, ATs_.data(), sms_, limit, s_, tAT_) &&
                  worth(tAT_, nnz);
    if (!have_a) tA_ = tile_matrix{};
    if (!have_t) tAT_ = tile_matrix{};
    if (!have_a && !have_t) return false;
    const size_t smem = std::max(have_a ? tA_.smem_bytes() : 0, have_t ? tAT_.smem_bytes() : 0);
    allow_max_dynamic_smem((const void*)tile_sweep_kernel);
    (void)smem;
    tpart_.resize(std::max(have_a ? (size_t)tA_.groups * in_.m : 1,
                           have_t ? (size_t)tAT_.groups * in_.n : 1));
    terr_.resize(1);
    terr_.zero(s_);
    if (p_.tiled_sweeps == 1 || cached) {
      tile_primal_ = have_t;
      tile_dual_   = have_a;
      return false;
    }
    set_scalars(0);
    cudaEvent_t e0, e1;
    B200_CUDA_CHECK(cudaEventCreate(&e0));
    B200_CUDA_CHECK(cudaEventCreate(&e1));
    auto time_of = [&](auto&& launch) {
      launch();
      B200_CUDA_CHECK(cudaEventRecord(e0, s_));
      for (int i = 0; i < 3; ++i) launch();
      B200_CUDA_CHECK(cudaEventRecord(e1, s_));
      B200_CUDA_CHECK(cudaEventSynchronize(e1));
      float ms = 0.f;
      B200_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      return (double)ms;
    };
    if (have_t) {
      const double sell = time_of([&] { launch_primal<false, true, false>(0); });
      const double tile = time_of([&] { launch_primal_tiled(0); });
      tile_primal_      = tile < sell;
      tune_ms_[0] = sell / 3, tune_ms_[1] = tile / 3;
    }
    if (have_a) {
      const double sell = time_of([&] { launch_dual<false, true, false>(0); });
      const double tile = time_of([&] { launch_dual_tiled(0); });
      tile_dual_        = tile < sell;
      tune_ms_[2] = sell / 3, tune_ms_[3] = tile / 3;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    check_tile_error();
    if (!tile_primal_) tAT_ = tile_matrix{};
    if (!tile_dual_) tA_ = tile_matrix{};
    {
      std::lock_guard<std::mutex> lock(tune_mutex());
      tune_cache()[key] = {tile_primal_, tile_dual_};
    }
    if (std::getenv("CUOPT_B200_TRACE"))
      std::fprintf(stderr,
                   "[cuopt_b200] sweep autotune: primal sell %.4f tiled %.4f ms -> %s; dual sell "
                   "%.4f tiled %.4f ms -> %s\n",
                   tune_ms_[0], tune_ms_[1], tile_primal_ ? "tiled" : "sell", tune_ms_[2],
                   tune_ms_[3], tile_dual_ ? "tiled" : "sell");
    return true;
  }

  // A tiled sweep whose panel copy did not complete in its bounded wait reports it here (read at
  // every termination check, where the host synchronises anyway).
  void check_tile_error()
  {
    if (!(tile_primal_ || tile_dual_) || terr_.size() == 0) return;
    int e = 0;
    B200_CUDA_CHECK(cudaMemcpyAsync(&e, terr_.data(), sizeof(int), cudaMemcpyDeviceToHost, s_));
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    if (e) throw cuda_error("tiled sweep: a panel copy did not complete within its wait limit");
  }

  // The plain (non-major, Halpern) sweeps in the form the autotuner chose.
  void plain_primal(int it_off)
  {
    if constexpr (std::is_same_v<TX, float>) {
      if (tile_primal_) return launch_primal_tiled(it_off);
    }
    launch_primal<false, true, false>(it_off);
  }
  void plain_dual(int it_off)
  {
    if constexpr (std::is_same_v<TX, float>) {
      if (tile_dual_) return launch_dual_tiled(it_off);
    }
    launch_dual<false, true, false>(it_off);
  }

  void plain_iterations(int L)  // L fused iterations, then t0 += L
  {
    for (int i = 0; i < L; ++i) {
      plain_primal(i);
      plain_dual(i);
    }
    advance_kernel<<<1, 1, 0, s_>>>(scalars_.data(), L);
    ++launches_;
  }

  // ------------------------------------------------------------------ persistent plain iterations
  using persist_pe = primal_epi<TX, false, true, false>;
  using persist_de = dual_epi<TX, false, true, false>;
  static const void* persistent_fn()
  {
    return (const void*)persistent_plain_kernel<TX, persist_pe, persist_de, advance_one>;
  }

  // Sizes the persistent launch (all co-resident blocks, at most one per virtual block of the
  // larger sweep) and sets up the choice of form for this solve.
  void init_plain_form()
  {
    int dev = 0, coop = 0, per_sm = 0;
    B200_CUDA_CHECK(cudaGetDevice(&dev));
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    B200_CUDA_CHECK(
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, persistent_fn(), kBlock, 0));
    const int need = std::max(sell_grid(ATs_view()), sell_grid(As_view()));
    persist_grid_  = std::min(need, per_sm * sms_);
    // The persistent and cluster kernels run the sliced-ELL sweeps only.
    const bool sell = !tile_primal_ && !tile_dual_;
    const bool ok   = coop && persist_grid_ > 0 && sell;
    pctl_.resize(1);
    pctl_.zero(s_);
    // The cluster form where both gathered vectors fit in one block's shared memory.
    int optin = 0;
    B200_CUDA_CHECK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    cluster_smem_ = ((size_t)((in_.m + 15) & ~15) + (size_t)in_.n) * sizeof(TX);
    bool cl_ok    = sell && cluster_smem_ <= max_dynamic_smem(cluster_fn());
    if (cl_ok) {
      allow_max_dynamic_smem(cluster_fn());
      cudaLaunchConfig_t cfg{};
      cudaLaunchAttribute attr[1];
      cluster_config(cfg, attr);
      int clusters = 0;
      cl_ok = cudaOccupancyMaxActiveClusters(&clusters, cluster_fn(), &cfg) == cudaSuccess &&
              clusters > 0;
      (void)cudaGetLastError();
    }
    form_key_ = form_key{in_.m, in_.n, L_.nnz, dev, (int)sizeof(TX)};
    int known = -1;
    for (double& u : form_us_) u = 0.0;
    if (p_.persistent == -1) {
      std::lock_guard<std::mutex> lock(tune_mutex());
      auto it = form_cache().find(form_key_);
      if (it != form_cache().end()) {
        known = it->second.form;
        std::memcpy(form_us_, it->second.us, sizeof(form_us_));
      }
    }
    cycle_open_ = false;
    const bool avail[plain_form_tuner::kForms] = {true, ok, cl_ok};
    form_.reset(p_.persistent, known, avail);
  }

  // ------------------------------------------------------------------ cluster plain iterations
  static constexpr int kClusterBlocks = 8;  // blocks per cluster (the portable maximum)
  static const void* cluster_fn()
  {
    return (const void*)cluster_plain_kernel<TX>;
  }
  void cluster_config(cudaLaunchConfig_t& cfg, cudaLaunchAttribute (&attr)[1]) const
  {
    cfg                              = cudaLaunchConfig_t{};
    cfg.gridDim                      = dim3(kClusterBlocks);
    cfg.blockDim                     = dim3(kClusterThreads);
    cfg.dynamicSmemBytes             = cluster_smem_;
    cfg.stream                       = s_;
    attr[0].id                       = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x         = kClusterBlocks;
    attr[0].val.clusterDim.y         = 1;
    attr[0].val.clusterDim.z         = 1;
    cfg.attrs                        = attr;
    cfg.numAttrs                     = 1;
  }
  // Returns true for the first launch of the engine (which may include loading the kernel).
  bool launch_cluster(int L)
  {
    const auto AT = ATs_view(), A = As_view();
    persist_pe pe{x_.data(),   cs_.data(),   ls_.data(),    us_.data(),  xa_.data(),
                  xbar_.data(), x_.data(),   xhat_.data(),  slack_.data(), aty_.data(),
                  scalars_.data(), 0};
    persist_de de{y_.data(),    lcs_.data(), ucs_.data(),  ya_.data(),      ybar_.data(),
                  y_.data(),    yhat_.data(), scalars_.data(), 0};
    cudaLaunchConfig_t cfg{};
    cudaLaunchAttribute attr[1];
    cluster_config(cfg, attr);
    B200_CUDA_CHECK(cudaLaunchKernelEx(&cfg, cluster_plain_kernel<TX>, AT, A, pe, de, L, in_.m,
                                       sell_grid(AT), sell_grid(A), scalars_.data()));
    ++launches_;
    return cluster_launches_++ == 0;
  }

  // Returns true for the first launch of the engine (which may include loading the kernel).
  bool launch_persistent(int L)
  {
    const auto AT = ATs_view(), A = As_view();
    persist_pe pe{x_.data(),   cs_.data(),   ls_.data(),    us_.data(),  xa_.data(),
                  xbar_.data(), x_.data(),   xhat_.data(),  slack_.data(), aty_.data(),
                  scalars_.data(), 0};
    persist_de de{y_.data(),    lcs_.data(), ucs_.data(),  ya_.data(),      ybar_.data(),
                  y_.data(),    yhat_.data(), scalars_.data(), 0};
    advance_one adv{scalars_.data()};
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
    return persist_launches_++ == 0;
  }

  // After a synchronisation: timings of the forms, and the decision once made.
  void collect_form_timing()
  {
    const bool before = form_.decided();
    form_.collect();
    if (!before && form_.decided()) {
      for (int f = 0; f < plain_form_tuner::kForms; ++f) form_us_[f] = form_.us_per_iteration(f);
      {
        std::lock_guard<std::mutex> lock(tune_mutex());
        form_choice c{form_.chosen(), {}};
        std::memcpy(c.us, form_us_, sizeof(form_us_));
        form_cache()[form_key_] = c;
      }
      if (std::getenv("CUOPT_B200_TRACE"))
        std::fprintf(stderr,
                     "[cuopt_b200] plain iterations: graphs %.2f us, persistent (%d blocks) %.2f "
                     "us, cluster %.2f us per iteration -> %s\n",
                     form_.us_per_iteration(0), persist_grid_, form_.us_per_iteration(1),
                     form_.us_per_iteration(2),
                     form_.chosen() == 2 ? "cluster" : form_.chosen() ? "persistent" : "graphs");
    }
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
    cycle_one_time_ |= cycle_form_ == 2   ? launch_cluster((int)R)
                       : cycle_form_ == 1 ? launch_persistent((int)R)
                                          : run_graphs(R);
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
          launches_ = before;  // captured, not launched
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

  void set_scalars(long long t0)
  {
    set_scalars_kernel<<<1, 1, 0, s_>>>(scalars_.data(), eta_ / omega_, eta_ * omega_, eta_,
                                        omega_, t0);
    ++launches_;
    B200_LAUNCH_CHECK();
  }

  // ------------------------------------------------------------------ termination
  conv_info evaluate()
  {
    const int m = in_.m, n = in_.n;
    unscale_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(xhat_.data(), yhat_.data(), slack_.data(),
                                                  dc_.data(), dr_.data(), 1.0 / beta_,
                                                  1.0 / gamma_, n, m, xu_.data(), yu_.data(),
                                                  su_.data());
    ++launches_;
    return evaluate_unscaled();
  }

  // Residuals and objectives of (xu_, yu_, su_) on the unscaled problem (c64_, lc64_, uc64_).
  conv_info evaluate_unscaled()
  {
    enqueue_conv(hres_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    collect_form_timing();
    return read_conv(hres_);
  }

  // The kernels of a termination check on (xu_, yu_, su_) and the copy of their results to the
  // pinned host buffer h: h[0..6] the sums, h[8] two error flags (the persistent kernel's barrier
  // status and the tiled sweeps' bounded-wait flag).
  void enqueue_conv(double* h)
  {
    const auto A = view64(L_.A), AT = view64(L_.AT);
    sell_map_kernel<double, double, term_primal_epi><<<sell_grid(A), kBlock, 0, s_>>>(
      A, xu_.data(), term_primal_epi{lc64_.data(), uc64_.data(), yu_.data()}, partials_.data());
    finalize_sum_kernel<2><<<1, kBlock, 0, s_>>>(partials_.data(), sell_grid(A), dres_.data());
    sell_map_kernel<double, double, term_dual_epi><<<sell_grid(AT), kBlock, 0, s_>>>(
      AT, yu_.data(), term_dual_epi{c64_.data(), xu_.data(), su_.data()}, partials_.data());
    finalize_sum_kernel<3><<<1, kBlock, 0, s_>>>(partials_.data(), sell_grid(AT),
                                                 dres_.data() + 2);
    launches_ += 4;
    int nres = 5;
    if (p_.per_constraint_residual) {
      sell_map_kernel<double, double, term_linf_primal_epi><<<sell_grid(A), kBlock, 0, s_>>>(
        A, xu_.data(), term_linf_primal_epi{lc64_.data(), uc64_.data(), p_.rel_primal},
        partials_.data());
      finalize_max_kernel<1><<<1, kBlock, 0, s_>>>(partials_.data(), sell_grid(A),
                                                   dres_.data() + 5);
      sell_map_kernel<double, double, term_linf_dual_epi><<<sell_grid(AT), kBlock, 0, s_>>>(
        AT, yu_.data(), term_linf_dual_epi{c64_.data(), su_.data(), p_.rel_dual},
        partials_.data());
      finalize_max_kernel<1><<<1, kBlock, 0, s_>>>(partials_.data(), sell_grid(AT),
                                                   dres_.data() + 6);
      launches_ += 4;
      nres = 7;
    }
    B200_LAUNCH_CHECK();
    B200_CUDA_CHECK(
      cudaMemcpyAsync(h, dres_.data(), nres * sizeof(double), cudaMemcpyDeviceToHost, s_));
    int* flags = reinterpret_cast<int*>(h + 8);
    flags[0] = flags[1] = 0;
    if (persist_launches_ > 0)
      B200_CUDA_CHECK(cudaMemcpyAsync(flags, &pctl_.data()->status, sizeof(int),
                                      cudaMemcpyDeviceToHost, s_));
    if ((tile_primal_ || tile_dual_) && terr_.size() > 0)
      B200_CUDA_CHECK(
        cudaMemcpyAsync(flags + 1, terr_.data(), sizeof(int), cudaMemcpyDeviceToHost, s_));
  }

  // The check's results from h once the copies have completed.  Throws when a persistent launch's
  // barrier or a tiled sweep's panel copy gave up its wait since the solve began.
  conv_info read_conv(const double* h)
  {
    const int* flags = reinterpret_cast<const int*>(h + 8);
    if (flags[0] != 0)
      throw cuda_error(flags[0] == kBarrierTimedOut
                         ? "persistent iterations: a grid barrier passed its deadline"
                         : "persistent iterations: a grid barrier passed its poll limit");
    if (flags[1] != 0)
      throw cuda_error("tiled sweep: a panel copy did not complete within its wait limit");
    conv_info cv;
    if (p_.per_constraint_residual) {
      cv.linf_primal = h[5];
      cv.linf_dual   = h[6];
    }
    cv.l2_primal  = std::sqrt(h[0]);
    cv.l2_dual    = std::sqrt(h[2]);
    cv.primal_obj = h[3];
    cv.dual_obj   = h[4] + h[1];
    if (obj_scale_ != 1.0 || obj_offset_ != 0.0) {
      cv.primal_obj = obj_scale_ * (cv.primal_obj + obj_offset_);
      cv.dual_obj   = obj_scale_ * (cv.dual_obj + obj_offset_);
    }
    cv.gap     = std::fabs(cv.primal_obj - cv.dual_obj);
    cv.abs_obj = std::fabs(cv.primal_obj) + std::fabs(cv.dual_obj);
    return cv;
  }

  void finish(pdlp_result& r, int status, const conv_info& cv, long k)
  {
    r.status     = status;
    r.iterations = k;
    r.primal_obj = cv.primal_obj;
    r.dual_obj   = cv.dual_obj;
    // With per_constraint_residual the statistics carry the per-constraint forms (reference
    // termination_strategy.cu:540-566).
    r.l2_primal  = p_.per_constraint_residual ? cv.linf_primal : cv.l2_primal;
    r.l2_dual    = p_.per_constraint_residual ? cv.linf_dual : cv.l2_dual;
    r.rel_primal = cv.l2_primal / (1.0 + b_norm_);
    r.rel_dual   = cv.l2_dual / (1.0 + c_norm_);
    r.gap        = cv.gap;
    r.rel_gap    = cv.gap / (1.0 + cv.abs_obj);
    r.step_size  = eta_;
    r.primal_weight = omega_;
    r.restarts   = restarts_;
    r.kernel_launches = launches_;
    // -1: the solve ended while both forms were still being timed.
    r.plain_form          = form_.decided() ? form_.chosen() : -1;
    r.persistent_blocks   = persist_grid_;
    r.us_plain_graphs     = form_.decided() ? form_us_[0] : form_.us_per_iteration(0);
    r.us_plain_persistent = form_.decided() ? form_us_[1] : form_.us_per_iteration(1);
    r.us_plain_cluster    = form_.decided() ? form_us_[2] : form_.us_per_iteration(2);
    r.wpb_primal          = wpb_primal_;
    r.wpb_dual            = wpb_dual_;
    std::memcpy(r.wpb_ms, wpb_ms_, sizeof(wpb_ms_));
  }

  bool meets(const conv_info& cv, double tol) const
  {
    return cv.l2_primal <= tol + tol * b_norm_ && cv.l2_dual <= tol + tol * c_norm_ &&
           cv.gap <= tol + tol * cv.abs_obj;
  }
  static double rel_kkt(const conv_info& cv, double bn, double cn)
  {
    return std::max({cv.l2_primal / (1.0 + bn), cv.l2_dual / (1.0 + cn), cv.gap / (1.0 + cv.abs_obj)});
  }

  void copy_d(double* dst, const double* src, int n)
  {
    B200_CUDA_CHECK(cudaMemcpyAsync(dst, src, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, s_));
  }

  // Solution in the user's order; duals and reduced costs negated for maximisation
  // (reference solve.cu:584-588).
  void write_outputs()
  {
    const int m = in_.m, n = in_.n;
    const double sgn = in_.maximize ? -1.0 : 1.0;
    if (x_out_) permute_scatter(xu_.data(), L_.col_new2old.data(), n, 1.0, x_out_, s_);
    if (rc_out_) permute_scatter(su_.data(), L_.col_new2old.data(), n, sgn, rc_out_, s_);
    if (y_out_) permute_scatter(yu_.data(), L_.row_new2old.data(), m, sgn, y_out_, s_);
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
  }

  void finish_times(pdlp_result& r)
  {
    const double t = now_s();
    r.solve_time   = t - t_start_;
    r.setup_time   = (t_loop_ > 0 ? t_loop_ : t) - t_start_;
    r.loop_time    = t_loop_ > 0 ? t - t_loop_ : 0.0;
  }

  // Host-side sum / maximum of block statistics (fixed order).
  template <bool MAX>
  double stat(const double* a, int count)
  {
    block_stat_kernel<MAX><<<vgrid_, kBlock, 0, s_>>>(a, count, partials_.data());
    ++launches_;
    B200_LAUNCH_CHECK();
    std::vector<double> h(vgrid_);
    B200_CUDA_CHECK(cudaMemcpyAsync(h.data(), partials_.data(), vgrid_ * sizeof(double),
                                    cudaMemcpyDeviceToHost, s_));
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    double v = 0.0;
    for (double p : h) v = MAX ? std::max(v, p) : v + p;
    return v;
  }

  // Ray statistics of the infeasibility test (reference infeasibility_information.cu:230-490,
  // cuPDLPx branch) from x_bar - x and y_bar - y of the current step.
  void ray_statistics()
  {
    const int m = in_.m, n = in_.n;
    dbuf<double> d(n), cd(n), e(m), pe(m), vm(m), sn(n), vn(n);
    ray_vectors_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(
      x_.data(), xbar_.data(), ls_.data(), us_.data(), cs_.data(), n, y_.data(), ybar_.data(),
      lcs_.data(), ucs_.data(), m, d.data(), cd.data(), e.data(), pe.data());
    ++launches_;
    B200_LAUNCH_CHECK();
    const double nd = stat<true>(d.data(), n), ne = stat<true>(e.data(), m);
    const double sum_cd = stat<false>(cd.data(), n), sum_ps = stat<false>(pe.data(), m);
    const auto A = As_view(), AT = ATs_view();
    sell_map_kernel<TX, double, ray_primal_epi<TX>><<<sell_grid(A), kBlock, 0, s_>>>(
      A, d.data(),
      ray_primal_epi<TX>{lcs_.data(), ucs_.data(), dr_.data(), nd > 0.0 ? 1.0 / nd : 1.0,
                         vm.data()},
      partials_.data());
    sell_map_kernel<TX, double, ray_dual_epi<TX>><<<sell_grid(AT), kBlock, 0, s_>>>(
      AT, e.data(), ray_dual_epi<TX>{ls_.data(), us_.data(), dc_.data(), sn.data(), vn.data()},
      partials_.data());
    launches_ += 2;
    B200_LAUNCH_CHECK();
    const double br  = beta_ * gamma_;
    const double sum_ds = stat<false>(sn.data(), n);
    const double mdi    = stat<true>(vn.data(), n);
    sched_.max_primal_ray_inf = stat<true>(vm.data(), m);
    sched_.primal_ray_obj     = (nd > 0.0 ? sum_cd / nd : sum_cd) / br;
    const double sf = std::max(mdi, ne);
    sched_.max_dual_ray_inf = sf > 0.0 ? mdi / sf : 0.0;
    sched_.dual_ray_obj     = sf > 0.0 ? ((sum_ps + sum_ds) / br) / sf : 0.0;
  }

  // ------------------------------------------------------------------ main loop
  void loop(pdlp_result& r)
  {
    const int m = in_.m, n = in_.n;
    const double inf = std::numeric_limits<double>::infinity();
    // The schedule / restart state lives in sched_ so that an FP64 continuation resumes it.
    long& k            = sched_.k;
    long& since        = sched_.since;
    double& fpe        = sched_.fpe;
    double& fpe0       = sched_.fpe0;
    double& last_trial = sched_.last_trial;
    double& pid_sum    = sched_.pid_sum;
    double& pid_last   = sched_.pid_last;
    double& best_gap   = sched_.best_gap;
    if (sched_.fresh) set_scalars(0);
    sched_.fresh = false;
    const auto A = As_view(), AT = ATs_view();

    for (;;) {
      const bool major = (k % kMajor == 0 && k > 0) || k <= 0;
      const bool cond  = (k % conditional_major(k)) == 0;
      bool restarted   = false;
      if (major || cond) {
        close_cycle(k);
        const conv_info cv = evaluate();
        const int st       = decide(cv, k);
        if (st != kKeepGoing) return finish(r, st, cv, k);

        if (major) {
          // should_cupdlpx_restart (reference pdlp_restart_strategy.cu:689-754)
          bool restart = false;
          if (k == kMajor)
            restart = true;
          else if (k > kMajor) {
            if (fpe <= kSufficientReduction * fpe0)
              restart = true;
            else if (fpe <= kNecessaryReduction * fpe0 && fpe > last_trial)
              restart = true;
            else if ((double)since >= kArtificialRestart * (double)k)
              restart = true;
          }
          last_trial = fpe;
          if (restart) {
            // cupdlpx_restart + PID primal weight (reference pdlp_restart_strategy.cu:758-986)
            const double pd = reduce<1>(xa_.data(), xhat_.data(), n);
            const double dd = reduce<1>(ya_.data(), yhat_.data(), m);
            const double rel_dual   = cv.l2_dual / (1.0 + c_norm_);
            const double rel_primal = cv.l2_primal / (1.0 + b_norm_);
            const double lp = std::sqrt(pd), ld = std::sqrt(dd);
            const double ratio = rel_primal == 0.0 ? inf : rel_dual / rel_primal;
            if (lp > 1e-16 && ld > 1e-16 && lp < 1e12 && ld < 1e12 && ratio > 1e-8 &&
                ratio < 1e8) {
              const double err  = std::log(ld) - std::log(lp) - std::log(omega_);
              pid_sum           = pid_sum * kISmooth + err;
              const double derr = err - pid_last;
              omega_   = std::exp(kKp * err + kKi * pid_sum + kKd * derr) * omega_;
              pid_last = err;
            } else {
              omega_   = best_omega_;
              pid_sum  = 0.0;
              pid_last = 0.0;
            }
            const double rgap = std::fabs(std::log10(ratio));
            if (rgap < best_gap) {
              best_gap    = rgap;
              best_omega_ = omega_;
            }
            B200_CUDA_CHECK(cudaMemcpyAsync(x_.data(), xhat_.data(), n * sizeof(TX),
                                            cudaMemcpyDeviceToDevice, s_));
            B200_CUDA_CHECK(cudaMemcpyAsync(xa_.data(), xhat_.data(), n * sizeof(TX),
                                            cudaMemcpyDeviceToDevice, s_));
            B200_CUDA_CHECK(cudaMemcpyAsync(y_.data(), yhat_.data(), m * sizeof(TX),
                                            cudaMemcpyDeviceToDevice, s_));
            B200_CUDA_CHECK(cudaMemcpyAsync(ya_.data(), yhat_.data(), m * sizeof(TX),
                                            cudaMemcpyDeviceToDevice, s_));
            since      = 0;
            last_trial = inf;
            restarted  = true;
            ++restarts_;
            set_scalars(0);
          }
        }
      }

      const bool mstep = is_major_step(k);
      const bool fpe_it = ((k + 1) % kMajor == 0) || restarted;
      if (!mstep && !fpe_it) {
        long R = 1;
        while (R < 255) {
          const long kk = k + R;
          if (is_check(kk) || is_major_step(kk) || ((kk + 1) % kMajor == 0)) break;
          ++R;
        }
        run_plain(R, k);
        k += R;
        since += R;
        continue;
      }

      // A step that keeps x_hat / y_hat / slack (major) and/or measures the fixed-point error.
      if (fpe_it) {
        if (mstep) {
          launch_primal<true, false, true>(0);
          launch_dual<true, false, true>(0);
        } else {
          launch_primal<false, false, true>(0);
          launch_dual<false, false, true>(0);
        }
        finalize_sum_kernel<1><<<1, kBlock, 0, s_>>>(partials_.data(), sell_grid(A),
                                                     dres_.data() + 8);
        // compute_fixed_error (reference pdlp.cu:1749-1857)
        sell_map_kernel<TX, TX, fpe_epi<TX>><<<sell_grid(AT), kBlock, 0, s_>>>(
          AT, ybar_.data(), fpe_epi<TX>{aty_.data(), xbar_.data(), x_.data()}, partials_.data());
        finalize_sum_kernel<2><<<1, kBlock, 0, s_>>>(partials_.data(), sell_grid(AT),
                                                     dres_.data() + 9);
        // Infeasibility information from this step's deltas, for the checks at iterations 200
        // and 400 only (reference termination_strategy.cu:187-199).
        if (p_.detect_infeasibility && (k + 1) % kMajor == 0 && (k + 1) < 3 * kMajor)
          ray_statistics();
        halpern_kernel<TX><<<vgrid_, kBlock, 0, s_>>>(x_.data(), xbar_.data(), xa_.data(), n,
                                                      y_.data(), ybar_.data(), ya_.data(), m,
                                                      scalars_.data());
        advance_kernel<<<1, 1, 0, s_>>>(scalars_.data(), 1);
        launches_ += 5;
        B200_LAUNCH_CHECK();
        B200_CUDA_CHECK(cudaMemcpyAsync(hres_ + 8, dres_.data() + 8, 3 * sizeof(double),
                                        cudaMemcpyDeviceToHost, s_));
        B200_CUDA_CHECK(cudaStreamSynchronize(s_));
        const double ndy = hres_[8], inter = hres_[9], ndx = hres_[10];
        const double movement = ndx * omega_ + ndy / omega_;
        fpe = std::sqrt(movement + 2.0 * inter * eta_);
        if (restarted) fpe0 = fpe;
      } else {
        launch_primal<true, true, false>(0);
        launch_dual<true, true, false>(0);
        advance_kernel<<<1, 1, 0, s_>>>(scalars_.data(), 1);
        ++launches_;
        B200_LAUNCH_CHECK();
      }
      ++k;
      ++since;
    }
  }

  // Termination decision of the check at iteration k on its results cv (reference
  // check_termination_criteria_kernel, termination_strategy.cu:311-376): the status that ends the
  // loop (kStalled included), or kKeepGoing.
  static constexpr int kKeepGoing = -1000;
  int decide(const conv_info& cv, long k)
  {
    const bool pcr       = p_.per_constraint_residual;
    const bool primal_ok = pcr ? cv.linf_primal <= p_.abs_primal
                               : cv.l2_primal <= p_.abs_primal + p_.rel_primal * b_norm_;
    const bool dual_ok   = pcr ? cv.linf_dual <= p_.abs_dual
                               : cv.l2_dual <= p_.abs_dual + p_.rel_dual * c_norm_;
    int status           = kNoTermination;
    if (dual_ok && primal_ok && cv.gap <= p_.abs_gap + p_.rel_gap * cv.abs_obj)
      status = kOptimal;
    else if (primal_ok)
      status = kPrimalFeasible;
    if (p_.log_to_console && (k % 1000 == 0))
      std::printf("%7ld %+.8e %+.8e  %8.2e   %8.2e     %8.2e   %.3fs\n", k, cv.primal_obj,
                  cv.dual_obj, cv.gap, cv.l2_primal, cv.l2_dual, now_s() - t_start_);
    if (k > 1 && status == kOptimal) return kOptimal;
    // Stable3 returns any current infeasibility (never_restart_to_average, pdlp.cu:1089-1109).
    if (p_.detect_infeasibility && status == kNoTermination) {
      if (sched_.dual_ray_obj > 0.0 &&
          sched_.max_dual_ray_inf / sched_.dual_ray_obj <= p_.primal_infeasible_tol)
        return kPrimalInfeasible;
      if (sched_.primal_ray_obj < 0.0 &&
          sched_.max_primal_ray_inf / -sched_.primal_ray_obj <= p_.dual_infeasible_tol)
        return kDualInfeasible;
    }
    if (now_s() - t_start_ >= p_.time_limit) return kTimeLimit;
    if (k >= p_.iteration_limit) return kIterationLimit;
    if (!std::isfinite(cv.l2_primal) || !std::isfinite(cv.l2_dual)) return kNumericalError;
    if constexpr (std::is_same_v<TX, float>) {
      const double q = termination_distance(
        pcr ? cv.linf_primal : cv.l2_primal,
        pcr ? p_.abs_primal : p_.abs_primal + p_.rel_primal * b_norm_,
        pcr ? cv.linf_dual : cv.l2_dual, pcr ? p_.abs_dual : p_.abs_dual + p_.rel_dual * c_norm_,
        cv.gap, p_.abs_gap + p_.rel_gap * cv.abs_obj);
      if (q <= 0.5 * sched_.stall_ref) {
        sched_.stall_ref = q;
        sched_.stall_k   = k;
      } else if (k - sched_.stall_k >= kStallWindow)
        return kStalled;
    }
    return kKeepGoing;
  }

  // ------------------------------------------------------------------ state
  const lp_device_input& in_;
  const pdlp_params& p_;
  cudaStream_t s_ = nullptr;
  double *x_out_ = nullptr, *y_out_ = nullptr, *rc_out_ = nullptr;
  int sms_ = 148, vgrid_ = 592;
  double* hres_ = nullptr;
  double t_start_ = 0, t_loop_ = 0;

  device_layout L_;
  dbuf<TX> As_, ATs_;
  dbuf<double> c64_, l64_, u64_, lc64_, uc64_, dr_, dc_;
  dbuf<TX> cs_, ls_, us_, lcs_, ucs_;
  dbuf<TX> x_, xhat_, slack_, xbar_, xa_, aty_, y_, yhat_, ybar_, ya_;
  dbuf<double> xu_, yu_, su_;
  dbuf<double> partials_, dres_;
  dbuf<pdlp_scalars> scalars_;
  std::map<int, cudaGraphExec_t> graphs_;
  // Tiled sweeps (mixed precision): the tiled copies of A (dual sweep) and A^T (primal sweep), the
  // form each plain sweep uses, the groups' partial sums and the bounded-wait error flag.
  tile_matrix tA_, tAT_;
  bool tile_primal_ = false, tile_dual_ = false;
  dbuf<float> tpart_;
  dbuf<int> terr_;
  double tune_ms_[4] = {0, 0, 0, 0};
  // Persistent plain iterations: the launch's control block (barrier count, status), its grid,
  // the choice of form and its cache key.
  dbuf<persist_ctl> pctl_;
  bool cycle_open_ = false, cycle_one_time_ = false;
  int cycle_form_  = 0;
  long cycle_k0_   = 0;
  int persist_grid_      = 0;
  long persist_launches_ = 0;
  plain_form_tuner form_;
  form_key form_key_{};
  double form_us_[3] = {0, 0, 0};  // the timings behind the choice (this solve's or cached)
  size_t cluster_smem_ = 0;         // dynamic shared memory of the cluster form
  int cluster_blocks_  = 0;         // blocks of the cluster power iteration (0: not used)
  long cluster_launches_ = 0;
  // Warps per block of the plain sweeps and the timings they were chosen by.
  int wpb_primal_ = kWarpsPerBlock, wpb_dual_ = kWarpsPerBlock;
  double wpb_ms_[2][3] = {{0, 0, 0}, {0, 0, 0}};

  double obj_scale_ = 1.0, obj_offset_ = 0.0;
  double c_norm_ = 0, b_norm_ = 0, beta_ = 1, gamma_ = 1;
  loop_state sched_;
  double eta_ = 0, omega_ = 1, best_omega_ = 1;
  int power_iters_ = 0, restarts_ = 0;
  double launches_ = 0;

 public:
  // The plain sweeps split by row-length class: the long-row blocks and the slice blocks of each
  // sweep launched alone (8 warps per block), `iterations` times each after one warm-up.
  void profile_classes(sweep_profile& p, int iterations)
  {
    const auto A = As_view(), AT = ATs_view();
    persist_pe pe{x_.data(),   cs_.data(),   ls_.data(),    us_.data(),  xa_.data(),
                  xbar_.data(), x_.data(),   xhat_.data(),  slack_.data(), aty_.data(),
                  scalars_.data(), 0};
    persist_de de{y_.data(),    lcs_.data(), ucs_.data(),  ya_.data(),      ybar_.data(),
                  y_.data(),    yhat_.data(), scalars_.data(), 0};
    cudaEvent_t e0, e1;
    B200_CUDA_CHECK(cudaEventCreate(&e0));
    B200_CUDA_CHECK(cudaEventCreate(&e1));
    auto time_of = [&](auto&& launch) {
      launch();
      B200_CUDA_CHECK(cudaEventRecord(e0, s_));
      for (int i = 0; i < iterations; ++i) launch();
      B200_CUDA_CHECK(cudaEventRecord(e1, s_));
      B200_CUDA_CHECK(cudaEventSynchronize(e1));
      float ms = 0.f;
      B200_CUDA_CHECK(cudaEventElapsedTime(&ms, e0, e1));
      return (double)ms / iterations;
    };
    auto classes = [&](const dev_matrix& M, const dev_sell<TX>& V, auto&& launch, double* out) {
      int64_t long_nnz = 0;
      B200_CUDA_CHECK(cudaMemcpyAsync(&long_nnz, M.long_off.data() + M.n_long, sizeof(int64_t),
                                      cudaMemcpyDeviceToHost, s_));
      B200_CUDA_CHECK(cudaStreamSynchronize(s_));
      const int lb = long_blocks(V.long_count()), g = sell_grid(V);
      out[0] = M.n_long;
      out[1] = (double)long_nnz;
      out[2] = lb > 0 ? time_of([&] { launch(lb, 0); }) : 0.0;
      out[3] = M.rows - M.n_long;
      out[4] = (double)(L_.nnz - long_nnz);
      out[5] = (double)(M.stored() - (long_nnz + kChunk - 1) / kChunk * kChunk);
      out[6] = g > lb ? time_of([&] { launch(g - lb, lb); }) : 0.0;
    };
    classes(L_.AT, AT, [&](int grid, int vb0) {
      sell_map_range_kernel<TX, TX, persist_pe><<<grid, kBlock, 0, s_>>>(AT, y_.data(), pe,
                                                                         partials_.data(), vb0);
    }, p.classes[0]);
    classes(L_.A, A, [&](int grid, int vb0) {
      sell_map_range_kernel<TX, TX, persist_de><<<grid, kBlock, 0, s_>>>(A, xbar_.data(), de,
                                                                         partials_.data(), vb0);
    }, p.classes[1]);
    B200_LAUNCH_CHECK();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }

  // Times plain iterations sweep by sweep (measurement hook).
  sweep_profile profile(int iterations)
  {
    alloc_scope scope(s_);
    t_start_ = now_s();
    setup();
    set_scalars(0);
    const int m = in_.m, n = in_.n;
    const auto A = As_view(), AT = ATs_view();
    std::vector<cudaEvent_t> ev(3 * iterations);
    for (auto& e : ev) B200_CUDA_CHECK(cudaEventCreate(&e));
    for (int i = 0; i < 3; ++i) plain_iterations(1);  // warm-up
    for (int i = 0; i < iterations; ++i) {
      B200_CUDA_CHECK(cudaEventRecord(ev[3 * i], s_));
      plain_primal(0);
      B200_CUDA_CHECK(cudaEventRecord(ev[3 * i + 1], s_));
      plain_dual(0);
      B200_CUDA_CHECK(cudaEventRecord(ev[3 * i + 2], s_));
      advance_kernel<<<1, 1, 0, s_>>>(scalars_.data(), 1);
    }
    B200_CUDA_CHECK(cudaStreamSynchronize(s_));
    sweep_profile p;
    for (int i = 0; i < iterations; ++i) {
      float a = 0, b = 0;
      B200_CUDA_CHECK(cudaEventElapsedTime(&a, ev[3 * i], ev[3 * i + 1]));
      B200_CUDA_CHECK(cudaEventElapsedTime(&b, ev[3 * i + 1], ev[3 * i + 2]));
      p.ms_primal += a;
      p.ms_dual += b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    p.ms_primal /= iterations;
    p.ms_dual /= iterations;
    profile_classes(p, iterations);
    // Algorithmic bytes (CSR accounting): matrix values + indices, row offsets, one gather pass,
    // epilogue vectors (primal: read x c l u x_anchor, write x_bar x; dual: read y lc uc y_anchor,
    // write y).
    const double nnz = (double)L_.nnz, sv = sizeof(TX), sf = sizeof(TX);
    p.bytes_primal = nnz * (sv + 4) + (n + 1) * 4.0 + m * sf + 7.0 * n * sf;
    p.bytes_dual   = nnz * (sv + 4) + (m + 1) * 4.0 + n * sf + 5.0 * m * sf;
    (void)A;
    (void)AT;
    return p;
  }
};

#include "climber_engine.cuh"

}  // namespace

pdlp_result pdlp_solve_device(const lp_device_input& in, const pdlp_params& p, cudaStream_t stream,
                              double* x_out, double* y_out, double* rc_out)
{
  joined_stream js(stream);
  if (p.precision == 1) {
    engine<float> e(in, p, js.own);
    pdlp_result r = e.run(x_out, y_out, rc_out);
    const bool stalled = r.status == kStalled;
    if (!stalled && (p.refinement_passes <= 0 || r.status != kOptimal)) return r;
    // FP64 continuation: to the refinement tolerance when one is asked for, else (a stalled mixed
    // solve) to the solve's own tolerances.  It resumes the iteration count, so the limits stay
    // those of the solve.
    pdlp_params q = p;
    if (p.refinement_passes > 0) {
      q.abs_primal = q.rel_primal = p.refinement_tol;
      q.abs_dual = q.rel_dual = p.refinement_tol;
      q.abs_gap = q.rel_gap = p.refinement_tol;
    }
    engine<double> d(in, q, js.own);
    return d.continue_from(e, x_out, y_out, rc_out);
  }
  engine<double> e(in, p, js.own);
  return e.run(x_out, y_out, rc_out);
}

std::vector<pdlp_result> pdlp_climber_solve_device(const lp_device_input& in, const pdlp_params& p,
                                                   const std::vector<int>& var,
                                                   const std::vector<double>& lo,
                                                   const std::vector<double>& up,
                                                   cudaStream_t stream, double* x_out,
                                                   double* y_out, double* rc_out)
{
  joined_stream js(stream);
  engine<double> base(in, p, js.own);
  base.prepare();
  climber_engine ce(base, p, var, lo, up);
  return ce.run(x_out, y_out, rc_out);
}

sweep_profile pdlp_profile_sweeps(const lp_device_input& in, const pdlp_params& p,
                                  cudaStream_t stream, int iterations)
{
  joined_stream js(stream);
  if (p.precision == 1) {
    engine<float> e(in, p, js.own);
    return e.profile(iterations);
  }
  engine<double> e(in, p, js.own);
  return e.profile(iterations);
}

device_solution::~device_solution()
{
  if (!base) return;
  int cur = -1;
  cudaGetDevice(&cur);
  if (cur != device) cudaSetDevice(device);
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess) {
    cudaFreeAsync(base, s);
    cudaStreamDestroy(s);
  }
  if (cur >= 0 && cur != device) cudaSetDevice(cur);
  cudaGetLastError();
}

namespace {
// Makes d's device current for the lifetime of the object.
struct on_device {
  int prev = -1, dev;
  explicit on_device(int d) : dev(d)
  {
    cudaGetDevice(&prev);
    if (prev != dev) B200_CUDA_CHECK(cudaSetDevice(dev));
  }
  ~on_device()
  {
    if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  }
};
// A non-blocking stream for the lifetime of the object (synchronised before it is destroyed).
struct temp_stream {
  cudaStream_t s = nullptr;
  temp_stream() { B200_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
  ~temp_stream()
  {
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
  }
};
}  // namespace

void ensure_host(pdlp_result& r)
{
  if (!r.dev) return;
  const device_solution& d = *r.dev;
  on_device scope(d.device);
  temp_stream ts;
  r.x.resize(d.n);
  r.y.resize(d.m);
  r.rc.resize(d.n);
  staged_download(r.x.data(), d.x, (size_t)d.n * sizeof(double), ts.s);
  staged_download(r.y.data(), d.y, (size_t)d.m * sizeof(double), ts.s);
  staged_download(r.rc.data(), d.rc, (size_t)d.n * sizeof(double), ts.s);
  r.dev.reset();
}

void copy_solution_vector(const pdlp_result& r, int which, double* dst)
{
  const device_solution& d = *r.dev;
  const double* src  = which == 0 ? d.x : which == 1 ? d.y : d.rc;
  const size_t bytes = (size_t)(which == 1 ? d.m : d.n) * sizeof(double);
  if (bytes == 0) return;
  on_device scope(d.device);
  cudaPointerAttributes attr{};
  const bool dma = cudaPointerGetAttributes(&attr, dst) == cudaSuccess &&
                   attr.type != cudaMemoryTypeUnregistered;
  cudaGetLastError();
  if (dma) {  // pinned host or device memory: one copy
    B200_CUDA_CHECK(cudaMemcpy(dst, src, bytes, cudaMemcpyDefault));
    return;
  }
  temp_stream ts;
  staged_download(dst, src, bytes, ts.s);
}

pdlp_result pdlp_solve(const lp_input& in, const pdlp_params& p)
{
  // Declared before the stream guard, so that on an early exit the stream's work has ended (the
  // guard synchronises) before the solution's memory is released.
  auto sol = std::make_shared<device_solution>();
  cudaStream_t s;
  B200_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  struct stream_guard {  // the stream's work ends before its buffers are released
    cudaStream_t s;
    ~stream_guard()
    {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  } guard{s};
  alloc_scope scope(s);
  configure_pool_once();
  const int m = in.m, n = in.n;
  const int64_t nnz = in.row_off[m];
  // A device copy made at problem creation (same device) replaces the upload of its arrays.
  const device_problem* dv = in.dev;
  if (dv) {
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != dv->device) dv = nullptr;
  }
  dbuf<int> off, idx;
  dbuf<double> val, c, lo, up, vl, vu, ip, id;
  // The solution stays on the device (one allocation for x, reduced costs and y).
  B200_CUDA_CHECK(cudaGetDevice(&sol->device));
  sol->n = n;
  sol->m = m;
  B200_CUDA_CHECK(cudaMallocAsync(&sol->base, (2 * (size_t)n + m) * sizeof(double), s));
  sol->x  = static_cast<double*>(sol->base);
  sol->rc = sol->x + n;
  sol->y  = sol->rc + n;
  lp_device_input d;
  {
    staged_upload h2d(s);
    auto put = [&](auto& buf, const auto* host, const auto* mirrored, int64_t count) {
      if (mirrored) return mirrored;
      buf.resize((size_t)std::max<int64_t>(count, 1));
      h2d.put(buf.data(), host, (size_t)count);
      return static_cast<decltype(mirrored)>(buf.data());
    };
    d.row_off = put(off, in.row_off, dv ? dv->row_off : nullptr, m + 1);
    d.col_idx = put(idx, in.col_idx, dv ? dv->col_idx : nullptr, nnz);
    d.val     = put(val, in.val, dv ? dv->val : nullptr, nnz);
    d.c       = put(c, in.c, dv ? dv->c : nullptr, n);
    d.con_lo  = put(lo, in.con_lo, dv ? dv->con_lo : nullptr, m);
    d.con_up  = put(up, in.con_up, dv ? dv->con_up : nullptr, m);
    d.var_lo  = put(vl, in.var_lo, dv ? dv->var_lo : nullptr, n);
    d.var_up  = put(vu, in.var_up, dv ? dv->var_up : nullptr, n);
    h2d.finish();
  }
  d.m          = m;
  d.n          = n;
  d.obj_offset = in.obj_offset;
  d.maximize   = in.maximize;
  if ((int)p.initial_primal.size() == n) {
    ip.resize(n);
    ip.upload(p.initial_primal.data(), n, s);
    d.initial_primal = ip.data();
  }
  if ((int)p.initial_dual.size() == m) {
    id.resize(m);
    id.upload(p.initial_dual.data(), m, s);
    d.initial_dual = id.data();
  }
  trace("host path: upload");
  pdlp_result r = pdlp_solve_device(d, p, s, sol->x, sol->y, sol->rc);
  B200_CUDA_CHECK(cudaStreamSynchronize(s));
  trace("host path: device solve");
  if (r.status != kNumericalError || r.iterations > 0) r.dev = std::move(sol);
  return r;
}

}  // namespace cuopt_b200
