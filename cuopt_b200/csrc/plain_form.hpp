// Choice between the forms of a run of plain PDHG iterations (iterations that need neither a
// termination test, a major step nor a fixed-point error):
//   form 0: replays of cached CUDA graphs of 2^k iterations (two sweep kernels per iteration);
//   form 1: one cooperative launch of the persistent kernel (persistent_plain_kernel), with a grid
//           barrier after every sweep;
//   form 2: one launch of a thread-block cluster that keeps the gathered vectors in the shared
//           memory of each of its blocks (cluster_plain_kernel, small LPs only), with a cluster
//           barrier after every sweep.
// All forms run the same per-row arithmetic, so the iterates do not depend on the choice, and the
// choice can be made online: with pdlp_persistent_iterations = -1 the first cycles of a solve (a
// cycle: the iterations from one termination check to the next, with their major steps and every
// launch boundary) rotate through the available forms, each timed with CUDA events on the solve's
// stream, and once each has kSamples timed cycles the one with the lowest median time per iteration
// is kept.  A cycle that included one-time work (a graph captured and instantiated, the first
// launch of a kernel) is not counted.
#pragma once

#include "common.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

namespace cuopt_b200 {

class plain_form_tuner {
 public:
  static constexpr int kForms   = 3;
  static constexpr int kSamples = 4;

  plain_form_tuner() = default;
  plain_form_tuner(const plain_form_tuner&)            = delete;
  plain_form_tuner& operator=(const plain_form_tuner&) = delete;
  ~plain_form_tuner()
  {
    for (auto& p : pending_) {
      cudaEventDestroy(p.e0);
      cudaEventDestroy(p.e1);
    }
    for (auto& p : spare_) {
      cudaEventDestroy(p.e0);
      cudaEventDestroy(p.e1);
    }
  }

  // mode: -1 tune among the available forms, or the form to use (0, 1, 2; an unavailable one
  // falls back to 0).  `known` >= 0 is a form chosen before for the same work (kept without
  // timing).  `available[f]` tells whether form f can run on this problem and device.
  void reset(int mode, int known, const bool (&available)[kForms])
  {
    collect_all_dropped();
    for (auto& u : us_) u.clear();
    for (int f = 0; f < kForms; ++f) avail_[f] = f == 0 || available[f];
    turn_ = 0;
    if (mode >= 0)
      chosen_ = mode < kForms && avail_[mode] ? mode : 0;
    else if (known >= 0 && known < kForms && avail_[known])
      chosen_ = known;
    else if (count_available() == 1)
      chosen_ = 0;
    else
      chosen_ = -1;  // tuning
  }

  bool decided() const { return chosen_ >= 0; }
  int chosen() const { return chosen_; }
  bool available(int f) const { return f >= 0 && f < kForms && avail_[f]; }
  // The form of the next cycle.
  int next() const { return decided() ? chosen_ : turn_; }

  // Brackets one cycle (only while tuning).
  void begin(cudaStream_t s)
  {
    if (decided()) return;
    cur_ = take();
    B200_CUDA_CHECK(cudaEventRecord(cur_.e0, s));
  }
  // `one_time`: the cycle included work that later cycles of the form will not repeat; it is not
  // counted, and the same form runs again next.
  void end(cudaStream_t s, int form, long iters, bool one_time)
  {
    if (decided()) return;
    cur_.form     = form;
    cur_.iters    = iters;
    cur_.one_time = one_time;
    B200_CUDA_CHECK(cudaEventRecord(cur_.e1, s));
    pending_.push_back(cur_);
    if (!one_time) advance_turn();
  }

  // Folds the cycles whose closing event has completed into the samples (in launch order; the
  // others stay pending) and decides once every available form has enough samples.
  void collect()
  {
    size_t done = 0;
    for (; done < pending_.size(); ++done) {
      run& p                 = pending_[done];
      const cudaError_t qerr = cudaEventQuery(p.e1);
      if (qerr == cudaErrorNotReady) break;
      B200_CUDA_CHECK(qerr);
      if (!p.one_time && p.iters > 0) {
        float ms = 0.f;
        B200_CUDA_CHECK(cudaEventElapsedTime(&ms, p.e0, p.e1));
        us_[p.form].push_back(1e3 * (double)ms / (double)p.iters);
      }
      spare_.push_back(p);
    }
    pending_.erase(pending_.begin(), pending_.begin() + done);
    if (decided()) return;
    for (int f = 0; f < kForms; ++f)
      if (avail_[f] && (int)us_[f].size() < kSamples) return;
    int best = 0;
    for (int f = 1; f < kForms; ++f)
      if (avail_[f] && us_per_iteration(f) < us_per_iteration(best)) best = f;
    chosen_ = best;
  }

  // Median time per iteration of a form over its counted cycles (0 when it was not timed).
  double us_per_iteration(int form) const
  {
    std::vector<double> v = us_[form];
    if (v.empty()) return 0.0;
    std::sort(v.begin(), v.end());
    const size_t h = v.size() / 2;
    return v.size() % 2 ? v[h] : 0.5 * (v[h - 1] + v[h]);
  }

 private:
  struct run {
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int form      = 0;
    long iters    = 0;
    bool one_time = false;
  };
  int count_available() const
  {
    int c = 0;
    for (bool a : avail_) c += a;
    return c;
  }
  void advance_turn()
  {
    for (int k = 1; k <= kForms; ++k) {
      const int f = (turn_ + k) % kForms;
      if (avail_[f]) {
        turn_ = f;
        return;
      }
    }
  }
  run take()
  {
    if (!spare_.empty()) {
      run r = spare_.back();
      spare_.pop_back();
      return r;
    }
    run r;
    B200_CUDA_CHECK(cudaEventCreate(&r.e0));
    B200_CUDA_CHECK(cudaEventCreate(&r.e1));
    return r;
  }
  void collect_all_dropped()
  {
    for (auto& p : pending_) spare_.push_back(p);
    pending_.clear();
  }

  std::vector<run> pending_, spare_;
  run cur_;
  std::vector<double> us_[kForms];  // microseconds per iteration of each counted cycle, per form
  bool avail_[kForms] = {true, false, false};
  int turn_           = 0;
  int chosen_         = 0;  // graphs until reset() is called
};

}  // namespace cuopt_b200
