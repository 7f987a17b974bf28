// Stable3 constants and the iteration schedule shared by the single-LP and the batch engines.
#pragma once

#include <algorithm>
#include <cmath>
#include <memory>
#include <mutex>
#include <random>
#include <vector>

namespace cuopt_b200 {

constexpr int kOptimal = 1, kIterationLimit = 4, kTimeLimit = 5, kNumericalError = 6,
              kPrimalFeasible = 7, kNoTermination = 0, kPrimalInfeasible = 2, kDualInfeasible = 3;

// Mixed precision only (never returned to callers): the FP32 iterates stopped making progress, so
// the solve continues in FP64.  A mixed solve counts as stalled when its distance to termination
// (the largest of primal residual, dual residual and gap, each divided by its threshold) has not
// halved during the last kStallWindow iterations.
constexpr int kStalled     = -1;
constexpr long kStallWindow = 1000;

// Distance to termination of a check: >= 1 until the tolerances hold.
inline double termination_distance(double primal, double primal_thr, double dual, double dual_thr,
                                   double gap, double gap_thr)
{
  const double q = primal / primal_thr;
  return std::fmax(q, std::fmax(dual / dual_thr, gap / gap_thr));
}

// Stable3 constants (reference solve.cu:167-209, pdlp_hyper_params.cuh:12-56,
// pdlp_restart_strategy.cu:689-836, pdlp.cu:2620-2731).
constexpr long kMajor                 = 200;
constexpr double kArtificialRestart   = 0.36;
constexpr double kSufficientReduction = 0.2;
constexpr double kNecessaryReduction  = 0.8;
constexpr double kKp = 0.99, kKi = 0.01, kKd = 0.0, kISmooth = 0.3;
constexpr int kPowerMaxIters          = 5000;
constexpr double kPowerTol            = 1e-4;
constexpr double kStepScaling         = 0.998;
constexpr int kRuizIterations         = 10;
constexpr double kPcAlpha             = 1.0;

inline long conditional_major(long k)  // reference utils.cuh:63-81
{
  long step = 10, threshold = 1000;
  while (k >= threshold) {
    step *= 10;
    threshold *= 10;
  }
  return step;
}

inline bool is_check(long k) { return (k % kMajor == 0 && k > 0) || k <= 0 || k % conditional_major(k) == 0; }
inline bool is_major_step(long k) { return ((k + 1) % kMajor == 0) || ((k + 2) % conditional_major(k + 2)) == 0; }

// sigma_max^2 of the (k+1) x k lower bidiagonal matrix with diagonal a[0..k-1] and subdiagonal
// b[0..k-1]: the largest eigenvalue of the tridiagonal B^T B, by Sturm-sequence bisection.
inline double largest_bidiagonal_sigma2(const double* a, const double* b, int k)
{
  if (k <= 0) return 0.0;
  std::vector<double> d(k), e(std::max(k - 1, 0));
  for (int j = 0; j < k; ++j) d[j] = a[j] * a[j] + b[j] * b[j];
  for (int j = 0; j + 1 < k; ++j) e[j] = a[j + 1] * b[j];
  double hi = 0.0;
  for (int j = 0; j < k; ++j)
    hi = std::max(hi, d[j] + (j > 0 ? std::fabs(e[j - 1]) : 0.0) + (j + 1 < k ? std::fabs(e[j]) : 0.0));
  double lo = 0.0;
  // count of eigenvalues below x (Sturm sequence of T - x I)
  auto below = [&](double x) {
    int cnt  = 0;
    double q = d[0] - x;
    if (q < 0) ++cnt;
    for (int j = 1; j < k; ++j) {
      const double prevq = q != 0.0 ? q : 1e-300;
      q = d[j] - x - e[j - 1] * e[j - 1] / prevq;
      if (q < 0) ++cnt;
    }
    return cnt;
  };
  for (int it = 0; it < 200 && hi - lo > 1e-15 * hi; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (below(mid) >= k)
      hi = mid;
    else
      lo = mid;
  }
  return hi;
}

// Start vector of the step-size iterations: normals of std::mt19937(1) (reference
// pdlp.cu:2632-2638).  The sequence does not depend on the LP, so its values are generated once
// per process and shared; a solve (or batch instance) with m rows takes the first m.
inline std::shared_ptr<const std::vector<double>> power_start_sequence(size_t count)
{
  static std::mutex mu;
  static std::shared_ptr<const std::vector<double>> cached;
  std::lock_guard<std::mutex> lock(mu);
  if (!cached || cached->size() < count) {
    auto v = std::make_shared<std::vector<double>>(count);
    std::mt19937 gen(1);
    std::normal_distribution<double> dist(0.0, 1.0);
    for (auto& x : *v) x = dist(gen);
    cached = std::move(v);
  }
  return cached;
}

// Stopping rule of the Golub-Kahan-Lanczos step size: steps run in chunks of kLanczosChunk; after
// each chunk sigma_max^2 of the bidiagonal so far is compared with the previous chunk's value.
// The estimate approaches sigma_max from below, so the step 0.998 / sigma keeps a margin of 2e-3
// over the stability limit; a relative change of 1e-8 leaves it untouched (on the 1M x 2M LP the
// step agrees with that of 1e-10 to ten digits, in 64 steps instead of 80).
constexpr int kLanczosChunk = 16, kLanczosMaxSteps = 512;
constexpr double kLanczosTol = 1e-8;

}  // namespace cuopt_b200
