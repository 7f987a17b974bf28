// Stable3 constants and the iteration schedule shared by the single-LP and the batch engines.
#pragma once

namespace cuopt_b200 {

constexpr int kOptimal = 1, kIterationLimit = 4, kTimeLimit = 5, kNumericalError = 6,
              kPrimalFeasible = 7, kNoTermination = 0, kPrimalInfeasible = 2, kDualInfeasible = 3;

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

}  // namespace cuopt_b200
