// host_stats.hpp -- FP64 tally statistics and convergence policies (host side).
//
// Mirrors mcSCRAM src/mc/stats/ci_utils.h (point estimates, confidence
// intervals, sample-size formulas), src/mc/stats/tally.h (the tally record),
// src/mc/stats/info_gain.h (Beta-posterior information gain) and
// src/mc/scheduler/convergence_policy.h (Wald and Jeffreys-Bayes updates).
// The reference takes the Beta quantile and digamma from Boost.Math; this
// file has its own implementations (see beta_quantile / digamma below),
// which only influence when the pass loop stops, never the tallies.
#pragma once
#include <array>
#include <cstddef>
#include <cstdint>

namespace mcg {
namespace host {
namespace stats {

constexpr double kDeltaEpsilon = 1.0e-12;  // ci_utils.h DELTA_EPSILON
constexpr double kZ95 = 1.959963984540054;
constexpr double kZ99 = 2.5758293035489004;

// z with P(|Z| <= z) = confidence (ci_utils.h:30-92).
double normal_quantile_two_sided(double confidence);
double normal_cdf(double z);

std::size_t required_trials(double p, double eps, double confidence);
std::size_t required_trials_from_normal_quantile_two_sided(double p, double eps, double z);
std::size_t required_trials_log10_from_normal_quantile_two_sided(double p, double eps_log10, double z);
double epsilon_from_trials(double p, std::size_t n, double z);

// Quantile of Beta(a, b) at probability q in (0, 1).
double beta_quantile(double a, double b, double q);
// Regularised incomplete beta I_x(a, b).
double beta_cdf(double a, double b, double x);
double digamma(double x);

struct convergence_result {
    double epsilon = 0.0;
    double target_epsilon = 0.0;
    std::size_t target_trials = 0;
};

class info_gain {
  public:
    explicit info_gain(double alpha0 = 0.5, double beta0 = 0.5) : alpha_(alpha0), beta_(beta0) {}
    double add_batch(std::size_t successes, std::size_t failures);
    double alpha() const { return alpha_; }
    double beta() const { return beta_; }
    double cumulative_bits() const { return cumulative_bits_; }
    double last_bits() const { return last_bits_; }

  private:
    double alpha_, beta_;
    double cumulative_bits_ = 0.0;
    double last_bits_ = 0.0;
};

double beta_entropy_bits(double alpha, double beta);

struct tally {
    std::size_t num_one_bits = 0;
    std::size_t total_bits = 0;
    double mean = 0.0;
    double std_err = 0.0;
    std::array<double, 4> ci = {0., 0., 0., 0.};  // lower95, upper95, lower99, upper99
    convergence_result linear{};
    convergence_result log10{};
    info_gain gain{};

    double half_width(double z) const { return std_err * z; }
    static tally &compute_moments(tally &t);
    static tally &compute_ci(tally &t);
    tally &update(std::size_t ones, std::size_t all);
};

double half_width_log10(const tally &t, double z);

enum class policy { bayes, wald };

void update_wald(tally &t, double rel_margin_error, double z);
void update_bayes(tally &t, double rel_margin_error, double z);
inline void update_convergence(policy p, tally &t, double rel_margin_error, double z) {
    if (p == policy::wald) update_wald(t, rel_margin_error, z);
    else update_bayes(t, rel_margin_error, z);
}

}  // namespace stats
}  // namespace host
}  // namespace mcg
