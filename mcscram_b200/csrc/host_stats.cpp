// host_stats.cpp -- FP64 statistics for the convergence loop.
#include "host_stats.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

namespace mcg {
namespace host {
namespace stats {

// Inverse normal CDF by P. J. Acklam's rational approximation (2003), the
// method the reference uses (src/mc/stats/ci_utils.h:30-92); the published
// coefficients must be the same for z to be the same.
double normal_quantile_two_sided(double confidence) {
    const double p = std::clamp(confidence, kDeltaEpsilon, 1.0 - kDeltaEpsilon);
    const double q = 1.0 - (1.0 - p) / 2.0;
    static const double a[6] = {-3.969683028665376e+01, 2.209460984245205e+02, -2.759285104469687e+02,
                                1.383577518672690e+02,  -3.066479806614716e+01, 2.506628277459239e+00};
    static const double b[5] = {-5.447609879822406e+01, 1.615858368580409e+02, -1.556989798598866e+02,
                                6.680131188771972e+01,  -1.328068155288572e+01};
    static const double c[6] = {-7.784894002430293e-03, -3.223964580411365e-01, -2.400758277161838e+00,
                                -2.549732539343734e+00, 4.374664141464968e+00,  2.938163982698783e+00};
    static const double d[4] = {7.784695709041462e-03, 3.224671290700398e-01, 2.445134137142996e+00,
                                3.754408661907416e+00};
    const double lo = 0.02425, hi = 1.0 - lo;
    auto tail = [&](double u) {
        return (((((c[0] * u + c[1]) * u + c[2]) * u + c[3]) * u + c[4]) * u + c[5]) /
               ((((d[0] * u + d[1]) * u + d[2]) * u + d[3]) * u + 1.0);
    };
    if (q < lo) return tail(std::sqrt(-2.0 * std::log(q)));
    if (q > hi) return -tail(std::sqrt(-2.0 * std::log(1.0 - q)));
    const double u = q - 0.5, t = u * u;
    return (((((a[0] * t + a[1]) * t + a[2]) * t + a[3]) * t + a[4]) * t + a[5]) * u /
           (((((b[0] * t + b[1]) * t + b[2]) * t + b[3]) * t + b[4]) * t + 1.0);
}

double normal_cdf(double z) { return 0.5 * std::erfc(-z / std::sqrt(2.0)); }

std::size_t required_trials(double p, double eps, double confidence) {
    return required_trials_from_normal_quantile_two_sided(p, eps, normal_quantile_two_sided(confidence));
}

std::size_t required_trials_from_normal_quantile_two_sided(double p, double eps, double z) {
    return (std::size_t)std::ceil((z * z * p * (1.0 - p)) / (eps * eps));
}

std::size_t required_trials_log10_from_normal_quantile_two_sided(double p, double eps_log10, double z) {
    const double ln10 = std::log(10.0);
    const double denom = p * eps_log10 * eps_log10 * ln10 * ln10;
    return (std::size_t)std::ceil(z * z * (1.0 - p) / denom);
}

double epsilon_from_trials(double p, std::size_t n, double z) {
    if (n == 0) return std::numeric_limits<double>::infinity();
    return z * std::sqrt(p * (1.0 - p) / (double)n);
}

double half_width_log10(const tally &t, double z) {
    const double p = std::max(t.mean, kDeltaEpsilon);
    return z * t.std_err / (p * std::log(10.0));
}

// ---------------------------------------------------------------- special functions

// Digamma: recurrence up to x >= 8, then the asymptotic (Bernoulli) series.
double digamma(double x) {
    double r = 0.0;
    while (x < 8.0) {
        r -= 1.0 / x;
        x += 1.0;
    }
    const double f = 1.0 / (x * x);
    const double series = f * (1.0 / 12 - f * (1.0 / 120 - f * (1.0 / 252 - f * (1.0 / 240 - f * (1.0 / 132)))));
    return r + std::log(x) - 0.5 / x - series;
}

namespace {

// Continued fraction of the incomplete beta (modified Lentz).
double beta_cf(double a, double b, double x) {
    const double tiny = 1e-300;
    double qab = a + b, qap = a + 1.0, qam = a - 1.0;
    double c = 1.0, d = 1.0 - qab * x / qap;
    if (std::fabs(d) < tiny) d = tiny;
    d = 1.0 / d;
    double h = d;
    for (int m = 1; m <= 200000; ++m) {
        const double m2 = 2.0 * m;
        double aa = m * (b - m) * x / ((qam + m2) * (a + m2));
        d = 1.0 + aa * d;
        if (std::fabs(d) < tiny) d = tiny;
        c = 1.0 + aa / c;
        if (std::fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        h *= d * c;
        aa = -(a + m) * (qab + m) * x / ((a + m2) * (qap + m2));
        d = 1.0 + aa * d;
        if (std::fabs(d) < tiny) d = tiny;
        c = 1.0 + aa / c;
        if (std::fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < 1e-15) break;
    }
    return h;
}

double log_beta_fn(double a, double b) { return std::lgamma(a) + std::lgamma(b) - std::lgamma(a + b); }

// Regularised lower incomplete gamma P(a, x).
double gamma_p(double a, double x) {
    if (x <= 0) return 0.0;
    const double lg = std::lgamma(a);
    if (x < a + 1.0) {
        double ap = a, sum = 1.0 / a, del = sum;
        for (int n = 0; n < 100000; ++n) {
            ap += 1.0;
            del *= x / ap;
            sum += del;
            if (std::fabs(del) < std::fabs(sum) * 1e-16) break;
        }
        return sum * std::exp(-x + a * std::log(x) - lg);
    }
    const double tiny = 1e-300;
    double b = x + 1.0 - a, c = 1.0 / tiny, d = 1.0 / b, h = d;
    for (int i = 1; i < 100000; ++i) {
        const double an = -i * (i - a);
        b += 2.0;
        d = an * d + b;
        if (std::fabs(d) < tiny) d = tiny;
        c = b + an / c;
        if (std::fabs(c) < tiny) c = tiny;
        d = 1.0 / d;
        const double del = d * c;
        h *= del;
        if (std::fabs(del - 1.0) < 1e-16) break;
    }
    return 1.0 - std::exp(-x + a * std::log(x) - lg) * h;
}

double gamma_quantile(double a, double q) {
    double lo = 0.0, hi = std::max(1.0, a);
    while (gamma_p(a, hi) < q) hi *= 2.0;
    for (int i = 0; i < 200; ++i) {
        const double mid = 0.5 * (lo + hi);
        if (gamma_p(a, mid) < q) lo = mid;
        else hi = mid;
        if (hi - lo <= 1e-15 * hi) break;
    }
    return 0.5 * (lo + hi);
}

}  // namespace

double beta_cdf(double a, double b, double x) {
    if (x <= 0.0) return 0.0;
    if (x >= 1.0) return 1.0;
    const double lbt = a * std::log(x) + b * std::log1p(-x) - log_beta_fn(a, b);
    if (x < (a + 1.0) / (a + b + 2.0)) return std::exp(lbt) * beta_cf(a, b, x) / a;
    return 1.0 - std::exp(lbt) * beta_cf(b, a, 1.0 - x) / b;
}

// Beta(a, b) quantile.  Three regimes:
//  * both shapes large (min >= 1000): normal approximation with the
//    first-order Cornish-Fisher skewness term;
//  * one shape much larger than the other (max >= 1e5): the small side is a
//    Gamma variable scaled by a + b (Beta(a, b) -> Gamma(a) / (a + b));
//  * otherwise: bisection on the incomplete beta continued fraction.
double beta_quantile(double a, double b, double q) {
    if (q <= 0.0) return 0.0;
    if (q >= 1.0) return 1.0;
    const double n = a + b;
    if (std::min(a, b) >= 1000.0) {
        const double mu = a / n;
        const double sd = std::sqrt(a * b / (n * n * (n + 1.0)));
        const double skew = 2.0 * (b - a) * std::sqrt(n + 1.0) / ((n + 2.0) * std::sqrt(a * b));
        // z of the one-sided quantile q
        const double z = (q < 0.5 ? -1.0 : 1.0) * normal_quantile_two_sided(std::fabs(2.0 * q - 1.0));
        return std::clamp(mu + sd * (z + (z * z - 1.0) * skew / 6.0), 0.0, 1.0);
    }
    if (std::max(a, b) >= 1e5) {
        if (a <= b) return std::clamp(gamma_quantile(a, q) / n, 0.0, 1.0);
        return std::clamp(1.0 - gamma_quantile(b, 1.0 - q) / n, 0.0, 1.0);
    }
    double lo = 0.0, hi = 1.0;
    for (int i = 0; i < 200; ++i) {
        const double mid = 0.5 * (lo + hi);
        if (beta_cdf(a, b, mid) < q) lo = mid;
        else hi = mid;
        if (hi - lo <= 1e-15 * std::max(hi, 1e-300)) break;
    }
    return 0.5 * (lo + hi);
}

double beta_entropy_bits(double alpha, double beta) {
    const double nats = log_beta_fn(alpha, beta) - (alpha - 1.0) * digamma(alpha) - (beta - 1.0) * digamma(beta) +
                        (alpha + beta - 2.0) * digamma(alpha + beta);
    return nats / 0.693147180559945309417232121458176568;
}

double info_gain::add_batch(std::size_t successes, std::size_t failures) {
    const double ap = alpha_, bp = beta_;
    alpha_ += (double)successes;
    beta_ += (double)failures;
    last_bits_ = beta_entropy_bits(ap, bp) - beta_entropy_bits(alpha_, beta_);
    cumulative_bits_ += last_bits_;
    return last_bits_;
}

// ---------------------------------------------------------------- tally

tally &tally::compute_moments(tally &t) {
    const double total = (double)t.total_bits;
    t.mean = total ? (double)t.num_one_bits / total : 0.0;
    t.std_err = total ? std::sqrt(t.mean * (1.0 - t.mean) / total) : 0.0;
    return t;
}

tally &tally::compute_ci(tally &t) {
    const double hw95 = t.half_width(kZ95), hw99 = t.half_width(kZ99);
    t.ci = {std::clamp(t.mean - hw95, 0.0, 1.0), std::clamp(t.mean + hw95, 0.0, 1.0),
            std::clamp(t.mean - hw99, 0.0, 1.0), std::clamp(t.mean + hw99, 0.0, 1.0)};
    return t;
}

// stats/tally.h:83-100: replace the counters, recompute, track information gain.
tally &tally::update(std::size_t ones, std::size_t all) {
    if (all == 0) return *this;
    const std::size_t prev_ones = num_one_bits, prev_total = total_bits;
    num_one_bits = ones;
    total_bits = all;
    compute_ci(compute_moments(*this));
    const std::size_t d_ones = num_one_bits - prev_ones;
    const std::size_t zeros = total_bits - num_one_bits, prev_zeros = prev_total - prev_ones;
    gain.add_batch(d_ones, zeros - prev_zeros);
    return *this;
}

// convergence_policy.h:28-61
void update_wald(tally &t, double rel, double z) {
    tally::compute_moments(t);
    const double p_hat = std::max(t.mean, kDeltaEpsilon);
    const double target = rel * p_hat;
    t.linear.epsilon = t.half_width(z);
    t.linear.target_epsilon = target;
    t.linear.target_trials = required_trials_from_normal_quantile_two_sided(p_hat, target, z);
    t.log10.epsilon = half_width_log10(t, z);
    t.log10.target_epsilon = rel;
    t.log10.target_trials = required_trials_log10_from_normal_quantile_two_sided(p_hat, rel, z);
}

// convergence_policy.h:66-143: Jeffreys prior Beta(1/2, 1/2), central
// credible interval at the level z encodes (2 Phi(z) - 1).
void update_bayes(tally &t, double rel, double z) {
    tally::compute_moments(t);
    const double a0 = 0.5, b0 = 0.5;
    const double alpha = a0 + (double)t.num_one_bits;
    const double beta = b0 + (double)(t.total_bits - t.num_one_bits);
    const double p_hat = alpha / (alpha + beta);
    const double cred = std::clamp(2.0 * normal_cdf(z) - 1.0, 0.0, 1.0);
    const double tail = (1.0 - cred) / 2.0;
    const double lower = beta_quantile(alpha, beta, tail);
    const double upper = beta_quantile(alpha, beta, 1.0 - tail);
    const double eps = (upper - lower) / 2.0;
    t.linear.epsilon = eps;
    t.log10.epsilon = eps / (p_hat * std::log(10.0));
    const double target_lin = rel * p_hat;
    t.linear.target_epsilon = target_lin;
    t.log10.target_epsilon = rel;
    const double var = p_hat * (1.0 - p_hat);
    const double ln10 = std::log(10.0);
    const double rhs_lin = (z * z * var) / (target_lin * target_lin);
    const double rhs_log = (z * z * (1.0 - p_hat)) / (p_hat * rel * rel * ln10 * ln10);
    const double corr = a0 + b0 + 1.0;
    const auto n_lin = (std::size_t)std::ceil(std::max(0.0, rhs_lin - corr));
    const auto n_log = (std::size_t)std::ceil(std::max(0.0, rhs_log - corr));
    t.linear.target_trials = std::max<std::size_t>(n_lin, t.total_bits);
    t.log10.target_trials = std::max<std::size_t>(n_log, t.total_bits);
}

}  // namespace stats
}  // namespace host
}  // namespace mcg
