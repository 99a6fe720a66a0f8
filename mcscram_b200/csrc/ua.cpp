// ua.cpp -- batched uncertainty analysis driver (mcg_ua_run, include/mcg_batch.h).
//
// Mirrors UncertaintyAnalyzer<Calculator>::Sample / CalculateStatistics
// (mcSCRAM src/uncertainty_analysis.h:154-168, .cc:108-158): draw every
// deviate, clip the probability, evaluate the top event, then summarise the
// samples.  The reference evaluates one trial at a time; here all draws of
// all trees are one batched launch.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "error.hpp"
#include "graph.hpp"
#include "host_stats.hpp"
#include "mcg_batch.h"

uint32_t mcg_batch_tree_count(const mcg_batch *b);
uint32_t mcg_batch_tree_n_be(const mcg_batch *b, uint32_t t);

namespace {

double quantile(std::vector<double> v, double q) {
    std::sort(v.begin(), v.end());
    if (v.empty()) return 0.0;
    const double h = (double)(v.size() - 1) * q;
    const size_t lo = (size_t)std::floor(h);
    const size_t hi = std::min(lo + 1, v.size() - 1);
    return v[lo] + (h - (double)lo) * (v[hi] - v[lo]);
}

}  // namespace

extern "C" mcg_status mcg_ua_run(mcg_batch *b, const mcg_ua_desc *d, double *p_top, mcg_ua_stats *stats,
                                 uint64_t *thresholds_out, double *kernel_ms) {
    mcg::clear_error();
    if (!b || !d || !d->base_p || !p_top) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (d->draws_per_tree == 0 || d->words_per_instance == 0) return mcg::fail(MCG_ERR_INVALID, "empty run");
    if (!(d->error_factor >= 1.0) || !(d->level > 0.5 && d->level < 1.0))
        return mcg::fail(MCG_ERR_INVALID, "error factor must be >= 1 and level in (0.5, 1)");
    const uint32_t n_trees = mcg_batch_tree_count(b);
    const uint32_t draws = d->draws_per_tree;
    // z of the error factor's level: EF = exp(z * sigma)
    const double z = mcg::host::stats::normal_quantile_two_sided(2.0 * d->level - 1.0);
    const double sigma = std::log(d->error_factor) / z;
    std::mt19937_64 rng(d->seed);
    std::normal_distribution<double> normal(0.0, 1.0);
    std::vector<uint32_t> inst_tree;
    std::vector<uint64_t> thr_off, thr;
    uint64_t base_off = 0;
    for (uint32_t t = 0; t < n_trees; ++t) {
        const uint32_t nb = mcg_batch_tree_n_be(b, t);
        for (uint32_t k = 0; k < draws; ++k) {
            inst_tree.push_back(t);
            thr_off.push_back(thr.size());
            for (uint32_t e = 0; e < nb; ++e) {
                const double base = d->base_p[base_off + e];
                if (!(base >= 0.0 && base <= 1.0)) return mcg::fail(MCG_ERR_INVALID, "base probability outside [0, 1]");
                double p = 0.0;
                if (base > 0.0) {
                    const double mu = d->parameterization == MCG_UA_MEAN ? std::log(base) - sigma * sigma / 2.0
                                                                         : std::log(base);
                    p = std::exp(mu + sigma * normal(rng));
                } else {
                    (void)normal(rng);
                }
                p = std::min(std::max(p, 0.0), std::min(d->clip_max, 1.0));
                thr.push_back(mcg::probability_threshold(p));
            }
        }
        base_off += nb;
    }
    std::vector<uint64_t> ones(inst_tree.size());
    const uint32_t iteration = d->iteration ? d->iteration : 1u;
    const mcg_status st = mcg_batch_run(b, (uint32_t)inst_tree.size(), inst_tree.data(), thr_off.data(), thr.data(),
                                        thr.size(), iteration, d->words_per_instance, ones.data());
    if (st != MCG_OK) return st;
    const double n_samples = (double)d->words_per_instance * 64.0;
    for (size_t i = 0; i < ones.size(); ++i) p_top[i] = (double)ones[i] / n_samples;
    if (thresholds_out) std::copy(thr.begin(), thr.end(), thresholds_out);
    if (stats) {
        for (uint32_t t = 0; t < n_trees; ++t) {
            std::vector<double> v(p_top + (size_t)t * draws, p_top + (size_t)(t + 1) * draws);
            mcg_ua_stats &s = stats[t];
            double mean = 0.0;
            for (double x : v) mean += x;
            mean /= draws;
            double var = 0.0;
            for (double x : v) var += (x - mean) * (x - mean);
            const double sd = draws > 1 ? std::sqrt(var / (draws - 1)) : 0.0;
            s.mean = mean;
            s.sigma = sd;
            s.error_factor = std::exp(1.96 * sd);
            s.ci_low = mean - sd * 1.96 / std::sqrt((double)draws);
            s.ci_high = mean + sd * 1.96 / std::sqrt((double)draws);
            s.p05 = quantile(v, 0.05);
            s.p50 = quantile(v, 0.50);
            s.p95 = quantile(v, 0.95);
            s.min = *std::min_element(v.begin(), v.end());
            s.max = *std::max_element(v.begin(), v.end());
        }
    }
    if (kernel_ms) {
        mcg_batch_info info;
        mcg_batch_info_get(b, &info);
        *kernel_ms = info.last_kernel_ms;
    }
    return MCG_OK;
}
