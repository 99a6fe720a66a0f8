/*
 * mcg_batch.h -- batched instances and uncertainty analysis (libmcg.so).
 *
 * The reference runs uncertainty analysis as N outer trials, each sampling
 * new basic-event probabilities and calling CalculateTotalProbability
 * (mcSCRAM src/uncertainty_analysis.h:154-168), which builds a fresh
 * layer_manager per trial (src/mc/core/probability_analysis.cc:112); its
 * Monte Carlo engine then reads the nominal probabilities, not the sampled
 * ones (src/mc/queue/kernel_builder.h:179-183).  Here every (tree, draw)
 * instance is evaluated with its own sampled thresholds, all instances in
 * one persistent work-queue launch captured in a CUDA graph.  Each instance
 * uses the counters of a fresh manager's pass `iteration` (by default 1), so
 * the draws of one tree share their random numbers: what varies between
 * draws is the parameters, not the Monte Carlo noise.
 */
#ifndef MCG_BATCH_H
#define MCG_BATCH_H

#include "mcg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mcg_batch mcg_batch;

typedef struct mcg_batch_info {
    uint32_t n_trees;
    uint32_t smem_slots;       /* shared-memory slots per thread (common budget) */
    uint32_t max_global_slots; /* largest global-scratch need over the trees */
    uint32_t grid_ctas;
    uint64_t total_ops;
    uint64_t launches;         /* kernel launches so far (graph replays count once each) */
    double last_kernel_ms;     /* duration of the last batched launch (CUDA events) */
    uint32_t instances_per_item; /* instances of one tree evaluated together, sharing their
                                  * Philox calls (4; 1 when a tree has an ATLEAST gate of
                                  * more than 15 inputs) */
} mcg_batch_info;

/* Compiles every tree (a flattened graph whose tally_nodes are the nodes to
 * count, normally the root) for threshold tables supplied per instance. */
mcg_status mcg_batch_create(const mcg_graph_desc *trees, uint32_t n_trees, const mcg_run_desc *run,
                            mcg_batch **out);
mcg_status mcg_batch_destroy(mcg_batch *b);

/* Runs n_instances instances in one persistent launch: instance i evaluates
 * tree inst_tree[i] with thresholds[thr_offset[i] .. thr_offset[i] + n_be of
 * that tree) over sample words [0, words_per_instance) of pass `iteration`;
 * ones[i] receives the sum of its tallied nodes' ones.  Host arrays; the
 * copies in and out are on the batch's stream.  The launch is captured in a
 * CUDA graph on first use and replayed while the shapes stay the same. */
mcg_status mcg_batch_run(mcg_batch *b, uint32_t n_instances, const uint32_t *inst_tree, const uint64_t *thr_offset,
                         const uint64_t *thresholds, uint64_t n_thresholds, uint32_t iteration,
                         uint64_t words_per_instance, uint64_t *ones);

mcg_status mcg_batch_info_get(mcg_batch *b, mcg_batch_info *info);

#define MCG_UA_MEDIAN 0 /* base probability is the lognormal median */
#define MCG_UA_MEAN 1   /* base probability is the lognormal mean (LognormalDeviate, src/expression/random_deviate.cc:101-109) */

typedef struct mcg_ua_desc {
    const double *base_p;        /* per tree, its n_be basic-event probabilities, trees concatenated */
    uint32_t draws_per_tree;
    double error_factor;         /* EF, e.g. 3 */
    double level;                /* EF confidence level, e.g. 0.95 (z = 1.6449) */
    uint32_t parameterization;   /* MCG_UA_MEDIAN or MCG_UA_MEAN */
    double clip_max;             /* sampled probabilities are clipped to [0, clip_max] */
    uint64_t seed;
    uint64_t words_per_instance;
    uint32_t iteration;          /* 0 = 1 */
} mcg_ua_desc;

/* Per-tree statistics of the top-event probability over its draws, as
 * UncertaintyAnalysis::CalculateStatistics reports them
 * (src/uncertainty_analysis.cc:122-158); quantiles are empirical with linear
 * interpolation. */
typedef struct mcg_ua_stats {
    double mean;
    double sigma;          /* sample standard deviation (n - 1) */
    double error_factor;   /* exp(1.96 sigma) */
    double ci_low, ci_high;/* mean -/+ 1.96 sigma / sqrt(n) */
    double p05, p50, p95;
    double min, max;
} mcg_ua_stats;

/* Samples lognormal basic-event probabilities for every (tree, draw),
 * evaluates all instances with mcg_batch_run and fills p_top[tree * draws +
 * draw] and stats[tree].  thresholds_out (optional) receives the thresholds
 * used, instance-major.  *kernel_ms gets the batched launch's duration. */
mcg_status mcg_ua_run(mcg_batch *b, const mcg_ua_desc *desc, double *p_top, mcg_ua_stats *stats,
                      uint64_t *thresholds_out, double *kernel_ms);

#ifdef __cplusplus
}
#endif

#endif /* MCG_BATCH_H */
