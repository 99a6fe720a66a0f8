/*
 * mcg_host.h -- C ABI of the host layer above the engine (libmcg.so).
 *
 * Mirrors the caller-facing side of mcSCRAM's Monte Carlo probability path
 * (paths inside the mcSCRAM project):
 *   mcg_pdag_*     the PDAG the engine is built from (core::Pdag, src/pdag.h)
 *                  and its layering (layer_manager::layered_toposort,
 *                  src/mc/queue/layer_manager.tpp:63-118)
 *   mcg_manager_*  scram::mc::queue::layer_manager (src/mc/queue/layer_manager.h:284-375)
 *   mcg_run_to_convergence
 *                  convergence_controller::run_to_convergence
 *                  (src/mc/scheduler/convergence_controller.h:371-381)
 *   mcg_compute_tallies
 *                  ProbabilityAnalyzer<DirectEval>::ComputeTallies
 *                  (src/mc/core/probability_analysis.cc:98-209)
 * C++ callers can use the classes in mcscram_b200/csrc/host_manager.hpp
 * directly; these functions wrap them and turn exceptions into status codes.
 */
#ifndef MCG_HOST_H
#define MCG_HOST_H

#include "mcg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mcg_pdag mcg_pdag;
typedef struct mcg_manager mcg_manager;

/* One tally as the reference's stats::tally holds it (src/mc/stats/tally.h:18-101). */
typedef struct mcg_tally {
    int32_t index;            /* PDAG index of the node */
    uint64_t num_one_bits;
    uint64_t total_bits;
    double mean;
    double std_err;
    double ci[4];             /* lower95, upper95, lower99, upper99 */
    double linear_epsilon;
    double linear_target_epsilon;
    uint64_t linear_target_trials;
    double log10_epsilon;
    double log10_target_epsilon;
    uint64_t log10_target_trials;
} mcg_tally;

#define MCG_POLICY_BAYES 0
#define MCG_POLICY_WALD 1

/* The Monte Carlo fields of core::Settings (src/settings.h:439-464). */
typedef struct mcg_settings {
    uint64_t num_trials;         /* 0 = until convergence (early stop forced on) */
    uint32_t early_stop;
    uint32_t policy;             /* MCG_POLICY_BAYES (default) or MCG_POLICY_WALD */
    double ci_confidence;        /* two-sided level, default 0.99 */
    double ci_rel_margin_error;  /* delta, default 0.001 */
    double ci_burnin_trials;     /* default 2^20 */
    double overhead_ratio;       /* default 0.05 (accepted, not needed by the fused kernel) */
    double oracle_p;             /* < 0: unset */
    uint64_t max_words_per_iteration; /* words per pass cap; 0 = 2^24 */
    uint32_t pipelined;          /* 1 (default): judge pass k while pass k + 1 runs, same results
                                    as 0 (wait for every pass) at the cost of one discarded pass */
} mcg_settings;

typedef struct mcg_convergence_report {
    uint64_t burn_in_steps;
    uint64_t steps;
    uint64_t passes;
    uint64_t trials;
    uint64_t projected_trials;
    uint32_t epsilon_converged;
    uint32_t log10_converged;
    uint32_t iteration_limit_reached;
    double epsilon;
    double target_epsilon;
    double epsilon_log10;
    double target_epsilon_log10;
    double info_gain_bits;
    double seconds;
} mcg_convergence_report;

/* Defaults of core::Settings for the Monte Carlo path. */
mcg_status mcg_settings_default(mcg_settings *out);

mcg_status mcg_pdag_create(mcg_pdag **out);
mcg_status mcg_pdag_destroy(mcg_pdag *pdag);
/* A Variable (basic event); index >= 2 like Pdag::kVariableStartIndex. */
mcg_status mcg_pdag_add_variable(mcg_pdag *pdag, int32_t index, double probability);
/* A Gate; args are signed node indices (negative = complemented argument) in
 * the order of the gate's argument containers. */
mcg_status mcg_pdag_add_gate(mcg_pdag *pdag, int32_t index, uint8_t connective, uint32_t min_number,
                             const int32_t *args, uint32_t n_args);
mcg_status mcg_pdag_set_root(mcg_pdag *pdag, int32_t index);
mcg_status mcg_pdag_set_probability(mcg_pdag *pdag, int32_t index, double probability);
/* Basic events in layer-0 block order (position = event_idx); *n_out gets the
 * count, at most `capacity` indices are written. */
mcg_status mcg_pdag_event_order(const mcg_pdag *pdag, int32_t *pdag_indices, uint32_t capacity, uint32_t *n_out);
/* Node counts of the flattened graph (gathered basic events and gates). */
mcg_status mcg_pdag_flat_sizes(const mcg_pdag *pdag, uint32_t *n_be, uint32_t *n_gates, uint64_t *n_inputs);
/* The flattened graph itself, into caller arrays sized by mcg_pdag_flat_sizes
 * (tally list = tally_indices).  Any output pointer may be NULL. */
mcg_status mcg_pdag_flatten(const mcg_pdag *pdag, const int32_t *tally_indices, uint32_t n_tally,
                            int32_t *be_pdag_idx, uint32_t *be_event_idx, uint64_t *be_threshold,
                            int32_t *gate_pdag_idx, uint8_t *gate_op, uint32_t *gate_k, uint32_t *gate_in_begin,
                            uint32_t *gate_in_count, uint32_t *gate_neg_count, uint32_t *inputs,
                            uint32_t *tally_nodes);

/* layer_manager(pdag, num_trials, to_tally, overhead_ratio). */
mcg_status mcg_manager_create(const mcg_pdag *pdag, uint64_t num_trials, const int32_t *tally_indices,
                              uint32_t n_tally, double overhead_ratio, const mcg_run_desc *run,
                              uint64_t max_words_per_iteration, mcg_manager **out);
mcg_status mcg_manager_destroy(mcg_manager *m);
mcg_status mcg_manager_single_pass(mcg_manager *m);
mcg_status mcg_manager_pass(mcg_manager *m, uint64_t count);
mcg_status mcg_manager_single_pass_and_tally(mcg_manager *m, int32_t index, mcg_tally *out);
/* pass_wait_collect(map, total_passes, passes_between_waits); out gets the
 * n_tally tallies in the order of tally_indices at creation. */
mcg_status mcg_manager_pass_wait_collect(mcg_manager *m, uint64_t total_passes, uint64_t passes_between_waits,
                                         mcg_tally *out, uint32_t capacity);
mcg_status mcg_manager_collect_tallies(mcg_manager *m, mcg_tally *out, uint32_t capacity);
mcg_status mcg_manager_node_count(mcg_manager *m, uint64_t *count);
mcg_status mcg_manager_shape(mcg_manager *m, uint64_t *batch_size, uint64_t *bitpacks_per_batch,
                             uint64_t *total_iterations);
mcg_status mcg_manager_engine(mcg_manager *m, mcg_engine **engine);

/* Burn-in then convergence steps until the policy's criterion, the pass limit,
 * or (without early stop) the trial budget; out gets every tally. */
mcg_status mcg_run_to_convergence(mcg_manager *m, const mcg_settings *settings, mcg_tally *out, uint32_t capacity,
                                  mcg_convergence_report *report);

/* ComputeTallies: builds the engine for the PDAG root plus the watched nodes,
 * runs to convergence, collects.  out[0] is the root, then watch[i]. */
mcg_status mcg_compute_tallies(const mcg_pdag *pdag, const mcg_settings *settings, const int32_t *watch,
                               uint32_t n_watch, const mcg_run_desc *run, mcg_tally *out,
                               mcg_convergence_report *report);

/* Statistics helpers (src/mc/stats/ci_utils.h, convergence_policy.h). */
double mcg_normal_quantile_two_sided(double confidence);
double mcg_beta_quantile(double a, double b, double q);
mcg_status mcg_sample_shape(uint64_t num_trials, uint64_t max_words_per_iteration, uint64_t *words_per_iteration,
                            uint64_t *total_iterations, uint64_t *rounded_trials);

/* Monte Carlo importance factors: one pass of word_count words (pass
 * `iteration`) over the graph, tallying the top event graph->tally_nodes[0]
 * and, for each requested basic event (flattened ids in [0, n_be); NULL =
 * every event), the conjunction of the top event and that event.  Fills
 * out[n_events] with the estimates
 *     P(top | x=1) = P(top and x) / p,  P(top | x=0) = (P(top) - P(top and x)) / (1 - p),
 *     mif = P(top | x=1) - P(top | x=0)  (Birnbaum),
 * and cif, raw, dif, rrw from mif as the exact analysis defines them
 * (src/importance_analysis.cc:50-56), p being the probability the sampler
 * draws (threshold / 2^32); as there, cif, raw, dif and rrw stay 0 when
 * P(top) = 0, and rrw stays 0 when P(top) = p * mif.  A conditional that no
 * sample can estimate (p = 0 or p = 1) and the mif from it are NaN.
 * Replaces the Monte Carlo importance analysis
 * the reference leaves as a stub (src/mc/core/importance_analysis.cc).
 * run may be NULL (strip mode, device 0).  Conditional estimates of an
 * event with small p rest on about p * samples draws. */
typedef struct mcg_importance_factor {
    uint32_t event;
    uint64_t samples;
    double p, p_top, p_joint, p_top_given_1, p_top_given_0;
    double mif, cif, dif, raw, rrw;
} mcg_importance_factor;

mcg_status mcg_importance_factors(const mcg_graph_desc *graph, const uint32_t *events, uint32_t n_events,
                                  const mcg_run_desc *run, uint32_t iteration, uint64_t word_count,
                                  mcg_importance_factor *out);

/* The factors of one event from its probability p and the top event's
 * P(top), P(top | x=1) and P(top | x=0) (exact, or estimated elsewhere), by
 * the same relations as mcg_importance_factors; p_joint = p * P(top | x=1),
 * samples = 0.  Host only: it needs no device. */
mcg_status mcg_importance_from_conditionals(double p, double p_top, double p_top_given_1, double p_top_given_0,
                                            mcg_importance_factor *out);

#ifdef __cplusplus
}
#endif

#endif /* MCG_HOST_H */
