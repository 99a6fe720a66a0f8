/*
 * mcg_is.h -- importance sampling for rare top events and the proposal MLP
 * (libmcg.so).  No counterpart in the reference, whose Monte Carlo path only
 * samples the nominal probabilities (src/mc/kernel/basic_event.h:125-142).
 *
 * A proposal q_i replaces p_i in the Bernoulli threshold, thr_i = q_i * 2^32,
 * so sampling stays the bit-exact bit-packed Philox sampler and gate
 * evaluation stays the same kernels.  For every sample where the top event
 * fires, the likelihood ratio
 *     log w = C + sum_i a_i x_i,  C = sum_i ln((1 - p_i) / (1 - q_i)),
 *     a_i = ln(p_i / q_i) - ln((1 - p_i) / (1 - q_i))
 * is accumulated in FP64, and so are sum w, sum w^2 (the estimator
 * P = sum w / N and its variance) and, for the cross-entropy update,
 * sum w x_i per basic event.  p_i and q_i are taken at their quantised
 * values thr / 2^32, the probabilities the sampler actually draws.
 */
#ifndef MCG_IS_H
#define MCG_IS_H

#include "mcg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mcg_is mcg_is;

typedef struct mcg_is_result {
    uint64_t samples;      /* N */
    uint64_t hits;         /* samples where the top event fired */
    double sum_w;          /* sum over hits of w */
    double sum_w2;         /* sum over hits of w^2 */
    double estimate;       /* sum_w / N */
    double std_err;        /* sqrt((sum_w2 / N - estimate^2) / (N - 1)) */
    double rel_err;        /* std_err / estimate */
    double ess;            /* (sum_w)^2 / sum_w2 */
    double max_log_w;      /* largest log-weight seen */
    double kernel_ms;      /* device time of the run (CUDA events) */
} mcg_is_result;

/* Engine over a flattened graph whose tally list holds exactly the top
 * event.  Nominal thresholds come from graph->be_threshold.  Uses the
 * staged kernels (layered_max_words = words per chunk). */
mcg_status mcg_is_create(const mcg_graph_desc *graph, const mcg_run_desc *run, mcg_is **out);
mcg_status mcg_is_destroy(mcg_is *is);

/* Samples pass `iteration`, words [word_begin, word_begin + word_count),
 * with proposal thresholds q_threshold[n_be] (host array; each in
 * [1, 2^32 - 1] where the nominal threshold is in that range, else equal to
 * it).  ce_num (host, n_be doubles, optional) receives sum over hits of
 * w * x_i for the cross-entropy update. */
mcg_status mcg_is_run(mcg_is *is, const uint64_t *q_threshold, uint32_t iteration, uint64_t word_begin,
                      uint64_t word_count, mcg_is_result *result, double *ce_num);

/* Batched form: many independent trees joined into one graph (no node read
 * by two trees), sampled together in one staged pass per call.  Tree k owns
 * basic events [be_begin[k], be_begin[k + 1]) (be_begin has n_tree + 1
 * entries, from 0 to n_be) and its top event is graph->tally_nodes[k]
 * (n_tally == n_tree); create rejects graphs where a gate reads two trees
 * or a tallied node is not in its tree.  Each tree gets its own likelihood
 * ratio (the C and a_i of its events) and its own sums.  With
 * run->layered_max_words = 0 a chunk holds at most 2^17 words (the staged
 * engine's memory budget otherwise), since joined graphs are rebuilt as trees
 * finish. */
typedef struct mcg_is_batch mcg_is_batch;

mcg_status mcg_is_batch_create(const mcg_graph_desc *graph, uint32_t n_tree, const uint32_t *be_begin,
                               const mcg_run_desc *run, mcg_is_batch **out);
mcg_status mcg_is_batch_destroy(mcg_is_batch *b);

/* Samples pass `iteration`, words [word_begin, word_begin + word_count) of
 * every tree with proposal thresholds q_threshold[n_be] (rules as for
 * mcg_is_run).  With n_defensive > 0 defensive proposals
 * (q_defensive[n_defensive][n_be], component-major, and their word counts
 * words_defensive[n_defensive], together at most word_count) the main
 * proposal draws the first word_count - sum(words_defensive) words and
 * defensive proposal c the next words_defensive[c], and every sample is
 * weighted by the balance heuristic of multiple importance sampling,
 *     w = p(x) / sum_c pi_c q_c(x),   pi_c = words of c / word_count,
 * which stays unbiased and keeps w <= p / (pi_c q_c) for every component
 * (a failure region the main proposal misses is still sampled through
 * the defensive ones).  At most 7 defensive proposals.
 * words_cutset > 0 adds, after them, a cut-set component for trees of
 * AND/OR/ATLEAST gates (threshold <= 8) without negations and without gates
 * read by several gates: each of its samples draws a minimal cut set C of
 * its tree with probability prod_{i in C} p_i / S (S the sum of that product
 * over all minimal cut sets), forces C's events and draws the others at
 * their nominal probabilities; its density p(x) N(x) / S (N(x): minimal cut
 * sets inside x) enters the same mixture, bounding every weight by
 * S / pi_cutset -- the mixture form of importance sampling for a union of
 * rare events.  Basic events read by several gates (shared events) are
 * drawn first, from q_cutset's thresholds (NULL: their nominal ones), and
 * the cut set is then drawn on the tree conditioned on them; the density
 * becomes r(z) p(x_private) N(x) / S_z (z: the shared events, r their
 * proposal, S_z the sum over the conditioned tree's cut sets).  q_cutset's
 * entries for other events are ignored.
 * tree_sums (host, 4 * n_tree doubles) receives per tree {sum w, sum w^2,
 * hits, max log w} over its word_count * 64 samples; ce_num (host, n_be
 * doubles, optional) sum over hits of w * x_i; kernel_ms (optional) the
 * device time of the call (CUDA events). */
mcg_status mcg_is_batch_run(mcg_is_batch *b, const uint64_t *q_threshold, uint32_t n_defensive,
                            const uint64_t *q_defensive, const uint64_t *words_defensive, uint64_t words_cutset,
                            const uint64_t *q_cutset, uint32_t iteration, uint64_t word_begin, uint64_t word_count,
                            double *tree_sums, double *ce_num, double *kernel_ms);

/* Host only.  For the tree rooted at `root` (AND / OR / ATLEAST /
 * pass-through gates without complemented inputs, each gate read by one gate
 * at most; basic events may be read by several): *p_top = its cut-set sum S
 * (event p = threshold / 2^32; AND product; OR sum; ATLEAST k-th elementary
 * symmetric sum), every basic event counted once per product however many of
 * its leaves it covers, and posterior[e] ~ P(x_e = 1 | top) = p_e S(top |
 * x_e = 1) / S for every event e read by several gates (-1 for the others).
 * S is the rare-event approximation of P(top) (the sum over cut sets).  Below
 * the lowest common ancestor of a shared event's leaves a node's value is a
 * polynomial in that event's indicator; more than max_terms monomials at one
 * gate (0: 4096) gives MCG_ERR_INVALID.  Seeds the cut-set component's
 * proposal for shared events (no reference counterpart). */
mcg_status mcg_shared_posteriors(const mcg_graph_desc *graph, uint32_t root, uint64_t max_terms, double *p_top,
                                 double *posterior);

/* The proposal network: 16 features -> 64 -> 64 -> 1, ReLU, sigmoid output.
 * BF16 weights for the tensor-core products (tcgen05.mma with FP32
 * accumulators in tensor memory), FP32 master weights and Adam state.  The gradient runs in
 * persistent CTAs whose partial gradients are summed in a fixed order, so
 * the same rows give the same gradient bit for bit.  Parameter layout
 * (5,313 floats): W1[16][64], b1[64], W2[64][64], b2[64], W3[64], b3. */
typedef struct mcg_mlp mcg_mlp;
#define MCG_MLP_IN 16
#define MCG_MLP_HIDDEN 64
#define MCG_MLP_PARAMS (16 * 64 + 64 + 64 * 64 + 64 + 64 + 1)

mcg_status mcg_mlp_create(int32_t device, uint64_t seed, mcg_mlp **out);
mcg_status mcg_mlp_destroy(mcg_mlp *m);
mcg_status mcg_mlp_set_params(mcg_mlp *m, const float *params);
mcg_status mcg_mlp_get_params(mcg_mlp *m, float *params);
/* q_out[n] = sigmoid(MLP(features[n][16])). Host arrays. */
mcg_status mcg_mlp_forward(mcg_mlp *m, const float *features, uint32_t n, float *q_out);
/* Gradient of the weighted binary cross-entropy
 *     L = sum_i w_i * -(t_i log q_i + (1 - t_i) log(1 - q_i)) / sum_i w_i
 * with respect to every parameter (BF16 forward, FP32 accumulation).
 * weights may be NULL (all 1). */
mcg_status mcg_mlp_grad(mcg_mlp *m, const float *features, const float *targets, const float *weights, uint32_t n,
                        float *grad_out, float *loss_out);
/* `steps` Adam steps (lr, beta1 0.9, beta2 0.999, eps 1e-8) on that loss. */
mcg_status mcg_mlp_train(mcg_mlp *m, const float *features, const float *targets, const float *weights, uint32_t n,
                         uint32_t steps, float lr, float *loss_out);
/* Device time of the steps of the last mcg_mlp_train call (CUDA events on
 * the network's stream, row upload excluded). */
mcg_status mcg_mlp_train_time(mcg_mlp *m, double *ms);

#ifdef __cplusplus
}
#endif

#endif /* MCG_IS_H */
