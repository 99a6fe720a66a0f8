/*
 * oracle/mc_oracle.c -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * CPU restatement of the reference's Monte Carlo dataflow over a layered
 * PDAG: basic-event words, gate words, popcount tallies.  It is the checker
 * for the CUDA path and the timed CPU baseline; the product never links it.
 *
 * Built twice by oracle/Makefile:
 *   liboracle.so          -- with the plain-C Philox restatement (philox_oracle.h)
 *   _ref/libref_mc.so     -- with ORC_WITH_REF_PHILOX: every basic-event word
 *                            comes from the reference's own philox128.h,
 *                            compiled from its sources (ref_philox_shim.cc)
 * Comparing the two pins the restated sampler to the reference's code.
 *
 * Followed reference lines (paths inside the mcSCRAM project):
 *   src/mc/kernel/basic_event.h:68-142  word w of event e at pass t
 *   src/mc/kernel/gate.h:262-264        init: all-ones for AND/NAND, else 0
 *   src/mc/kernel/gate.h:325-351        positives [0, off), then ~inputs [off, n)
 *   src/mc/kernel/gate.h:356-358        final NOT for NAND/NOR/NOT
 *   src/mc/kernel/gate.h:529-553        ATLEAST: uint8 per-lane count, cnt >= k
 *   src/mc/kernel/tally.h:337-360       ones += popcount(word)
 *   src/mc/event/node.h:655-662         negated inputs stored after the positives
 *   src/mc/queue/queueable.h:725-731    pass numbering starts at 1
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "philox_oracle.h"

#ifdef ORC_WITH_REF_PHILOX
uint64_t ref_pack_word(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t threshold);
#define ORC_WORD(c0, c1, c2, c3, thr) ref_pack_word((c0), (c1), (c2), (c3), (thr))
#else
#define ORC_WORD(c0, c1, c2, c3, thr) orc_pack_word((c0), (c1), (c2), (c3), (thr))
#endif

/* Connective values of the reference (src/pdag.h:265-276). */
enum { ORC_AND = 0, ORC_OR = 1, ORC_ATLEAST = 2, ORC_XOR = 3, ORC_NOT = 4,
       ORC_NAND = 5, ORC_NOR = 6, ORC_NULL = 7 };

/* Flattened PDAG.  Node ids: [0, n_be) basic events, [n_be, n_be + n_gates)
 * gates in a topological order (every input id is smaller than the gate's). */
typedef struct {
    uint32_t n_be;
    uint32_t n_gates;
    const int32_t *be_pdag_idx;
    const uint32_t *be_event_idx;
    const uint64_t *be_threshold;
    const uint8_t *gate_op;
    const uint32_t *gate_k;
    const uint32_t *gate_in_begin;
    const uint32_t *gate_in_count;
    const uint32_t *gate_neg_count;
    const uint32_t *inputs;
} orc_graph;

uint64_t orc_word(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint64_t thr) {
    return ORC_WORD(c0, c1, c2, c3, thr);
}

uint64_t orc_be_word_at(uint32_t pdag_idx, uint32_t event_idx, uint32_t sample_idx,
                        uint32_t iteration, uint64_t thr) {
    return ORC_WORD(pdag_idx + 1u, event_idx + 1u, sample_idx + 1u, (iteration + 1u) << 6, thr);
}

static uint64_t orc_gate_word(const orc_graph *g, uint32_t gi, const uint64_t *vals) {
    const uint8_t op = g->gate_op[gi];
    const uint32_t b = g->gate_in_begin[gi];
    const uint32_t n = g->gate_in_count[gi];
    const uint32_t off = n - g->gate_neg_count[gi];
    const uint32_t *in = g->inputs + b;
    if (op == ORC_ATLEAST) {
        const uint8_t k = (uint8_t)g->gate_k[gi];
        uint64_t out = 0;
        for (uint32_t lane = 0; lane < 64; ++lane) {
            const uint64_t mask = (uint64_t)1 << lane;
            uint8_t cnt = 0;
            for (uint32_t i = 0; i < off; ++i) cnt += (vals[in[i]] & mask) ? 1 : 0;
            for (uint32_t i = off; i < n; ++i) cnt += (~vals[in[i]] & mask) ? 1 : 0;
            if (cnt >= k) out |= mask;
        }
        return out;
    }
    uint64_t r = (op == ORC_AND || op == ORC_NAND) ? ~(uint64_t)0 : (uint64_t)0;
    for (uint32_t i = 0; i < n; ++i) {
        const uint64_t v = (i < off) ? vals[in[i]] : ~vals[in[i]];
        switch (op) {
            case ORC_OR: case ORC_NOR: r |= v; break;
            case ORC_AND: case ORC_NAND: r &= v; break;
            case ORC_XOR: r ^= v; break;
            case ORC_NULL: case ORC_NOT: r = v; break;
            default: break;
        }
    }
    if (op == ORC_NAND || op == ORC_NOR || op == ORC_NOT) r = ~r;
    return r;
}

/* Evaluate every node for one word column; vals has n_be + n_gates entries. */
static void orc_eval_column(const orc_graph *g, uint32_t iteration, uint32_t sample_idx,
                            uint64_t *vals) {
    for (uint32_t e = 0; e < g->n_be; ++e) {
        vals[e] = ORC_WORD((uint32_t)g->be_pdag_idx[e] + 1u, g->be_event_idx[e] + 1u,
                           sample_idx + 1u, (iteration + 1u) << 6, g->be_threshold[e]);
    }
    for (uint32_t gi = 0; gi < g->n_gates; ++gi) {
        vals[g->n_be + gi] = orc_gate_word(g, gi, vals);
    }
}

/* Validates node ids; returns 0 when the graph is well formed. */
int orc_check_graph(const orc_graph *g) {
    for (uint32_t gi = 0; gi < g->n_gates; ++gi) {
        if (g->gate_neg_count[gi] > g->gate_in_count[gi]) return -1;
        if (g->gate_op[gi] > ORC_NULL) return -2;
        for (uint32_t i = 0; i < g->gate_in_count[gi]; ++i) {
            if (g->inputs[g->gate_in_begin[gi] + i] >= g->n_be + gi) return -3;
        }
    }
    return 0;
}

/* Materialised words of every node for columns [word_begin, word_begin+n_words)
 * of pass `iteration`: out[node * n_words + w]. */
int orc_eval_words(const orc_graph *g, uint32_t iteration, uint64_t word_begin,
                   uint64_t n_words, uint64_t *out, int n_threads) {
    if (orc_check_graph(g)) return -1;
    const uint32_t n_nodes = g->n_be + g->n_gates;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel
#endif
    {
        uint64_t *vals = (uint64_t *)malloc(sizeof(uint64_t) * (n_nodes ? n_nodes : 1));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t w = 0; w < (int64_t)n_words; ++w) {
            orc_eval_column(g, iteration, (uint32_t)(word_begin + (uint64_t)w), vals);
            for (uint32_t n = 0; n < n_nodes; ++n) out[(uint64_t)n * n_words + (uint64_t)w] = vals[n];
        }
        free(vals);
    }
    return 0;
}

/* Tallies (sum of popcounts) of the listed nodes over passes
 * [iteration_first, iteration_first + n_iterations) and columns
 * [word_begin, word_begin + n_words).  ones_out[i] is accumulated into. */
int orc_tallies(const orc_graph *g, uint32_t iteration_first, uint32_t n_iterations,
                uint64_t word_begin, uint64_t n_words, uint32_t n_tally,
                const uint32_t *tally_nodes, uint64_t *ones_out, int n_threads) {
    if (orc_check_graph(g)) return -1;
    const uint32_t n_nodes = g->n_be + g->n_gates;
    for (uint32_t i = 0; i < n_tally; ++i)
        if (tally_nodes[i] >= n_nodes) return -2;
    const int64_t total = (int64_t)n_words * (int64_t)n_iterations;
#ifdef _OPENMP
    if (n_threads > 0) omp_set_num_threads(n_threads);
#pragma omp parallel
#endif
    {
        uint64_t *vals = (uint64_t *)malloc(sizeof(uint64_t) * (n_nodes ? n_nodes : 1));
        uint64_t *acc = (uint64_t *)calloc(n_tally ? n_tally : 1, sizeof(uint64_t));
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t j = 0; j < total; ++j) {
            const uint32_t it = iteration_first + (uint32_t)(j / (int64_t)n_words);
            const uint64_t w = word_begin + (uint64_t)(j % (int64_t)n_words);
            orc_eval_column(g, it, (uint32_t)w, vals);
            for (uint32_t i = 0; i < n_tally; ++i)
                acc[i] += (uint64_t)__builtin_popcountll(vals[tally_nodes[i]]);
        }
#ifdef _OPENMP
#pragma omp critical
#endif
        for (uint32_t i = 0; i < n_tally; ++i) ones_out[i] += acc[i];
        free(acc);
        free(vals);
    }
    return 0;
}

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
