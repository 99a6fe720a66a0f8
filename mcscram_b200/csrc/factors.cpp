// factors.cpp -- Monte Carlo importance factors (mcg_importance_factors).
//
// The reference's Monte Carlo importance analysis is an empty stub
// (src/mc/core/importance_analysis.cc); its exact analysis defines the
// factors from the Birnbaum factor (src/importance_analysis.cc:50-56).  Here
// one pass tallies, next to the top event, the conjunction "top and x_i" for
// every requested event (an AND gate per event appended after the graph's
// gates), and the factors follow from those counts.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

#include "error.hpp"
#include "graph.hpp"
#include "mcg.h"
#include "mcg_host.h"

// mif from the conditionals, then the exact analysis's relations and its
// zeros where they are undefined (src/importance_analysis.cc:50-56)
static void factors_from_conditionals(double p, double p_top, double given_1, double given_0,
                                      mcg_importance_factor &f) {
    f.p = p;
    f.p_top = p_top;
    f.p_top_given_1 = given_1;
    f.p_top_given_0 = given_0;
    f.mif = given_1 - given_0;
    f.cif = f.raw = f.dif = f.rrw = 0.0;
    if (p_top != 0) {
        f.cif = p * f.mif / p_top;
        f.raw = 1.0 + (1.0 - p) * f.mif / p_top;
        f.dif = p * f.raw;
        if (p_top != p * f.mif) f.rrw = p_top / (p_top - p * f.mif);
    }
}

extern "C" mcg_status mcg_importance_from_conditionals(double p, double p_top, double p_top_given_1,
                                                       double p_top_given_0, mcg_importance_factor *out) {
    mcg::clear_error();
    if (!out) return mcg::fail(MCG_ERR_INVALID, "out must not be NULL");
    if (!(p >= 0.0 && p <= 1.0) || !(p_top >= 0.0 && p_top <= 1.0))
        return mcg::fail(MCG_ERR_INVALID, "p and p_top must be probabilities");
    std::memset(out, 0, sizeof(*out));
    out->p_joint = p * p_top_given_1;
    factors_from_conditionals(p, p_top, p_top_given_1, p_top_given_0, *out);
    return MCG_OK;
}

extern "C" mcg_status mcg_importance_factors(const mcg_graph_desc *graph, const uint32_t *events, uint32_t n_events,
                                             const mcg_run_desc *run_in, uint32_t iteration, uint64_t word_count,
                                             mcg_importance_factor *out) {
    mcg::clear_error();
    if (!graph || !out) return mcg::fail(MCG_ERR_INVALID, "graph and out must not be NULL");
    mcg::Graph g;
    std::string err = mcg::Graph::from_desc(*graph, g);
    if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, err);
    if (g.tally_nodes.empty()) return mcg::fail(MCG_ERR_INVALID, "tally_nodes[0] must name the top event");
    if (word_count == 0 || word_count > (1ull << 32)) return mcg::fail(MCG_ERR_INVALID, "word_count must be in [1, 2^32]");
    const uint32_t root = g.tally_nodes[0];
    std::vector<uint32_t> ev;
    if (events) ev.assign(events, events + n_events);
    else
        for (uint32_t i = 0; i < g.n_be; ++i) ev.push_back(i);
    for (uint32_t e : ev)
        if (e >= g.n_be) return mcg::fail(MCG_ERR_INVALID, "event " + std::to_string(e) + " is not a basic event");

    // gates: the graph's, then AND(top, x_e) per event; tallies: top, then those gates
    const uint32_t n_add = (uint32_t)ev.size();
    std::vector<uint8_t> op(g.gate_op);
    std::vector<uint32_t> k(g.gate_k), in_begin(g.gate_in_begin), in_count(g.gate_in_count), neg(g.gate_neg_count);
    std::vector<int32_t> gpdag(g.gate_pdag_idx);
    std::vector<uint32_t> inputs(g.inputs), tally{root};
    int32_t next_pdag = 0;
    for (int32_t x : g.be_pdag_idx) next_pdag = std::max(next_pdag, x + 1);
    for (int32_t x : g.gate_pdag_idx) next_pdag = std::max(next_pdag, x + 1);
    for (uint32_t j = 0; j < n_add; ++j) {
        op.push_back(MCG_AND);
        k.push_back(0);
        in_begin.push_back((uint32_t)inputs.size());
        in_count.push_back(2);
        neg.push_back(0);
        gpdag.push_back(next_pdag + (int32_t)j);
        inputs.push_back(root);
        inputs.push_back(ev[j]);
        tally.push_back(g.n_nodes() + j);
    }
    mcg_graph_desc d = *graph;
    d.n_gates = g.n_gates + n_add;
    d.gate_pdag_idx = gpdag.data();
    d.gate_op = op.data();
    d.gate_k = k.data();
    d.gate_in_begin = in_begin.data();
    d.gate_in_count = in_count.data();
    d.gate_neg_count = neg.data();
    d.inputs = inputs.data();
    d.n_inputs = inputs.size();
    d.n_tally = (uint32_t)tally.size();
    d.tally_nodes = tally.data();
    mcg_run_desc run{};
    if (run_in) run = *run_in;
    else run.mode = MCG_MODE_STRIP;

    mcg_engine *e = nullptr;
    mcg_status st = mcg_create(&d, &run, &e);
    if (st != MCG_OK) return st;
    st = mcg_run(e, iteration, 1, 0, word_count);
    std::vector<uint64_t> ones(tally.size());
    uint64_t total = 0;
    if (st == MCG_OK) st = mcg_read_tallies(e, ones.data(), &total);
    const std::string keep = st == MCG_OK ? std::string() : mcg::last_error();
    mcg_destroy(e);
    if (st != MCG_OK) return mcg::fail(st, keep);

    const double n = (double)total;
    const double p_top = (double)ones[0] / n;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    for (uint32_t j = 0; j < n_add; ++j) {
        mcg_importance_factor &f = out[j];
        std::memset(&f, 0, sizeof(f));
        f.event = ev[j];
        const uint64_t thr = g.be_threshold[ev[j]];
        const double p = thr >= (1ull << 32) ? 1.0 : (double)thr / 4294967296.0;  // the probability sampled
        const double joint = (double)ones[1 + j] / n;
        f.samples = total;
        f.p_joint = joint;
        factors_from_conditionals(p, p_top, p > 0 ? joint / p : nan, p < 1 ? (p_top - joint) / (1.0 - p) : nan, f);
    }
    return MCG_OK;
}
