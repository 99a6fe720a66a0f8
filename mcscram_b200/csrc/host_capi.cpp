// host_capi.cpp -- C wrappers of the host layer (include/mcg_host.h).
#include <chrono>
#include <cstring>
#include <exception>
#include <memory>
#include <new>

#include "error.hpp"
#include "host_manager.hpp"
#include "mcg_host.h"

struct mcg_pdag {
    mcg::host::Pdag pdag;
};

struct mcg_manager {
    std::unique_ptr<mcg::host::layer_manager> mgr;
    mcg::host::TallyNodeMap map;
    std::vector<int32_t> order;  // tally indices in creation order
};

namespace {

template <typename F>
mcg_status guarded(F &&f) {
    mcg::clear_error();
    try {
        return f();
    } catch (const std::invalid_argument &e) {
        return mcg::fail(MCG_ERR_INVALID, e.what());
    } catch (const std::bad_alloc &) {
        return mcg::fail(MCG_ERR_OOM, "host allocation failed");
    } catch (const std::exception &e) {
        const std::string msg = e.what();
        if (msg.find("no CUDA device") != std::string::npos) return mcg::fail(MCG_ERR_NO_DEVICE, msg);
        return mcg::fail(msg.find("layer_manager: ") == 0 ? MCG_ERR_INVALID : MCG_ERR_CUDA, msg);
    }
}

mcg_status from_err(const std::string &err) { return err.empty() ? MCG_OK : mcg::fail(MCG_ERR_INVALID, err); }

void to_c(int32_t index, const mcg::host::stats::tally &t, mcg_tally &o) {
    o.index = index;
    o.num_one_bits = t.num_one_bits;
    o.total_bits = t.total_bits;
    o.mean = t.mean;
    o.std_err = t.std_err;
    for (int i = 0; i < 4; ++i) o.ci[i] = t.ci[i];
    o.linear_epsilon = t.linear.epsilon;
    o.linear_target_epsilon = t.linear.target_epsilon;
    o.linear_target_trials = t.linear.target_trials;
    o.log10_epsilon = t.log10.epsilon;
    o.log10_target_epsilon = t.log10.target_epsilon;
    o.log10_target_trials = t.log10.target_trials;
}

mcg_status export_map(mcg_manager *m, mcg_tally *out, uint32_t capacity) {
    if (!out) return MCG_OK;
    if (capacity < m->order.size()) return mcg::fail(MCG_ERR_INVALID, "tally output capacity too small");
    for (size_t i = 0; i < m->order.size(); ++i) to_c(m->order[i], m->map[m->order[i]].tally_stats, out[i]);
    return MCG_OK;
}

mcg::host::settings settings_from(const mcg_settings *s) {
    mcg::host::settings o;
    if (!s) return o;
    o.num_trials = s->num_trials;
    o.early_stop = s->early_stop != 0 || s->num_trials == 0;  // Settings::num_trials(0) forces early stop
    o.ci_policy = s->policy == MCG_POLICY_WALD ? mcg::host::stats::policy::wald : mcg::host::stats::policy::bayes;
    o.ci_confidence = s->ci_confidence;
    o.ci_rel_margin_error = s->ci_rel_margin_error;
    o.ci_burnin_trials = s->ci_burnin_trials;
    o.overhead_ratio = s->overhead_ratio;
    o.oracle_p = s->oracle_p;
    o.pipelined = s->pipelined != 0;
    return o;
}

void fill_report(const mcg::host::convergence_controller &c, const mcg::host::layer_manager &mgr, double seconds,
                 mcg_convergence_report *r) {
    if (!r) return;
    std::memset(r, 0, sizeof(*r));
    r->burn_in_steps = c.burn_in_steps();
    r->steps = c.steps();
    r->passes = mgr.iteration();
    r->trials = c.current_trials();
    r->projected_trials = c.projected_trials();
    r->epsilon_converged = c.epsilon_converged();
    r->log10_converged = c.epsilon_log10_converged();
    r->iteration_limit_reached = c.fixed_iteration_limit_reached();
    r->epsilon = c.epsilon();
    r->target_epsilon = c.target_epsilon();
    r->epsilon_log10 = c.epsilon_log10();
    r->target_epsilon_log10 = c.target_epsilon_log10();
    r->info_gain_bits = c.info_gain_cumulative();
    r->seconds = seconds;
}

}  // namespace

extern "C" {

mcg_status mcg_settings_default(mcg_settings *out) {
    mcg::clear_error();
    if (!out) return mcg::fail(MCG_ERR_INVALID, "out is NULL");
    std::memset(out, 0, sizeof(*out));
    out->num_trials = 0;
    out->early_stop = 1;
    out->policy = MCG_POLICY_BAYES;
    out->ci_confidence = 0.99;
    out->ci_rel_margin_error = 0.001;
    out->ci_burnin_trials = (double)(1 << 20);
    out->overhead_ratio = 0.05;
    out->oracle_p = -1.0;
    out->max_words_per_iteration = 0;
    out->pipelined = 1;
    return MCG_OK;
}

mcg_status mcg_pdag_create(mcg_pdag **out) {
    return guarded([&] {
        if (!out) return mcg::fail(MCG_ERR_INVALID, "out is NULL");
        *out = new mcg_pdag();
        return MCG_OK;
    });
}

mcg_status mcg_pdag_destroy(mcg_pdag *p) {
    delete p;
    return MCG_OK;
}

mcg_status mcg_pdag_add_variable(mcg_pdag *p, int32_t index, double probability) {
    return guarded([&] {
        if (!p) return mcg::fail(MCG_ERR_INVALID, "pdag is NULL");
        return from_err(p->pdag.add_variable(index, probability));
    });
}

mcg_status mcg_pdag_add_gate(mcg_pdag *p, int32_t index, uint8_t connective, uint32_t min_number,
                             const int32_t *args, uint32_t n_args) {
    return guarded([&] {
        if (!p) return mcg::fail(MCG_ERR_INVALID, "pdag is NULL");
        return from_err(p->pdag.add_gate(index, connective, min_number, args, n_args));
    });
}

mcg_status mcg_pdag_set_root(mcg_pdag *p, int32_t index) {
    return guarded([&] {
        if (!p) return mcg::fail(MCG_ERR_INVALID, "pdag is NULL");
        return from_err(p->pdag.set_root(index));
    });
}

mcg_status mcg_pdag_set_probability(mcg_pdag *p, int32_t index, double probability) {
    return guarded([&] {
        if (!p) return mcg::fail(MCG_ERR_INVALID, "pdag is NULL");
        return from_err(p->pdag.set_probability(index, probability));
    });
}

mcg_status mcg_pdag_event_order(const mcg_pdag *p, int32_t *idx, uint32_t capacity, uint32_t *n_out) {
    return guarded([&] {
        if (!p) return mcg::fail(MCG_ERR_INVALID, "pdag is NULL");
        mcg::host::Layering lay;
        const std::string err = p->pdag.layered_toposort(lay);
        if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, err);
        const auto &l0 = lay.nodes_by_layer[0];
        if (n_out) *n_out = (uint32_t)l0.size();
        for (size_t i = 0; idx && i < l0.size() && i < capacity; ++i) idx[i] = l0[i];
        return MCG_OK;
    });
}

mcg_status mcg_pdag_flat_sizes(const mcg_pdag *p, uint32_t *n_be, uint32_t *n_gates, uint64_t *n_inputs) {
    return guarded([&] {
        if (!p) return mcg::fail(MCG_ERR_INVALID, "pdag is NULL");
        mcg::Graph g;
        const std::string err = p->pdag.flatten({}, g);
        if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, err);
        if (n_be) *n_be = g.n_be;
        if (n_gates) *n_gates = g.n_gates;
        if (n_inputs) *n_inputs = g.inputs.size();
        return MCG_OK;
    });
}

mcg_status mcg_pdag_flatten(const mcg_pdag *p, const int32_t *tally_indices, uint32_t n_tally, int32_t *be_pdag_idx,
                            uint32_t *be_event_idx, uint64_t *be_threshold, int32_t *gate_pdag_idx, uint8_t *gate_op,
                            uint32_t *gate_k, uint32_t *gate_in_begin, uint32_t *gate_in_count,
                            uint32_t *gate_neg_count, uint32_t *inputs, uint32_t *tally_nodes) {
    return guarded([&] {
        if (!p) return mcg::fail(MCG_ERR_INVALID, "pdag is NULL");
        if (n_tally && !tally_indices) return mcg::fail(MCG_ERR_INVALID, "tally_indices is NULL");
        std::vector<int32_t> t(tally_indices, tally_indices + n_tally);
        mcg::Graph g;
        const std::string err = p->pdag.flatten(t, g);
        if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, err);
        auto cp = [](auto *dst, const auto &v) {
            if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
        };
        cp(be_pdag_idx, g.be_pdag_idx);
        cp(be_event_idx, g.be_event_idx);
        cp(be_threshold, g.be_threshold);
        cp(gate_pdag_idx, g.gate_pdag_idx);
        cp(gate_op, g.gate_op);
        cp(gate_k, g.gate_k);
        cp(gate_in_begin, g.gate_in_begin);
        cp(gate_in_count, g.gate_in_count);
        cp(gate_neg_count, g.gate_neg_count);
        cp(inputs, g.inputs);
        cp(tally_nodes, g.tally_nodes);
        return MCG_OK;
    });
}

mcg_status mcg_manager_create(const mcg_pdag *p, uint64_t num_trials, const int32_t *tally_indices, uint32_t n_tally,
                              double overhead_ratio, const mcg_run_desc *run, uint64_t max_words_per_iteration,
                              mcg_manager **out) {
    return guarded([&] {
        if (!p || !out) return mcg::fail(MCG_ERR_INVALID, "pdag and out must not be NULL");
        if (n_tally && !tally_indices) return mcg::fail(MCG_ERR_INVALID, "tally_indices is NULL");
        auto m = std::make_unique<mcg_manager>();
        mcg::host::TallyNodeMap to_tally;
        for (uint32_t i = 0; i < n_tally; ++i) {
            if (!to_tally.count(tally_indices[i])) m->order.push_back(tally_indices[i]);
            to_tally[tally_indices[i]] = mcg::host::TallyNode{1, {}};
        }
        mcg_run_desc r{};
        if (run) r = *run;
        m->mgr = std::make_unique<mcg::host::layer_manager>(
            p->pdag, num_trials, to_tally, overhead_ratio, r,
            max_words_per_iteration ? max_words_per_iteration : ((std::size_t)1 << 24));
        m->map = to_tally;
        *out = m.release();
        return MCG_OK;
    });
}

mcg_status mcg_manager_destroy(mcg_manager *m) {
    delete m;
    return MCG_OK;
}

mcg_status mcg_manager_single_pass(mcg_manager *m) {
    return guarded([&] {
        if (!m) return mcg::fail(MCG_ERR_INVALID, "manager is NULL");
        m->mgr->single_pass();
        return MCG_OK;
    });
}

mcg_status mcg_manager_pass(mcg_manager *m, uint64_t count) {
    return guarded([&] {
        if (!m) return mcg::fail(MCG_ERR_INVALID, "manager is NULL");
        m->mgr->pass(count);
        return MCG_OK;
    });
}

mcg_status mcg_manager_single_pass_and_tally(mcg_manager *m, int32_t index, mcg_tally *out) {
    return guarded([&] {
        if (!m || !out) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
        to_c(index, m->mgr->single_pass_and_tally(index), *out);
        return MCG_OK;
    });
}

mcg_status mcg_manager_pass_wait_collect(mcg_manager *m, uint64_t total, uint64_t between, mcg_tally *out,
                                         uint32_t capacity) {
    return guarded([&] {
        if (!m) return mcg::fail(MCG_ERR_INVALID, "manager is NULL");
        m->mgr->pass_wait_collect(m->map, total, between);
        return export_map(m, out, capacity);
    });
}

mcg_status mcg_manager_collect_tallies(mcg_manager *m, mcg_tally *out, uint32_t capacity) {
    return guarded([&] {
        if (!m) return mcg::fail(MCG_ERR_INVALID, "manager is NULL");
        m->mgr->collect_tallies(m->map);
        return export_map(m, out, capacity);
    });
}

mcg_status mcg_manager_node_count(mcg_manager *m, uint64_t *count) {
    return guarded([&] {
        if (!m || !count) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
        *count = m->mgr->node_count();
        return MCG_OK;
    });
}

mcg_status mcg_manager_shape(mcg_manager *m, uint64_t *bs, uint64_t *bpb, uint64_t *total_it) {
    return guarded([&] {
        if (!m) return mcg::fail(MCG_ERR_INVALID, "manager is NULL");
        const auto &sh = m->mgr->shaper();
        if (bs) *bs = sh.SAMPLE_SHAPE.batch_size;
        if (bpb) *bpb = sh.SAMPLE_SHAPE.bitpacks_per_batch;
        if (total_it) *total_it = sh.TOTAL_ITERATIONS;
        return MCG_OK;
    });
}

mcg_status mcg_manager_engine(mcg_manager *m, mcg_engine **engine) {
    return guarded([&] {
        if (!m || !engine) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
        *engine = m->mgr->engine();
        return MCG_OK;
    });
}

mcg_status mcg_run_to_convergence(mcg_manager *m, const mcg_settings *s, mcg_tally *out, uint32_t capacity,
                                  mcg_convergence_report *report) {
    return guarded([&] {
        if (!m || !s) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
        const auto t0 = std::chrono::steady_clock::now();
        mcg::host::convergence_controller c(*m->mgr, settings_from(s));
        c.run_to_convergence(m->map);
        m->mgr->collect_tallies(m->map);
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        fill_report(c, *m->mgr, secs, report);
        return export_map(m, out, capacity);
    });
}

mcg_status mcg_compute_tallies(const mcg_pdag *p, const mcg_settings *s, const int32_t *watch, uint32_t n_watch,
                               const mcg_run_desc *run, mcg_tally *out, mcg_convergence_report *report) {
    return guarded([&] {
        if (!p || !s || !out) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
        if (n_watch && !watch) return mcg::fail(MCG_ERR_INVALID, "watch is NULL");
        std::vector<int32_t> idx{p->pdag.root()};
        for (uint32_t i = 0; i < n_watch; ++i) idx.push_back(watch[i]);
        mcg_manager *m = nullptr;
        mcg_status st = mcg_manager_create(p, s->num_trials, idx.data(), (uint32_t)idx.size(), s->overhead_ratio, run,
                                           s->max_words_per_iteration, &m);
        if (st != MCG_OK) return st;
        std::unique_ptr<mcg_manager> hold(m);
        std::vector<mcg_tally> all(m->order.size());
        st = mcg_run_to_convergence(m, s, all.data(), (uint32_t)all.size(), report);
        if (st != MCG_OK) return st;
        for (size_t i = 0; i < idx.size(); ++i) {
            for (const auto &t : all)
                if (t.index == idx[i]) out[i] = t;
        }
        return MCG_OK;
    });
}

double mcg_normal_quantile_two_sided(double confidence) {
    return mcg::host::stats::normal_quantile_two_sided(confidence);
}

double mcg_beta_quantile(double a, double b, double q) { return mcg::host::stats::beta_quantile(a, b, q); }

mcg_status mcg_sample_shape(uint64_t num_trials, uint64_t max_words, uint64_t *words, uint64_t *total_it,
                            uint64_t *rounded) {
    return guarded([&] {
        mcg::host::sample_shaper sh(num_trials, 0, 0.0, max_words ? max_words : ((std::size_t)1 << 24));
        if (words) *words = sh.SAMPLE_SHAPE.num_bitpacks();
        if (total_it) *total_it = sh.TOTAL_ITERATIONS;
        if (rounded) *rounded = sh.num_trials;
        return MCG_OK;
    });
}

}  // extern "C"
