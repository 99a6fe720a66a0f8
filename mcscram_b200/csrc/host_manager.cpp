// host_manager.cpp -- sample_shaper, layer_manager and convergence_controller.
#include "host_manager.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

namespace mcg {
namespace host {

namespace {

void throw_status(mcg_status st, const char *what) {
    if (st == MCG_OK) return;
    const std::string msg = std::string(what) + ": " + mcg_last_error();
    if (st == MCG_ERR_INVALID) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

}  // namespace

// sample_shaper.h:59-147 (see the class comment for the capacity rule).
sample_shaper::sample_shaper(std::size_t requested, std::size_t num_nodes, double overhead_ratio,
                             std::size_t max_words_per_iteration) {
    (void)num_nodes;
    (void)overhead_ratio;
    requested_num_trials = requested;
    const bool no_limits = requested == 0;
    std::size_t req = no_limits ? (std::size_t)64 * 1024 * 1024 : requested;
    const std::size_t rem = req % 64;
    num_trials = rem == 0 ? req : (rem <= 32 ? req - rem : req + 64 - rem);
    const std::size_t total_bits = num_trials;
    const std::size_t cap_bits = std::max<std::size_t>(max_words_per_iteration, 1) * 64;
    const std::size_t target_bits = std::min(total_bits, cap_bits);
    const std::size_t target_words = (target_bits + 63) / 64;
    const std::size_t max_words = cap_bits / 64;
    std::size_t best = 1, best_diff = std::numeric_limits<std::size_t>::max();
    for (std::size_t p = 1; p && p <= max_words; p <<= 1) {
        const std::size_t diff = p > target_words ? p - target_words : target_words - p;
        if (diff < best_diff || (diff == best_diff && p < best)) {
            best_diff = diff;
            best = p;
        }
        if (best_diff == 0) break;
    }
    SAMPLE_SHAPE.batch_size = 1;
    SAMPLE_SHAPE.bitpacks_per_batch = best;
    bits_per_iteration = best * 64;
    num_iterations = (std::size_t)std::ceil((double)total_bits / (double)bits_per_iteration);
    TOTAL_ITERATIONS = no_limits ? 0 : num_iterations;
}

// layer_manager.tpp:345-375
layer_manager::layer_manager(const Pdag &pdag, std::size_t num_trials, const TallyNodeMap &to_tally,
                             double overhead_ratio, const mcg_run_desc &run, std::size_t max_words_per_iteration) {
    std::vector<int32_t> tally_indices;
    for (const auto &kv : to_tally) tally_indices.push_back(kv.first);
    const std::string err = pdag.flatten(tally_indices, graph_, &flat_);
    if (!err.empty()) throw std::runtime_error("layer_manager: " + err);
    tally_index_ = tally_indices;
    node_count_ = graph_.n_nodes();
    shaper_ = sample_shaper(num_trials, node_count_, overhead_ratio, max_words_per_iteration);
    mcg_graph_desc d{};
    d.n_be = graph_.n_be;
    d.n_gates = graph_.n_gates;
    d.be_pdag_idx = graph_.be_pdag_idx.data();
    d.be_event_idx = graph_.be_event_idx.data();
    d.be_threshold = graph_.be_threshold.data();
    d.gate_pdag_idx = graph_.gate_pdag_idx.data();
    d.gate_op = graph_.gate_op.data();
    d.gate_k = graph_.gate_k.data();
    d.gate_in_begin = graph_.gate_in_begin.data();
    d.gate_in_count = graph_.gate_in_count.data();
    d.gate_neg_count = graph_.gate_neg_count.data();
    d.inputs = graph_.inputs.data();
    d.n_inputs = graph_.inputs.size();
    d.n_tally = (uint32_t)graph_.tally_nodes.size();
    d.tally_nodes = graph_.tally_nodes.data();
    mcg_run_desc r = run;
    if (r.mode == MCG_MODE_AUTO && !r.tune_pass_words) r.tune_pass_words = shaper_.SAMPLE_SHAPE.num_bitpacks();
    throw_status(mcg_create(&d, &r, &engine_), "layer_manager");
}

layer_manager::~layer_manager() {
    if (engine_) mcg_destroy(engine_);
}

uint32_t layer_manager::event_index(int32_t pdag_index) const {
    auto it = flat_.find(pdag_index);
    if (it == flat_.end() || it->second >= graph_.n_be)
        throw std::runtime_error("event_index: unknown basic event " + std::to_string(pdag_index));
    return graph_.be_event_idx[it->second];
}

// layer_manager.tpp:203-208 / queueable.h:725-731: every submitted pass
// increments the iteration, starting from 1.
void layer_manager::single_pass() {
    ++iteration_;
    throw_status(mcg_run(engine_, iteration_, 1, 0, shaper_.SAMPLE_SHAPE.num_bitpacks()), "single_pass");
}

void layer_manager::pass(std::size_t count) {
    for (std::size_t i = 0; i < count; ++i) single_pass();
}

void layer_manager::wait() { throw_status(mcg_synchronize(engine_), "wait_and_throw"); }

stats::tally layer_manager::fetch_tally_for_event_with_index(int32_t evt_idx) {
    stats::tally t;
    auto pos = std::find(tally_index_.begin(), tally_index_.end(), evt_idx);
    if (pos == tally_index_.end()) return t;  // reference logs and returns an empty tally
    std::vector<uint64_t> ones(tally_index_.size());
    uint64_t total = 0;
    throw_status(mcg_read_tallies(engine_, ones.data(), &total), "collect_tallies");
    t.num_one_bits = ones[(size_t)(pos - tally_index_.begin())];
    t.total_bits = total;
    stats::tally::compute_ci(stats::tally::compute_moments(t));
    return t;
}

stats::tally layer_manager::single_pass_and_tally(int32_t evt_idx) {
    single_pass();
    wait();
    return fetch_tally_for_event_with_index(evt_idx);
}

// layer_manager.tpp:226-267
TallyNodeMap &layer_manager::pass_wait_collect(TallyNodeMap &tallies, std::size_t total_passes,
                                               std::size_t passes_between_waits) {
    if (total_passes == 0) throw std::invalid_argument("pass_wait_collect: total_passes must be greater than 0");
    const std::size_t interval = passes_between_waits == 0 ? total_passes : passes_between_waits;
    std::size_t remaining = total_passes;
    while (remaining > 0) {
        const std::size_t batch = std::min(interval, remaining);
        pass(batch);
        wait();
        remaining -= batch;
    }
    return collect_tallies(tallies);
}

// layer_manager.tpp:271-279
TallyNodeMap &layer_manager::collect_tallies(TallyNodeMap &tallies) {
    std::vector<uint64_t> ones(tally_index_.size());
    uint64_t total = 0;
    throw_status(mcg_read_tallies(engine_, ones.data(), &total), "collect_tallies");
    for (size_t i = 0; i < tally_index_.size(); ++i) tallies[tally_index_[i]].tally_stats.update(ones[i], total);
    return tallies;
}

void layer_manager::snapshot(uint32_t slot) { throw_status(mcg_snapshot_tallies(engine_, slot), "snapshot"); }

TallyNodeMap &layer_manager::collect_snapshot(uint32_t slot, TallyNodeMap &tallies) {
    std::vector<uint64_t> ones(tally_index_.size());
    uint64_t total = 0;
    throw_status(mcg_snapshot_read(engine_, slot, ones.data(), &total), "collect_snapshot");
    for (size_t i = 0; i < tally_index_.size(); ++i) tallies[tally_index_[i]].tally_stats.update(ones[i], total);
    return tallies;
}

void layer_manager::restore_snapshot(uint32_t slot, uint32_t iteration) {
    std::vector<uint64_t> ones(std::max<size_t>(tally_index_.size(), 1));
    uint64_t total = 0;
    throw_status(mcg_snapshot_read(engine_, slot, ones.data(), &total), "restore_snapshot");
    throw_status(mcg_set_tallies(engine_, ones.data(), total), "restore_snapshot");
    iteration_ = iteration;
}

// ------------------------------------------------------------------ controller

convergence_controller::convergence_controller(layer_manager &mgr, const settings &s) : manager_(mgr), settings_(s) {
    z_ = stats::normal_quantile_two_sided(settings_.ci_confidence);
    cur_eps_ = std::numeric_limits<double>::infinity();
    cur_eps_log10_ = std::numeric_limits<double>::infinity();
    target_eps_ = settings_.ci_rel_margin_error * std::max(0.0, stats::kDeltaEpsilon);
    projected_trials_ = settings_.num_trials;
}

// convergence_controller.h:143-250: worst case over every monitored tally.
void convergence_controller::process_tallies(TallyNodeMap &map) {
    if (map.empty()) return;
    double max_eps = 0.0, max_eps_log10 = 0.0;
    std::size_t max_n1 = 0, max_n2 = 0, sum_ones = 0, sum_total = 0, max_total = 0;
    const stats::tally *worst = nullptr;
    for (auto &kv : map) {
        stats::tally &t = kv.second.tally_stats;
        stats::update_convergence(settings_.ci_policy, t, settings_.ci_rel_margin_error, z_);
        if (t.linear.epsilon > max_eps) {
            max_eps = t.linear.epsilon;
            worst = &t;
        }
        max_eps_log10 = std::max(max_eps_log10, t.log10.epsilon);
        max_n1 = std::max(max_n1, t.linear.target_trials);
        max_n2 = std::max(max_n2, t.log10.target_trials);
        sum_ones += t.num_one_bits;
        sum_total += t.total_bits;
        max_total = std::max(max_total, t.total_bits);
    }
    // The reference only advances the trial count through the worst tally; when
    // every half-width is 0 (Wald with no ones anywhere) it would never leave
    // burn-in, so the trial count falls back to the tallies' own count.
    current_trials_ = worst ? worst->total_bits : max_total;
    cur_eps_ = max_eps;
    cur_eps_log10_ = max_eps_log10;
    if (worst) target_eps_ = settings_.ci_rel_margin_error * std::max(worst->mean, stats::kDeltaEpsilon);
    projected_trials_ = std::max(max_n1, max_n2);
    const std::size_t ds = sum_ones - prev_ones_;
    const std::size_t df = (sum_total - sum_ones) - (prev_total_ - prev_ones_);
    gain_.add_batch(ds, df);
    prev_ones_ = sum_ones;
    prev_total_ = sum_total;
    if (worst) current_tally_ = *worst;
}

bool convergence_controller::iteration_limit_reached() const {
    const std::size_t max_it = manager_.shaper().TOTAL_ITERATIONS;
    const std::size_t per = manager_.shaper().SAMPLE_SHAPE.num_bitpacks() * 64;
    const std::size_t iterations = (current_trials_ + per - 1) / per;
    return max_it && iterations >= max_it;
}

// convergence_controller.h:294-328
bool convergence_controller::step(TallyNodeMap &map) {
    if (all_converged() && settings_.early_stop) return false;
    if (!fixed_limit_reached_ && iteration_limit_reached()) {
        fixed_limit_reached_ = true;
        return false;
    }
    process_tallies(manager_.pass_wait_collect(map));
    if (!eps_converged_ && eps_bounded()) eps_converged_ = true;
    if (!log10_converged_ && log_eps_bounded()) log10_converged_ = true;
    ++steps_;
    return true;
}

// convergence_controller.h:351-365
bool convergence_controller::burn_in_step(TallyNodeMap &map) {
    if (burn_in_complete()) return false;
    process_tallies(manager_.pass_wait_collect(map));
    ++burn_in_steps_;
    return true;
}

// convergence_controller.h:371-381
stats::tally convergence_controller::run_to_convergence(TallyNodeMap &map) {
    if (settings_.pipelined) return run_to_convergence_pipelined(map);
    while (burn_in_step(map)) {
    }
    while (step(map)) {
    }
    return current_tally_;
}

// The decision the synchronous loop takes before each pass: burn-in while
// the burn-in trials are not reached, then steps until converged (early
// stop) or the iteration limit.
convergence_controller::phase convergence_controller::next_pass() {
    if (!burn_in_complete()) return phase::burn_in;
    if (all_converged() && settings_.early_stop) return phase::none;
    if (!fixed_limit_reached_ && iteration_limit_reached()) {
        fixed_limit_reached_ = true;
        return phase::none;
    }
    return phase::step;
}

void convergence_controller::after_pass(phase p) {
    if (p == phase::burn_in) {
        ++burn_in_steps_;
        return;
    }
    if (!eps_converged_ && eps_bounded()) eps_converged_ = true;
    if (!log10_converged_ && log_eps_bounded()) log10_converged_ = true;
    ++steps_;
}

// True when the synchronous loop would stop after a pass that brings the
// trial count to `trials` whatever that pass's tallies say: burn-in done and
// the trial budget reached (next_pass() then returns none).
bool convergence_controller::stops_after(std::size_t trials) const {
    const std::size_t max_it = manager_.shaper().TOTAL_ITERATIONS;
    const std::size_t per = manager_.shaper().SAMPLE_SHAPE.num_bitpacks() * 64;
    if (!max_it || fixed_limit_reached_ || static_cast<double>(trials) < settings_.ci_burnin_trials) return false;
    return (trials + per - 1) / per >= max_it;
}

// The same decisions as run_to_convergence's synchronous loop, taken one
// pass behind the GPU: while the tallies after pass k are read and judged,
// pass k + 1 already runs.  When the loop stops after pass k, the pass run
// ahead is discarded by rolling the counters, their total and the pass
// number back to the snapshot after pass k, so tallies, statistics and
// stopping point equal the synchronous loop's; the cost is one pass of GPU
// time that nobody uses -- except where the trial budget already says the
// pass in flight is the last one, when no pass is run ahead.  Pass k's
// snapshot sits in slot (k - 1) & 1.
stats::tally convergence_controller::run_to_convergence_pipelined(TallyNodeMap &map) {
    phase p = next_pass();
    if (p == phase::none) return current_tally_;
    const std::size_t per = manager_.shaper().SAMPLE_SHAPE.num_bitpacks() * 64;
    const uint32_t base = manager_.iteration();
    uint32_t done = 0, submitted = 0;        // passes judged, passes queued
    auto submit = [&] {
        manager_.single_pass();
        manager_.snapshot(submitted & 1u);
        ++submitted;
    };
    submit();                                // pass 1
    for (;;) {
        if (submitted == done + 1 && !stops_after(current_trials_ + per)) submit();  // ahead of the decision
        process_tallies(manager_.collect_snapshot(done & 1u, map));
        ++done;
        after_pass(p);
        p = next_pass();
        if (p == phase::none) break;
        if (submitted == done) submit();     // the budget said stop, the loop did not
    }
    if (submitted > done) manager_.restore_snapshot((done - 1) & 1u, base + done);
    return current_tally_;
}

}  // namespace host
}  // namespace mcg
