// host_manager.hpp -- C++ mirror of the reference's Monte Carlo engine API.
//
//   sample_shaper          src/mc/queue/sample_shaper.h:59-147
//   layer_manager          src/mc/queue/layer_manager.h:98-402 / .tpp
//   TallyNodeMap           src/mc/stats/tally_node_map.h (index -> tally)
//   convergence_controller src/mc/scheduler/convergence_controller.h
//
// Same names, argument meaning and error behaviour (exceptions) as the
// reference; the device work goes through the mcg_* C ABI (include/mcg.h).
#pragma once
#include <cstdint>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <vector>

#include "graph.hpp"
#include "host_pdag.hpp"
#include "host_stats.hpp"
#include "mcg.h"

namespace mcg {
namespace host {

struct sample_shape {
    std::size_t batch_size = 1;
    std::size_t bitpacks_per_batch = 1;
    std::size_t num_bitpacks() const { return batch_size * bitpacks_per_batch; }
};

// Picks words per pass and the pass count for a requested number of trials.
// Same rounding as the reference: trials to the nearest multiple of 64 (a
// remainder <= 32 rounds down), no request means 2^26 and no pass limit, and
// the words per pass are the power of two closest to the request (ties to the
// smaller) within the per-pass capacity, flattened to batch_size 1.  The
// reference's NVIDIA rule of filling the largest device allocation
// (sample_shaper.h:120-134) sizes materialised per-node buffers, which the
// fused kernel does not have; the per-pass capacity here is a parameter.
struct sample_shaper {
    std::size_t TOTAL_ITERATIONS = 0;
    sample_shape SAMPLE_SHAPE{};
    std::size_t requested_num_trials = 0;
    std::size_t num_trials = 0;
    std::size_t bits_per_iteration = 0;
    std::size_t num_iterations = 0;

    sample_shaper() = default;
    sample_shaper(std::size_t requested, std::size_t num_nodes, double overhead_ratio,
                  std::size_t max_words_per_iteration);
};

struct TallyNode {
    int status = 0;  // 0 not tracked, 1 not converged, 2 converged
    stats::tally tally_stats{};
};

using TallyNodeMap = std::map<int32_t, TallyNode>;

// The drop-in engine: constructed from a PDAG, a trial budget and the nodes
// to tally; runs passes on the device and harvests tallies.
class layer_manager {
  public:
    layer_manager(const Pdag &pdag, std::size_t num_trials, const TallyNodeMap &to_tally, double overhead_ratio,
                  const mcg_run_desc &run = {}, std::size_t max_words_per_iteration = (std::size_t)1 << 24);
    ~layer_manager();
    layer_manager(const layer_manager &) = delete;
    layer_manager &operator=(const layer_manager &) = delete;

    void single_pass();
    void pass(std::size_t count);
    stats::tally single_pass_and_tally(int32_t evt_idx);
    TallyNodeMap &pass_wait_collect(TallyNodeMap &tallies, std::size_t total_passes = 1,
                                    std::size_t passes_between_waits = 0);
    TallyNodeMap &collect_tallies(TallyNodeMap &tallies);
    stats::tally fetch_tally_for_event_with_index(int32_t evt_idx);
    std::size_t node_count() const { return node_count_; }
    const sample_shaper &shaper() const { return shaper_; }
    uint32_t iteration() const { return iteration_; }
    // Asynchronous harvest: snapshot the counters behind the passes so far,
    // fold a snapshot into the map, and roll the engine back to a snapshot.
    void snapshot(uint32_t slot);
    TallyNodeMap &collect_snapshot(uint32_t slot, TallyNodeMap &tallies);
    void restore_snapshot(uint32_t slot, uint32_t iteration);
    mcg_engine *engine() const { return engine_; }
    const Graph &graph() const { return graph_; }
    // Position of a basic event in the layer-0 block (the counter's event_idx).
    uint32_t event_index(int32_t pdag_index) const;

  private:
    void wait();
    mcg_engine *engine_ = nullptr;
    Graph graph_;
    std::unordered_map<int32_t, uint32_t> flat_;
    std::vector<int32_t> tally_index_;  // PDAG index of every tally slot
    std::size_t node_count_ = 0;
    sample_shaper shaper_;
    uint32_t iteration_ = 0;  // passes submitted so far (the reference's iteration_)
};

struct settings {
    std::size_t num_trials = 0;
    bool early_stop = true;
    double ci_confidence = 0.99;
    double ci_rel_margin_error = 0.001;
    double ci_burnin_trials = 1 << 20;
    stats::policy ci_policy = stats::policy::bayes;
    double overhead_ratio = 0.05;
    double oracle_p = -1.0;
    bool pipelined = true;  // decide on pass k while pass k + 1 runs (same results)
};

class convergence_controller {
  public:
    convergence_controller(layer_manager &mgr, const settings &s);
    void process_tallies(TallyNodeMap &map);
    bool check_convergence() const { return eps_bounded() && log_eps_bounded(); }
    bool step(TallyNodeMap &map);
    bool burn_in_step(TallyNodeMap &map);
    stats::tally run_to_convergence(TallyNodeMap &map);
    stats::tally run_to_convergence_pipelined(TallyNodeMap &map);

    bool all_converged() const { return log10_converged_ && eps_converged_; }
    bool iteration_limit_reached() const;
    bool burn_in_complete() const { return current_trials_ >= settings_.ci_burnin_trials; }
    std::size_t current_trials() const { return current_trials_; }
    std::size_t projected_trials() const { return projected_trials_; }
    double epsilon() const { return cur_eps_; }
    double epsilon_log10() const { return cur_eps_log10_; }
    double target_epsilon() const { return target_eps_; }
    double target_epsilon_log10() const { return settings_.ci_rel_margin_error; }
    double info_gain_cumulative() const { return gain_.cumulative_bits(); }
    bool epsilon_converged() const { return eps_converged_; }
    bool epsilon_log10_converged() const { return log10_converged_; }
    bool fixed_iteration_limit_reached() const { return fixed_limit_reached_; }
    std::size_t steps() const { return steps_; }
    std::size_t burn_in_steps() const { return burn_in_steps_; }
    const stats::tally &current_tally() const { return current_tally_; }

  private:
    enum class phase { none, burn_in, step };
    phase next_pass();  // the phase of the pass the synchronous loop would run next (none: stop)
    void after_pass(phase p);
    bool stops_after(std::size_t trials) const;
    bool eps_bounded() const { return cur_eps_ > 0 && cur_eps_ <= target_eps_; }
    bool log_eps_bounded() const { return cur_eps_log10_ > 0 && cur_eps_log10_ <= settings_.ci_rel_margin_error; }
    layer_manager &manager_;
    settings settings_;
    double z_ = 0.0;
    double cur_eps_ = 0.0, cur_eps_log10_ = 0.0, target_eps_ = 0.0;
    std::size_t current_trials_ = 0, projected_trials_ = 0;
    stats::info_gain gain_{};
    std::size_t prev_ones_ = 0, prev_total_ = 0;
    bool eps_converged_ = false, log10_converged_ = false, fixed_limit_reached_ = false;
    std::size_t steps_ = 0, burn_in_steps_ = 0;
    stats::tally current_tally_{};
};

}  // namespace host
}  // namespace mcg
