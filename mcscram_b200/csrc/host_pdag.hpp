// host_pdag.hpp -- the caller-side PDAG and the reference's layering.
//
// A minimal stand-in for core::Pdag (mcSCRAM src/pdag.h:246-298, 802+): nodes
// are Variables (basic events, index >= 2) and Gates with a connective, a
// min_number (ATLEAST k) and signed argument indices (negative = complement),
// kept per argument type in insertion order like Gate::args<Gate>() and
// Gate::args<Variable>().
//
// layered_toposort() reproduces layer_manager::layered_toposort
// (src/mc/queue/layer_manager.tpp:63-118) step by step, so the position of a
// basic event in the layer-0 block -- its event_idx, counter word 1 of every
// Philox draw -- comes out as the reference assigns it:
//   1. LayeredTopologicalOrder (src/preprocessor.cc:130-171): variables get
//      order 0, a gate 1 + the largest order of its arguments;
//   2. gather_all_nodes (tpp:34-60): depth-first from the root, a gate before
//      its gate arguments, then its not yet visited variable arguments;
//   3. std::sort of that list by order, bucketing by order, then a std::sort
//      of every bucket with "variables first, gates by connective, variables
//      all equivalent".  The same libstdc++ std::sort on the same sequence
//      with the same comparator yields the same (unstable) permutation.
#pragma once
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "graph.hpp"

namespace mcg {
namespace host {

struct PdagNode {
    int32_t index = 0;
    bool is_variable = false;
    double probability = 0.0;           // variables
    uint8_t connective = 0;             // gates
    uint32_t min_number = 0;            // gates (ATLEAST k)
    std::vector<int32_t> args;          // signed indices in insertion order
};

struct Layering {
    std::vector<std::vector<int32_t>> nodes_by_layer;  // PDAG indices per order value
    std::vector<int32_t> gather_order;                 // depth-first gather sequence
};

class Pdag {
  public:
    std::string add_variable(int32_t index, double probability);
    std::string add_gate(int32_t index, uint8_t connective, uint32_t min_number, const int32_t *args, uint32_t n_args);
    std::string set_root(int32_t index);
    int32_t root() const { return root_; }
    size_t size() const { return nodes_.size(); }
    const PdagNode *find(int32_t index) const;
    std::string set_probability(int32_t index, double p);

    // Layers the graph as the reference's layer_manager does.
    std::string layered_toposort(Layering &out) const;

    // Flattens the layered graph for the engine: basic events in layer-0
    // order (event_idx = position), gates layer by layer in the sorted order,
    // each gate's inputs as kernel_builder.h:324-379 lays them out (variable
    // arguments, then gate arguments; complemented ones moved to the tail).
    // tally_indices are PDAG indices; flat_index maps every gathered PDAG
    // index to its flat node id.
    std::string flatten(const std::vector<int32_t> &tally_indices, Graph &out,
                        std::unordered_map<int32_t, uint32_t> *flat_index = nullptr,
                        Layering *layering = nullptr) const;

  private:
    std::vector<PdagNode> nodes_;
    std::unordered_map<int32_t, size_t> by_index_;
    int32_t root_ = 0;
};

}  // namespace host
}  // namespace mcg
