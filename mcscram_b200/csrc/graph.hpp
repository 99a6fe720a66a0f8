// graph.hpp -- host copy of a flattened PDAG (the mcg_graph_desc of mcg.h).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "mcg.h"

namespace mcg {

struct Graph {
    uint32_t n_be = 0;
    uint32_t n_gates = 0;
    std::vector<int32_t> be_pdag_idx;
    std::vector<uint32_t> be_event_idx;
    std::vector<uint64_t> be_threshold;
    std::vector<int32_t> gate_pdag_idx;
    std::vector<uint8_t> gate_op;
    std::vector<uint32_t> gate_k;
    std::vector<uint32_t> gate_in_begin;
    std::vector<uint32_t> gate_in_count;
    std::vector<uint32_t> gate_neg_count;
    std::vector<uint32_t> inputs;
    std::vector<uint32_t> tally_nodes;

    uint32_t n_nodes() const { return n_be + n_gates; }

    // Copies and validates a descriptor.  Returns an empty string on success,
    // otherwise the reason the graph is rejected.
    static std::string from_desc(const mcg_graph_desc &d, Graph &out);
    std::string validate() const;
};

// Threshold of a probability exactly like the reference's basic-event block
// (src/mc/event/node.h:372-376): (uint64)(p * 2^32), truncated.
inline uint64_t probability_threshold(double p) { return (uint64_t)(p * 4294967296.0); }

}  // namespace mcg
