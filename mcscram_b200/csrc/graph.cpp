// graph.cpp -- validation of flattened PDAGs handed across the C ABI.
//
// The reference rejects unknown inputs by logging and exiting
// (src/mc/queue/kernel_builder.h:340-342, 358-361, 712-726); here the same
// conditions come back as an error string and MCG_ERR_INVALID.
#include "graph.hpp"

#include <cstring>

namespace mcg {

std::string Graph::from_desc(const mcg_graph_desc &d, Graph &g) {
    g = Graph{};
    if (d.n_be > 0 && (!d.be_pdag_idx || !d.be_event_idx || !d.be_threshold))
        return "basic-event arrays must not be NULL when n_be > 0";
    if (d.n_gates > 0 && (!d.gate_op || !d.gate_k || !d.gate_in_begin || !d.gate_in_count || !d.gate_neg_count))
        return "gate arrays must not be NULL when n_gates > 0";
    if (d.n_inputs > 0 && !d.inputs) return "inputs must not be NULL when n_inputs > 0";
    if (d.n_tally > 0 && !d.tally_nodes) return "tally_nodes must not be NULL when n_tally > 0";
    if ((uint64_t)d.n_be + (uint64_t)d.n_gates >= (uint64_t)1 << 31) return "too many nodes";
    g.n_be = d.n_be;
    g.n_gates = d.n_gates;
    g.be_pdag_idx.assign(d.be_pdag_idx, d.be_pdag_idx + d.n_be);
    g.be_event_idx.assign(d.be_event_idx, d.be_event_idx + d.n_be);
    g.be_threshold.assign(d.be_threshold, d.be_threshold + d.n_be);
    if (d.gate_pdag_idx)
        g.gate_pdag_idx.assign(d.gate_pdag_idx, d.gate_pdag_idx + d.n_gates);
    else
        g.gate_pdag_idx.assign(d.n_gates, -1);
    g.gate_op.assign(d.gate_op, d.gate_op + d.n_gates);
    g.gate_k.assign(d.gate_k, d.gate_k + d.n_gates);
    g.gate_in_begin.assign(d.gate_in_begin, d.gate_in_begin + d.n_gates);
    g.gate_in_count.assign(d.gate_in_count, d.gate_in_count + d.n_gates);
    g.gate_neg_count.assign(d.gate_neg_count, d.gate_neg_count + d.n_gates);
    g.inputs.assign(d.inputs, d.inputs + d.n_inputs);
    g.tally_nodes.assign(d.tally_nodes, d.tally_nodes + d.n_tally);
    return g.validate();
}

std::string Graph::validate() const {
    const uint64_t nn = (uint64_t)n_be + n_gates;
    for (uint32_t e = 0; e < n_be; ++e) {
        if (be_threshold[e] > ((uint64_t)1 << 32))
            return "basic event " + std::to_string(e) + ": threshold above 2^32";
    }
    for (uint32_t g = 0; g < n_gates; ++g) {
        if (gate_op[g] > MCG_NULL) return "gate " + std::to_string(g) + ": unknown connective";
        if (gate_neg_count[g] > gate_in_count[g])
            return "gate " + std::to_string(g) + ": neg_count exceeds in_count";
        const uint64_t end = (uint64_t)gate_in_begin[g] + gate_in_count[g];
        if (end > inputs.size()) return "gate " + std::to_string(g) + ": inputs out of range";
        for (uint64_t i = gate_in_begin[g]; i < end; ++i) {
            if (inputs[i] >= (uint64_t)n_be + g)
                return "gate " + std::to_string(g) + ": input " + std::to_string(inputs[i]) +
                       " is not an earlier node (unknown input or not topologically ordered)";
        }
    }
    for (uint32_t t : tally_nodes)
        if (t >= nn) return "tally node " + std::to_string(t) + " out of range";
    return {};
}

}  // namespace mcg
