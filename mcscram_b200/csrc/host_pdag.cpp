// host_pdag.cpp -- caller-side PDAG, reference layering, flattening.
#include "host_pdag.hpp"

#include <algorithm>
#include <cmath>
#include <functional>

#include "mcg.h"

namespace mcg {
namespace host {

std::string Pdag::add_variable(int32_t index, double probability) {
    if (index < 2) return "variable index must be >= 2 (kVariableStartIndex)";
    if (by_index_.count(index)) return "duplicate node index " + std::to_string(index);
    if (!(probability >= 0.0 && probability <= 1.0)) return "probability outside [0, 1]";
    PdagNode n;
    n.index = index;
    n.is_variable = true;
    n.probability = probability;
    by_index_[index] = nodes_.size();
    nodes_.push_back(std::move(n));
    return {};
}

std::string Pdag::add_gate(int32_t index, uint8_t connective, uint32_t min_number, const int32_t *args,
                           uint32_t n_args) {
    if (index < 1) return "gate index must be positive";
    if (by_index_.count(index)) return "duplicate node index " + std::to_string(index);
    if (connective > MCG_NULL) return "unknown connective";
    if (n_args && !args) return "args must not be NULL";
    PdagNode n;
    n.index = index;
    n.connective = connective;
    n.min_number = min_number;
    n.args.assign(args, args + n_args);
    for (int32_t a : n.args)
        if (a == 0) return "argument index 0 is not a node";
    by_index_[index] = nodes_.size();
    nodes_.push_back(std::move(n));
    return {};
}

std::string Pdag::set_root(int32_t index) {
    auto it = by_index_.find(index);
    if (it == by_index_.end()) return "unknown root index";
    if (nodes_[it->second].is_variable) return "root must be a gate";
    root_ = index;
    return {};
}

std::string Pdag::set_probability(int32_t index, double p) {
    auto it = by_index_.find(index);
    if (it == by_index_.end() || !nodes_[it->second].is_variable) return "unknown variable index";
    if (!(p >= 0.0 && p <= 1.0)) return "probability outside [0, 1]";
    nodes_[it->second].probability = p;
    return {};
}

const PdagNode *Pdag::find(int32_t index) const {
    auto it = by_index_.find(index);
    return it == by_index_.end() ? nullptr : &nodes_[it->second];
}

std::string Pdag::layered_toposort(Layering &out) const {
    out = Layering{};
    if (!root_) return "root not set";
    // 1. Orders (depths), memoised.
    std::unordered_map<int32_t, int> depth;
    std::string err;
    std::function<int(const PdagNode &, int)> compute = [&](const PdagNode &n, int guard) -> int {
        auto it = depth.find(n.index);
        if (it != depth.end()) return it->second;
        if (n.is_variable) {
            depth[n.index] = 0;
            return 0;
        }
        if (guard > (int)nodes_.size()) {
            err = "cycle in the PDAG";
            return 0;
        }
        int m = -1;
        // variable arguments first, then gate arguments (preprocessor.cc:150-162)
        for (int pass = 0; pass < 2; ++pass) {
            for (int32_t a : n.args) {
                const PdagNode *c = find(a < 0 ? -a : a);
                if (!c) {
                    err = "unknown argument " + std::to_string(a) + " of gate " + std::to_string(n.index);
                    return 0;
                }
                if (c->is_variable != (pass == 0)) continue;
                m = std::max(m, compute(*c, guard + 1));
            }
        }
        depth[n.index] = m + 1;
        return m + 1;
    };
    compute(*find(root_), 0);
    if (!err.empty()) return err;

    // 2. gather_all_nodes: gate, its gate args (recursively), its unvisited variable args.
    std::unordered_map<int32_t, uint8_t> visited;
    std::vector<int32_t> nodes;
    std::function<void(const PdagNode &)> gather = [&](const PdagNode &g) {
        if (visited[g.index]) return;
        visited[g.index] = 1;
        nodes.push_back(g.index);
        for (int32_t a : g.args) {
            const PdagNode *c = find(a < 0 ? -a : a);
            if (!c->is_variable) gather(*c);
        }
        for (int32_t a : g.args) {
            const PdagNode *c = find(a < 0 ? -a : a);
            if (c->is_variable && !visited[c->index]) {
                visited[c->index] = 1;
                nodes.push_back(c->index);
            }
        }
    };
    gather(*find(root_));
    out.gather_order = nodes;

    // 3. std::sort by order, bucket, std::sort each bucket.
    std::sort(nodes.begin(), nodes.end(), [&](int32_t a, int32_t b) { return depth[a] < depth[b]; });
    const int max_layer = depth[nodes.back()];
    out.nodes_by_layer.assign((size_t)max_layer + 1, {});
    for (int32_t v : nodes) out.nodes_by_layer[(size_t)depth[v]].push_back(v);
    for (auto &layer : out.nodes_by_layer) {
        std::sort(layer.begin(), layer.end(), [&](int32_t l, int32_t r) {
            const PdagNode *a = find(l), *b = find(r);
            if (a->is_variable && !b->is_variable) return true;
            if (!a->is_variable && b->is_variable) return false;
            if (a->is_variable && b->is_variable) return false;
            return a->connective < b->connective;
        });
    }
    return {};
}

std::string Pdag::flatten(const std::vector<int32_t> &tally_indices, Graph &g,
                          std::unordered_map<int32_t, uint32_t> *flat_index_out, Layering *layering_out) const {
    Layering lay;
    std::string err = layered_toposort(lay);
    if (!err.empty()) return err;
    g = Graph{};
    std::unordered_map<int32_t, uint32_t> flat;
    // basic events: every variable in layer 0 (variables only ever sit there)
    for (int32_t v : lay.nodes_by_layer[0]) {
        const PdagNode *n = find(v);
        if (!n->is_variable) return "internal: gate in layer 0";
        flat[v] = g.n_be;
        g.be_pdag_idx.push_back(v);
        g.be_event_idx.push_back(g.n_be);
        g.be_threshold.push_back(probability_threshold(n->probability));
        ++g.n_be;
    }
    uint32_t next = g.n_be;
    for (size_t l = 1; l < lay.nodes_by_layer.size(); ++l)
        for (int32_t v : lay.nodes_by_layer[l]) flat[v] = next++;
    for (size_t l = 1; l < lay.nodes_by_layer.size(); ++l) {
        for (int32_t v : lay.nodes_by_layer[l]) {
            const PdagNode *n = find(v);
            if (n->is_variable) return "internal: variable above layer 0";
            std::vector<uint32_t> pos, neg;
            for (int pass = 0; pass < 2; ++pass) {  // variable args, then gate args
                for (int32_t a : n->args) {
                    const PdagNode *c = find(a < 0 ? -a : a);
                    if (c->is_variable != (pass == 0)) continue;
                    (a < 0 ? neg : pos).push_back(flat.at(c->index));
                }
            }
            g.gate_pdag_idx.push_back(v);
            g.gate_op.push_back(n->connective);
            g.gate_k.push_back(n->min_number);
            g.gate_in_begin.push_back((uint32_t)g.inputs.size());
            g.gate_in_count.push_back((uint32_t)(pos.size() + neg.size()));
            g.gate_neg_count.push_back((uint32_t)neg.size());
            g.inputs.insert(g.inputs.end(), pos.begin(), pos.end());
            g.inputs.insert(g.inputs.end(), neg.begin(), neg.end());
            ++g.n_gates;
        }
    }
    for (int32_t t : tally_indices) {
        auto it = flat.find(t);
        if (it == flat.end()) return "Attempting to build tally for unknown event " + std::to_string(t);
        g.tally_nodes.push_back(it->second);
    }
    err = g.validate();
    if (!err.empty()) return "internal: " + err;
    if (flat_index_out) *flat_index_out = std::move(flat);
    if (layering_out) *layering_out = std::move(lay);
    return {};
}

}  // namespace host
}  // namespace mcg
