// program.cpp -- schedule and slot allocation for the fused kernel's program.
//
// The reference evaluates the PDAG layer by layer with every node's words
// materialised in device memory (src/mc/queue/layer_manager.tpp:143-164,
// 203-208).  Here the same node values are computed per sample word in a
// depth-first order that keeps few values alive at once:
//   * a gate's operands are produced right before it, the operand needing
//     the most slots first (Sethi-Ullman order);
//   * a basic event used once, and not tallied, is sampled directly into its
//     consumer's accumulator;
//   * basic events with probability 0 or 1 are constant words and need no
//     sampling at all (u < 0 never holds, u < 2^32 always does);
//   * NOT / NULL gates read only their last input, as the reference kernel's
//     "result = val" loop does (src/mc/kernel/gate.h:325-351).
// Live values get shared-memory slots by linear scan; when none is free, the
// value with the furthest last use is moved to a global scratch slot for its
// whole lifetime (no spill/reload ops are needed).
#include "program.hpp"

#include <algorithm>
#include <queue>

namespace mcg {
namespace {

constexpr uint64_t kFullThreshold = (uint64_t)1 << 32;

enum class BeKind : uint8_t { kUnused, kConst, kInline, kDef };

struct EffectiveInputs {
    uint32_t begin = 0, count = 0;  // range in Graph::inputs
    uint32_t neg_from = 0;          // index (within the range) where negated inputs start
};

EffectiveInputs effective_inputs(const Graph &g, uint32_t gi) {
    EffectiveInputs e;
    const uint32_t n = g.gate_in_count[gi];
    const uint32_t off = n - g.gate_neg_count[gi];
    const uint8_t op = g.gate_op[gi];
    if ((op == MCG_NOT || op == MCG_NULL) && n > 1) {
        // Only the last input determines the result.
        e.begin = g.gate_in_begin[gi] + n - 1;
        e.count = 1;
        e.neg_from = (n - 1 >= off) ? 0u : 1u;
    } else {
        e.begin = g.gate_in_begin[gi];
        e.count = n;
        e.neg_from = off;
    }
    return e;
}

uint32_t counter_bits(uint32_t n_inputs) {
    uint32_t b = 0;
    while (b < 8 && (n_inputs >> b) != 0) ++b;
    return b == 0 ? 1u : b;
}

Op make_op(uint32_t w0, uint32_t w1 = 0, uint32_t w2 = 0, uint32_t w3 = 0) {
    Op o;
    o.w[0] = w0;
    o.w[1] = w1;
    o.w[2] = w2;
    o.w[3] = w3;
    return o;
}

}  // namespace

std::string compile_program(const Graph &g, uint32_t smem_slot_budget, Program &out, bool variable_thresholds) {
    out = Program{};
    const uint32_t nb = g.n_be;
    const uint32_t nn = g.n_nodes();

    // 1. Nodes some tally depends on.
    std::vector<uint8_t> needed(nn, 0);
    {
        std::vector<uint32_t> stack(g.tally_nodes.begin(), g.tally_nodes.end());
        while (!stack.empty()) {
            const uint32_t v = stack.back();
            stack.pop_back();
            if (needed[v]) continue;
            needed[v] = 1;
            if (v >= nb) {
                const EffectiveInputs e = effective_inputs(g, v - nb);
                for (uint32_t i = 0; i < e.count; ++i) {
                    const uint32_t c = g.inputs[e.begin + i];
                    if (!needed[c]) stack.push_back(c);
                }
            }
        }
    }

    // 2. Uses and tallies.
    std::vector<uint32_t> uses(nn, 0);
    for (uint32_t gi = 0; gi < g.n_gates; ++gi) {
        if (!needed[nb + gi]) continue;
        const EffectiveInputs e = effective_inputs(g, gi);
        for (uint32_t i = 0; i < e.count; ++i) ++uses[g.inputs[e.begin + i]];
    }
    std::vector<std::vector<uint32_t>> tally_of(nn);
    for (uint32_t t = 0; t < (uint32_t)g.tally_nodes.size(); ++t) tally_of[g.tally_nodes[t]].push_back(t);

    std::vector<BeKind> kind(nb, BeKind::kUnused);
    for (uint32_t e = 0; e < nb; ++e) {
        if (!needed[e]) continue;
        const uint64_t thr = g.be_threshold[e];
        if (!variable_thresholds && (thr == 0 || thr >= kFullThreshold))
            kind[e] = BeKind::kConst;
        else if (uses[e] == 1 && tally_of[e].empty())
            kind[e] = BeKind::kInline;
        else
            kind[e] = BeKind::kDef;
    }
    auto is_slot_value = [&](uint32_t v) { return v >= nb || kind[v] == BeKind::kDef; };

    // 3. Slot need (Sethi-Ullman number, sharing ignored).
    std::vector<uint32_t> need(nn, 0);
    for (uint32_t v = 0; v < nn; ++v) {
        if (!needed[v]) continue;
        if (v < nb) {
            need[v] = (kind[v] == BeKind::kDef) ? 1u : 0u;
            continue;
        }
        const EffectiveInputs e = effective_inputs(g, v - nb);
        std::vector<uint32_t> cn;
        for (uint32_t i = 0; i < e.count; ++i) {
            const uint32_t c = g.inputs[e.begin + i];
            if (is_slot_value(c)) cn.push_back(need[c]);
        }
        std::sort(cn.rbegin(), cn.rend());
        uint32_t m = 1;
        for (uint32_t i = 0; i < (uint32_t)cn.size(); ++i) m = std::max(m, cn[i] + i);
        need[v] = m;
    }

    // 4. Depth-first emission.
    std::vector<Op> &ops = out.ops;
    std::vector<uint8_t> done(nn, 0);
    std::vector<std::pair<size_t, uint32_t>> def_sites;  // (op index, node)
    std::vector<std::pair<size_t, uint32_t>> use_sites;  // (op index, node)

    auto emit_tallies = [&](uint32_t v) {
        for (uint32_t t : tally_of[v]) ops.push_back(make_op(kOpTally, t));
    };
    auto emit_be_def = [&](uint32_t e) {
        if (kind[e] == BeKind::kConst) {
            // Only reached for tallied constant events; their uses read IN_CONST.
            const uint64_t val = (g.be_threshold[e] == 0) ? 0ull : ~0ull;
            ops.push_back(make_op(kOpConstDef | (kNoSlot << 8), (uint32_t)val, (uint32_t)(val >> 32)));
        } else {
            const size_t at = ops.size();
            ops.push_back(make_op(kOpBeDef, (uint32_t)g.be_pdag_idx[e] + 1u,
                                  variable_thresholds ? e : (uint32_t)g.be_threshold[e], g.be_event_idx[e] + 1u));
            if (uses[e] > 0) def_sites.push_back({at, e});
            else ops[at].w[0] |= (kNoSlot << 8);
        }
        emit_tallies(e);
        done[e] = 1;
    };
    auto emit_gate = [&](uint32_t v) {
        const uint32_t gi = v - nb;
        const EffectiveInputs e = effective_inputs(g, gi);
        const uint8_t op = g.gate_op[gi];
        const uint32_t k = g.gate_k[gi] & 0xFFu;
        const uint32_t nbits = (op == MCG_ATLEAST) ? counter_bits(e.count) : 0u;
        ops.push_back(make_op(kOpBegin | ((uint32_t)op << 8) | (k << 16) | (nbits << 24)));
        for (uint32_t i = 0; i < e.count; ++i) {
            const uint32_t c = g.inputs[e.begin + i];
            const uint32_t neg = (i >= e.neg_from) ? kNegBit : 0u;
            if (c < nb && kind[c] == BeKind::kConst) {
                const uint64_t val = (g.be_threshold[c] == 0) ? 0ull : ~0ull;
                ops.push_back(make_op(kOpInConst | neg, (uint32_t)val, (uint32_t)(val >> 32)));
            } else if (c < nb && kind[c] == BeKind::kInline) {
                ops.push_back(make_op(kOpInBe | neg, (uint32_t)g.be_pdag_idx[c] + 1u,
                                      variable_thresholds ? c : (uint32_t)g.be_threshold[c], g.be_event_idx[c] + 1u));
                ++out.n_inline_be;
                ++out.n_be_sampled;
            } else {
                use_sites.push_back({ops.size(), c});
                ops.push_back(make_op(kOpInSlot | neg, 0));
            }
        }
        const size_t at = ops.size();
        ops.push_back(make_op(kOpEnd, kNoSlot));
        if (uses[v] > 0) def_sites.push_back({at, v});
        ++out.n_gate_evals;
        emit_tallies(v);
        done[v] = 1;
    };

    struct Frame {
        uint32_t node;
        std::vector<uint32_t> children;
        uint32_t next;
    };
    for (uint32_t root : g.tally_nodes) {
        if (done[root]) continue;
        if (root < nb) {
            emit_be_def(root);
            continue;
        }
        std::vector<Frame> stack;
        auto push = [&](uint32_t v) {
            Frame f{v, {}, 0};
            const EffectiveInputs e = effective_inputs(g, v - nb);
            std::vector<uint32_t> gates, bes;
            for (uint32_t i = 0; i < e.count; ++i) {
                const uint32_t c = g.inputs[e.begin + i];
                if (c >= nb) gates.push_back(c);
                else if (kind[c] == BeKind::kDef) bes.push_back(c);
            }
            std::stable_sort(gates.begin(), gates.end(),
                             [&](uint32_t a, uint32_t b) { return need[a] > need[b]; });
            f.children = gates;
            f.children.insert(f.children.end(), bes.begin(), bes.end());
            stack.push_back(std::move(f));
        };
        push(root);
        while (!stack.empty()) {
            Frame &f = stack.back();
            if (f.next < f.children.size()) {
                const uint32_t c = f.children[f.next++];
                if (done[c]) continue;
                if (c < nb) emit_be_def(c);
                else push(c);
            } else {
                const uint32_t v = f.node;
                stack.pop_back();
                if (!done[v]) emit_gate(v);
            }
        }
    }
    for (uint32_t e = 0; e < nb; ++e)
        if (kind[e] == BeKind::kDef) ++out.n_def_be;
    out.n_be_sampled += out.n_def_be;

    // 5. Live ranges.
    std::vector<int64_t> start(nn, -1), end(nn, -1);
    for (auto &d : def_sites) start[d.second] = (int64_t)d.first;
    for (auto &u : use_sites) end[u.second] = std::max(end[u.second], (int64_t)u.first);
    for (auto &d : def_sites)
        if (end[d.second] < 0) return "internal: defined value without uses";

    // 6. Linear scan over shared-memory slots.
    const uint32_t budget = smem_slot_budget;
    std::vector<uint8_t> in_global(nn, 0);
    std::vector<uint32_t> smem_slot(nn, 0);
    std::vector<uint32_t> active;  // nodes currently holding a shared-memory slot
    std::vector<uint32_t> free_slots;
    for (int32_t s = (int32_t)budget - 1; s >= 0; --s) free_slots.push_back((uint32_t)s);
    uint32_t used_smem = 0;
    for (auto &d : def_sites) {
        const uint32_t v = d.second;
        const int64_t now = start[v];
        for (size_t i = 0; i < active.size();) {
            if (end[active[i]] < now) {
                free_slots.push_back(smem_slot[active[i]]);
                active[i] = active.back();
                active.pop_back();
            } else {
                ++i;
            }
        }
        if (!free_slots.empty()) {
            smem_slot[v] = free_slots.back();
            free_slots.pop_back();
            used_smem = std::max(used_smem, smem_slot[v] + 1);
            active.push_back(v);
            continue;
        }
        if (active.empty()) {  // budget 0
            in_global[v] = 1;
            continue;
        }
        size_t far = 0;
        for (size_t i = 1; i < active.size(); ++i)
            if (end[active[i]] > end[active[far]]) far = i;
        const uint32_t w = active[far];
        if (end[w] > end[v]) {
            in_global[w] = 1;
            smem_slot[v] = smem_slot[w];
            active[far] = v;
        } else {
            in_global[v] = 1;
        }
    }
    out.smem_slots = used_smem;

    // 7. Global slots by linear scan with reuse.
    std::vector<uint32_t> gslot(nn, 0);
    {
        using Item = std::pair<int64_t, uint32_t>;  // (end, slot)
        std::priority_queue<Item, std::vector<Item>, std::greater<Item>> busy;
        std::vector<uint32_t> gfree;
        uint32_t n_g = 0;
        for (auto &d : def_sites) {
            const uint32_t v = d.second;
            if (!in_global[v]) continue;
            while (!busy.empty() && busy.top().first < start[v]) {
                gfree.push_back(busy.top().second);
                busy.pop();
            }
            uint32_t s;
            if (!gfree.empty()) {
                s = gfree.back();
                gfree.pop_back();
            } else {
                s = n_g++;
            }
            gslot[v] = s;
            busy.push({end[v], s});
        }
        out.global_slots = n_g;
        if (n_g >= kSlotGlobal) return "too many global scratch slots";
    }

    // Peak number of simultaneously live values.
    {
        std::vector<std::pair<int64_t, int>> ev;
        for (auto &d : def_sites) {
            ev.push_back({start[d.second], +1});
            ev.push_back({end[d.second] + 1, -1});
        }
        std::sort(ev.begin(), ev.end());
        int cur = 0, best = 0;
        for (auto &x : ev) {
            cur += x.second;
            best = std::max(best, cur);
        }
        out.max_live = (uint32_t)best;
    }

    // 8. Patch slot references.
    auto ref_of = [&](uint32_t v) -> uint32_t {
        return in_global[v] ? (kSlotGlobal | gslot[v]) : smem_slot[v];
    };
    for (auto &d : def_sites) {
        Op &o = ops[d.first];
        const uint32_t code = o.w[0] & kOpMask;
        if (code == kOpEnd) o.w[1] = ref_of(d.second);
        else o.w[0] = (o.w[0] & 0xFFu) | (ref_of(d.second) << 8);
    }
    for (auto &u : use_sites) ops[u.first].w[1] = ref_of(u.second);

    ops.push_back(make_op(kOpHalt));
    ops.push_back(make_op(kOpHalt));  // padding: the interpreter prefetches one op ahead
    return {};
}

}  // namespace mcg
