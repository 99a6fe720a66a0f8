// shared_posterior.cpp -- the cut-set sum of a tree with shared basic events
// and its shared events' conditional probabilities (mcg_shared_posteriors in
// include/mcg_is.h).
//
// For a tree of AND / OR / ATLEAST / pass-through gates (each gate read by one
// gate at most) the cut-set sum S (event: p; AND: product; OR: sum; ATLEAST
// k: k-th elementary symmetric sum) approximates P(top) for rare events.  A
// basic event read by several gates must count once in a product, not once per
// leaf: below the lowest common ancestor (LCA) of its leaves a node's value is
// kept as a polynomial in the indicator z_i of each such "open" event (every
// product reduces z_i^2 to z_i), and at the LCA z_i is replaced by p_i (the
// polynomial is then affine in z_i, so this is its expectation).  S(top) is
// the constant left at the top.  P(z_i = 1 | top) ~ p_i S(top | z_i = 1) / S,
// where S(top | z_i = 1) replaces z_i by 1 at its LCA.  Every connective is
// linear in each input in this ring, and the substitutions at the LCAs above
// are ring homomorphisms, so the change D at the LCA reaches the top as the
// full evaluation of D * adj(LCA): one top-down pass of adjoints (the
// product of the partial derivatives along the path, with the events no
// longer open below evaluated at their p) serves every shared event.
#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>
#include <string>
#include <vector>

#include "error.hpp"
#include "mcg.h"
#include "mcg_is.h"

namespace {

using Mono = std::vector<uint32_t>;  // sorted shared-event ids
using Poly = std::map<Mono, double>;

struct PolyLimit {
    size_t max_terms;
    bool over = false;
};

void add_into(Poly &dst, const Poly &src, double scale = 1.0) {
    for (const auto &t : src) dst[t.first] += scale * t.second;
}

Mono mono_union(const Mono &a, const Mono &b) {
    Mono out;
    out.reserve(a.size() + b.size());
    std::set_union(a.begin(), a.end(), b.begin(), b.end(), std::back_inserter(out));
    return out;
}

Poly mul(const Poly &a, const Poly &b, PolyLimit &lim) {
    Poly out;
    for (const auto &x : a)
        for (const auto &y : b) {
            out[mono_union(x.first, y.first)] += x.second * y.second;
            if (out.size() > lim.max_terms) {
                lim.over = true;
                return out;
            }
        }
    return out;
}

Poly constant(double c) { return Poly{{Mono{}, c}}; }

// z_i := v in every monomial that holds i
Poly substitute(const Poly &f, uint32_t i, double v) {
    Poly out;
    for (const auto &t : f) {
        auto it = std::lower_bound(t.first.begin(), t.first.end(), i);
        if (it != t.first.end() && *it == i) {
            Mono m = t.first;
            m.erase(m.begin() + (it - t.first.begin()));
            out[m] += v * t.second;
        } else {
            out[t.first] += t.second;
        }
    }
    return out;
}

struct Tree {
    const mcg_graph_desc &g;
    uint32_t nb;
    std::vector<uint32_t> parent;                 // per node: reading gate, or kNone
    std::vector<char> shared;                     // per basic event
    std::vector<double> p;                        // per basic event
    std::vector<std::vector<uint32_t>> closes;    // per gate: shared events whose LCA it is
    std::vector<uint32_t> lca;                    // per basic event (shared)
    std::vector<Poly> value;                      // per gate: its polynomial after closing
};

constexpr uint32_t kNone = 0xFFFFFFFFu;
constexpr size_t kAdjointLimitFactor = 16;

// The gate's polynomial from its children's (child(x) gives a child's), before closing.
template <class Child>
Poly combine(const Tree &t, uint32_t gate, Child child, PolyLimit &lim) {
    const mcg_graph_desc &g = t.g;
    const uint32_t j = gate - t.nb;
    const uint32_t op = g.gate_op[j], n = g.gate_in_count[j], k = g.gate_k[j] & 0xFFu;
    const uint32_t *in = g.inputs + g.gate_in_begin[j];
    if (op == MCG_AND) {
        Poly acc = constant(1.0);
        for (uint32_t c = 0; c < n && !lim.over; ++c) acc = mul(acc, child(in[c]), lim);
        return acc;
    }
    if (op == MCG_OR) {
        Poly acc;
        for (uint32_t c = 0; c < n; ++c) add_into(acc, child(in[c]));
        return acc;
    }
    if (op == MCG_ATLEAST) {  // E[r] = e_r of the children so far
        std::vector<Poly> E(k + 1);
        E[0] = constant(1.0);
        for (uint32_t c = 0; c < n && !lim.over; ++c) {
            const Poly v = child(in[c]);
            for (int r = (int)k; r >= 1 && !lim.over; --r) add_into(E[r], mul(E[r - 1], v, lim));
        }
        return k == 0 ? constant(1.0) : E[k];
    }
    return n ? child(in[n - 1]) : Poly{};  // pass-through
}

Poly leaf(const Tree &t, uint32_t x) {
    if (t.shared[x]) return Poly{{Mono{x}, 1.0}};
    return constant(t.p[x]);
}

Poly close_all(const Tree &t, uint32_t gate, Poly f, uint32_t keep = kNone, double keep_value = 0.0) {
    for (uint32_t i : t.closes[gate - t.nb]) f = substitute(f, i, i == keep ? keep_value : t.p[i]);
    return f;
}

double constant_term(const Poly &f) {
    auto it = f.find(Mono{});
    return it == f.end() ? 0.0 : it->second;
}

// z_j := p_j for every event j not in `keep` (sorted).
Poly evaluate_except(const Tree &t, const Poly &f, const std::vector<uint32_t> &keep) {
    Poly out;
    for (const auto &term : f) {
        Mono m;
        double c = term.second;
        for (uint32_t j : term.first) {
            if (std::binary_search(keep.begin(), keep.end(), j)) m.push_back(j);
            else c *= t.p[j];
        }
        out[m] += c;
    }
    return out;
}

// The value with every z_j := p_j.
double evaluate_all(const Tree &t, const Poly &f) {
    double s = 0.0;
    for (const auto &term : f) {
        double c = term.second;
        for (uint32_t j : term.first) c *= t.p[j];
        s += c;
    }
    return s;
}

// d(gate) / d(input q) from the other inputs' values: the product of the
// others (AND), 1 (OR), the (k - 1)-th elementary symmetric sum of the
// others (ATLEAST k), 1 for a pass-through gate's last input and 0 for its
// others.  Every connective is linear in each input (z^2 = z keeps the
// product in the same ring), so a change D of input q changes the gate by
// D times this.
template <class Child>
Poly partial(const Tree &t, uint32_t gate, uint32_t q, Child child, PolyLimit &lim) {
    const mcg_graph_desc &g = t.g;
    const uint32_t j = gate - t.nb;
    const uint32_t op = g.gate_op[j], n = g.gate_in_count[j], k = g.gate_k[j] & 0xFFu;
    const uint32_t *in = g.inputs + g.gate_in_begin[j];
    if (op == MCG_AND) {
        Poly acc = constant(1.0);
        for (uint32_t c = 0; c < n && !lim.over; ++c)
            if (c != q) acc = mul(acc, child(in[c]), lim);
        return acc;
    }
    if (op == MCG_OR) return constant(1.0);
    if (op == MCG_ATLEAST) {
        if (k == 0) return Poly{};
        std::vector<Poly> E(k);  // e_r of the other inputs, r < k
        E[0] = constant(1.0);
        for (uint32_t c = 0; c < n && !lim.over; ++c) {
            if (c == q) continue;
            const Poly v = child(in[c]);
            for (int r = (int)k - 1; r >= 1 && !lim.over; --r) add_into(E[r], mul(E[r - 1], v, lim));
        }
        return E[k - 1];
    }
    return q + 1 == n ? constant(1.0) : Poly{};  // pass-through
}

}  // namespace

extern "C" mcg_status mcg_shared_posteriors(const mcg_graph_desc *graph, uint32_t root, uint64_t max_terms,
                                            double *p_top, double *posterior) {
    mcg::clear_error();
    if (!graph || !p_top || !posterior) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    const mcg_graph_desc &g = *graph;
    const uint32_t nb = g.n_be, nn = g.n_be + g.n_gates;
    if (root >= nn) return mcg::fail(MCG_ERR_INVALID, "root out of range");
    Tree t{g, nb, std::vector<uint32_t>(nn, kNone), std::vector<char>(nb, 0), std::vector<double>(nb, 0.0),
           std::vector<std::vector<uint32_t>>(g.n_gates), std::vector<uint32_t>(nb, kNone),
           std::vector<Poly>(g.n_gates)};
    for (uint32_t i = 0; i < nb; ++i) {
        const uint64_t th = g.be_threshold[i];
        t.p[i] = th >= (1ull << 32) ? 1.0 : (double)th / 4294967296.0;
    }
    // the gates and leaves below the root, each gate read once
    std::vector<std::vector<uint32_t>> leaf_parents(nb);
    std::vector<uint32_t> order;  // gates below the root, children before parents
    if (root >= nb) {
        std::vector<std::pair<uint32_t, uint32_t>> st{{root, 0}};
        while (!st.empty()) {
            auto &top = st.back();
            const uint32_t j = top.first - nb;
            const uint32_t op = g.gate_op[j];
            if (top.second == 0 && (g.gate_neg_count[j] ||
                                    !(op == MCG_AND || op == MCG_OR || op == MCG_ATLEAST || op == MCG_NULL)))
                return mcg::fail(MCG_ERR_INVALID, "AND/OR/ATLEAST/pass-through gates without complemented inputs "
                                                  "only; gate " + std::to_string(j) + " is not one");
            if (op == MCG_ATLEAST && (g.gate_k[j] & 0xFFu) > 64)
                return mcg::fail(MCG_ERR_INVALID, "ATLEAST threshold above 64");
            if (top.second < g.gate_in_count[j]) {
                const uint32_t x = g.inputs[g.gate_in_begin[j] + top.second++];
                if (x >= top.first) return mcg::fail(MCG_ERR_INVALID, "gate input not below the gate");
                if (x < nb) {
                    leaf_parents[x].push_back(top.first);
                } else {
                    if (t.parent[x] != kNone)
                        return mcg::fail(MCG_ERR_INVALID, "gate " + std::to_string(x - nb) +
                                                              " is read by several gates");
                    t.parent[x] = top.first;
                    st.push_back({x, 0});
                }
            } else {
                order.push_back(top.first);
                st.pop_back();
            }
        }
    }
    std::vector<uint32_t> depth(nn, 0);
    for (auto it = order.rbegin(); it != order.rend(); ++it)
        depth[*it] = t.parent[*it] == kNone ? 0 : depth[t.parent[*it]] + 1;
    auto lca2 = [&](uint32_t a, uint32_t b) {
        while (depth[a] > depth[b]) a = t.parent[a];
        while (depth[b] > depth[a]) b = t.parent[b];
        while (a != b) a = t.parent[a], b = t.parent[b];
        return a;
    };
    for (uint32_t i = 0; i < nb; ++i) {
        if (leaf_parents[i].size() < 2) continue;
        t.shared[i] = 1;
        uint32_t l = leaf_parents[i][0];
        for (size_t q = 1; q < leaf_parents[i].size(); ++q) l = lca2(l, leaf_parents[i][q]);
        t.lca[i] = l;
        t.closes[l - nb].push_back(i);
    }
    PolyLimit lim{max_terms ? (size_t)max_terms : (size_t)4096};
    auto child_value = [&](uint32_t x) -> Poly { return x < nb ? leaf(t, x) : t.value[x - nb]; };
    for (uint32_t v : order) {
        t.value[v - nb] = close_all(t, v, combine(t, v, child_value, lim));
        if (lim.over)
            return mcg::fail(MCG_ERR_INVALID, "more than " + std::to_string(lim.max_terms) +
                                                  " terms: too many shared events open below one gate");
    }
    const double S = root < nb ? t.p[root] : constant_term(t.value[root - nb]);
    *p_top = S;
    for (uint32_t i = 0; i < nb; ++i) posterior[i] = -1.0;
    if (!(S > 0.0)) return MCG_OK;
    // The events open at each gate: a leaf below it, their LCA above it.
    std::vector<std::vector<uint32_t>> open(g.n_gates);
    for (uint32_t v : order) {
        const uint32_t j = v - nb;
        std::vector<uint32_t> o;
        for (uint32_t q = 0; q < g.gate_in_count[j]; ++q) {
            const uint32_t x = g.inputs[g.gate_in_begin[j] + q];
            if (x < nb) {
                if (t.shared[x]) o.push_back(x);
            } else {
                o.insert(o.end(), open[x - nb].begin(), open[x - nb].end());
            }
        }
        std::sort(o.begin(), o.end());
        o.erase(std::unique(o.begin(), o.end()), o.end());
        std::vector<uint32_t> closing = t.closes[j];
        std::sort(closing.begin(), closing.end());
        std::set_difference(o.begin(), o.end(), closing.begin(), closing.end(), std::back_inserter(open[j]));
    }
    // Adjoints, top down: a change D of a gate's closed value changes S(top)
    // by the full evaluation of D * adj(gate).  adj(child) = adj(gate) *
    // d(gate)/d(child), with every event not open at the child set to its p
    // (D below that child holds only events open there).  The closings above
    // are ring homomorphisms that leave the factors from higher up unchanged,
    // so they commute with these products.
    std::vector<Poly> adj(g.n_gates);
    if (root >= nb) adj[root - nb] = constant(1.0);
    // The adjoints may hold more terms than the gates' values; they get
    // kAdjointLimitFactor times the limit (a product over it sends every event
    // to the per-path fallback below, which is far slower on such trees).
    const size_t gate_limit = lim.max_terms;
    lim.max_terms = gate_limit > SIZE_MAX / kAdjointLimitFactor ? SIZE_MAX : gate_limit * kAdjointLimitFactor;
    for (auto it = order.rbegin(); it != order.rend() && !lim.over; ++it) {
        const uint32_t u = *it, j = u - nb;
        if (adj[j].empty()) continue;  // the top does not depend on this gate
        for (uint32_t q = 0; q < g.gate_in_count[j] && !lim.over; ++q) {
            const uint32_t c = g.inputs[g.gate_in_begin[j] + q];
            if (c < nb) continue;
            const Poly d = partial(t, u, q, child_value, lim);
            adj[c - nb] = evaluate_except(t, mul(adj[j], d, lim), open[c - nb]);
        }
    }
    for (uint32_t i = 0; i < nb && !lim.over; ++i) {
        if (!t.shared[i]) continue;
        // S(top | z_i = 1) = S + the change of z_i := 1 (instead of p_i) at its LCA, carried up by the adjoint
        const uint32_t v = t.lca[i];
        Poly d = close_all(t, v, combine(t, v, child_value, lim), i, 1.0);
        add_into(d, t.value[v - nb], -1.0);
        const double delta = evaluate_all(t, mul(d, adj[v - nb], lim));
        posterior[i] = std::min(1.0, t.p[i] * (S + delta) / S);
    }
    if (!lim.over) return MCG_OK;
    // The adjoints hold more terms than their limit where the gates' own
    // values did not: S(top | z_i = 1) by re-evaluating the gates above each LCA.
    lim.over = false;
    lim.max_terms = gate_limit;
    for (uint32_t i = 0; i < nb; ++i) {
        if (!t.shared[i]) continue;
        uint32_t v = t.lca[i];
        Poly f = close_all(t, v, combine(t, v, child_value, lim), i, 1.0);
        while (t.parent[v] != kNone && !lim.over) {
            const uint32_t u = t.parent[v], changed = v;
            const Poly fv = f;
            f = close_all(t, u, combine(t, u, [&](uint32_t x) -> Poly {
                return x == changed ? fv : child_value(x);
            }, lim));
            v = u;
        }
        if (lim.over) return mcg::fail(MCG_ERR_INVALID, "term limit exceeded");
        posterior[i] = std::min(1.0, t.p[i] * constant_term(f) / S);
    }
    return MCG_OK;
}
