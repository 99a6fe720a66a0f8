// oracle/bdd_oracle.cc -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// Exact FP64 top-event probability of a flattened PDAG with a reduced
// ordered BDD.  It plays the part of the reference's BDD calculator
// (src/bdd.cc:41-306 builds the ROBDD with ITE/Apply over the PDAG;
// src/probability_analysis.cc:261-285 evaluates P by the Shannon recursion
// P(f) = p(x) P(f|x=1) + (1 - p(x)) P(f|x=0)).  This is an independent,
// simpler implementation: no complement edges, no modules; variables are
// ordered by first appearance in a depth-first walk from the root.
//
// Gate semantics follow the reference's MC kernels (src/mc/kernel/gate.h):
// AND/OR/XOR/NOT/NAND/NOR/NULL over positive then complemented inputs, and
// ATLEAST k-of-n (the true count; the kernels' uint8 count only differs for
// fan-in above 255).
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>

namespace {

struct Node {
    uint32_t var;  // variable level; terminals use UINT32_MAX
    uint32_t lo, hi;
};

struct Key3 {
    uint32_t a, b, c;
    bool operator==(const Key3 &o) const { return a == o.a && b == o.b && c == o.c; }
};
struct Key3Hash {
    size_t operator()(const Key3 &k) const {
        uint64_t h = (uint64_t)k.a * 0x9E3779B97F4A7C15ull;
        h ^= (uint64_t)k.b * 0xC2B2AE3D27D4EB4Full + (h << 6) + (h >> 2);
        h ^= (uint64_t)k.c * 0x165667B19E3779F9ull + (h << 6) + (h >> 2);
        return (size_t)h;
    }
};

class Bdd {
  public:
    explicit Bdd(size_t max_nodes) : max_nodes_(max_nodes) {
        nodes_.push_back({UINT32_MAX, 0, 0});  // 0 = false
        nodes_.push_back({UINT32_MAX, 1, 1});  // 1 = true
    }
    bool overflow() const { return overflow_; }
    size_t size() const { return nodes_.size(); }

    uint32_t var(uint32_t level) { return mk(level, 0, 1); }

    uint32_t ite(uint32_t f, uint32_t g, uint32_t h) {
        if (overflow_) return 0;
        if (f == 1) return g;
        if (f == 0) return h;
        if (g == h) return g;
        if (g == 1 && h == 0) return f;
        const Key3 key{f, g, h};
        auto it = ite_cache_.find(key);
        if (it != ite_cache_.end()) return it->second;
        uint32_t v = nodes_[f].var;
        if (nodes_[g].var < v) v = nodes_[g].var;
        if (nodes_[h].var < v) v = nodes_[h].var;
        uint32_t f1, f0, g1, g0, h1, h0;
        cof(f, v, f1, f0);
        cof(g, v, g1, g0);
        cof(h, v, h1, h0);
        const uint32_t t = ite(f1, g1, h1);
        const uint32_t e = ite(f0, g0, h0);
        const uint32_t r = mk(v, e, t);
        ite_cache_.emplace(key, r);
        return r;
    }
    uint32_t bnot(uint32_t f) { return ite(f, 0, 1); }
    uint32_t band(uint32_t f, uint32_t g) { return ite(f, g, 0); }
    uint32_t bor(uint32_t f, uint32_t g) { return ite(f, 1, g); }
    uint32_t bxor(uint32_t f, uint32_t g) { return ite(f, bnot(g), g); }

    double prob(uint32_t f, const std::vector<double> &p_by_level) {
        std::unordered_map<uint32_t, double> memo;
        return prob_rec(f, p_by_level, memo);
    }

  private:
    void cof(uint32_t f, uint32_t v, uint32_t &f1, uint32_t &f0) const {
        if (nodes_[f].var == v) {
            f1 = nodes_[f].hi;
            f0 = nodes_[f].lo;
        } else {
            f1 = f0 = f;
        }
    }
    uint32_t mk(uint32_t v, uint32_t lo, uint32_t hi) {
        if (lo == hi) return lo;
        const Key3 key{v, lo, hi};
        auto it = unique_.find(key);
        if (it != unique_.end()) return it->second;
        if (nodes_.size() >= max_nodes_) {
            overflow_ = true;
            return 0;
        }
        const uint32_t id = (uint32_t)nodes_.size();
        nodes_.push_back({v, lo, hi});
        unique_.emplace(key, id);
        return id;
    }
    double prob_rec(uint32_t f, const std::vector<double> &p,
                    std::unordered_map<uint32_t, double> &memo) const {
        if (f <= 1) return (double)f;
        auto it = memo.find(f);
        if (it != memo.end()) return it->second;
        const Node &n = nodes_[f];
        const double r = p[n.var] * prob_rec(n.hi, p, memo) + (1.0 - p[n.var]) * prob_rec(n.lo, p, memo);
        memo.emplace(f, r);
        return r;
    }

    size_t max_nodes_;
    bool overflow_ = false;
    std::vector<Node> nodes_;
    std::unordered_map<Key3, uint32_t, Key3Hash> unique_;
    std::unordered_map<Key3, uint32_t, Key3Hash> ite_cache_;
};

enum { AND = 0, OR = 1, ATLEAST = 2, XOR = 3, NOT = 4, NAND = 5, NOR = 6, NUL = 7 };

}  // namespace

extern "C" {

// Exact P(node `root`) for the flattened PDAG (same layout as orc_graph in
// mc_oracle.c).  p_be[e] is the probability of basic event e.  Returns 0 on
// success, -1 for a malformed graph, -2 when the BDD exceeds max_nodes.
// *out_nodes receives the number of BDD nodes built.
int bdd_top_probability(uint32_t n_be, uint32_t n_gates, const uint8_t *gate_op,
                        const uint32_t *gate_k, const uint32_t *gate_in_begin,
                        const uint32_t *gate_in_count, const uint32_t *gate_neg_count,
                        const uint32_t *inputs, const double *p_be, uint32_t root,
                        uint64_t max_nodes, double *out_p, uint64_t *out_nodes) {
    const uint32_t n_nodes = n_be + n_gates;
    if (root >= n_nodes) return -1;
    // Variable order: first appearance of each basic event in an iterative
    // depth-first walk from the root, children in input order.
    std::vector<uint32_t> level(n_be, UINT32_MAX);
    std::vector<uint8_t> seen(n_nodes, 0);
    std::vector<std::pair<uint32_t, uint32_t>> stack;
    uint32_t next_level = 0;
    stack.push_back({root, 0});
    seen[root] = 1;
    while (!stack.empty()) {
        auto &top = stack.back();
        const uint32_t node = top.first;
        if (node < n_be) {
            if (level[node] == UINT32_MAX) level[node] = next_level++;
            stack.pop_back();
            continue;
        }
        const uint32_t gi = node - n_be;
        if (top.second < gate_in_count[gi]) {
            const uint32_t child = inputs[gate_in_begin[gi] + top.second++];
            if (child >= node) return -1;
            if (!seen[child]) {
                seen[child] = 1;
                stack.push_back({child, 0});
            }
        } else {
            stack.pop_back();
        }
    }
    std::vector<double> p_level(next_level, 0.0);
    for (uint32_t e = 0; e < n_be; ++e)
        if (level[e] != UINT32_MAX) p_level[level[e]] = p_be[e];

    Bdd bdd((size_t)max_nodes);
    std::vector<uint32_t> f(n_nodes, 0);
    for (uint32_t e = 0; e < n_be; ++e)
        if (level[e] != UINT32_MAX) f[e] = bdd.var(level[e]);
    for (uint32_t gi = 0; gi < n_gates && gi + n_be <= root; ++gi) {
        const uint32_t node = n_be + gi;
        if (!seen[node]) continue;
        const uint32_t n = gate_in_count[gi];
        const uint32_t off = n - gate_neg_count[gi];
        std::vector<uint32_t> in(n);
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t c = inputs[gate_in_begin[gi] + i];
            in[i] = (i < off) ? f[c] : bdd.bnot(f[c]);
        }
        uint32_t r = 0;
        const uint8_t op = gate_op[gi];
        if (op == ATLEAST) {
            // at_least(i, j): at least j of in[i..n) are true.
            const uint32_t k = gate_k[gi] & 0xFFu;
            std::vector<uint32_t> row(k + 1, 0), next(k + 1, 0);
            // base i = n: true iff j == 0
            for (uint32_t j = 0; j <= k; ++j) row[j] = (j == 0) ? 1u : 0u;
            for (int64_t i = (int64_t)n - 1; i >= 0; --i) {
                next[0] = 1;
                for (uint32_t j = 1; j <= k; ++j) next[j] = bdd.ite(in[(size_t)i], row[j - 1], row[j]);
                row.swap(next);
            }
            r = row[k];
        } else {
            r = (op == AND || op == NAND) ? 1u : 0u;
            for (uint32_t i = 0; i < n; ++i) {
                switch (op) {
                    case OR: case NOR: r = bdd.bor(r, in[i]); break;
                    case AND: case NAND: r = bdd.band(r, in[i]); break;
                    case XOR: r = bdd.bxor(r, in[i]); break;
                    case NOT: case NUL: r = in[i]; break;
                    default: return -1;
                }
            }
            if (op == NAND || op == NOR || op == NOT) r = bdd.bnot(r);
        }
        f[node] = r;
        if (bdd.overflow()) {
            if (out_nodes) *out_nodes = bdd.size();
            return -2;
        }
    }
    *out_p = bdd.prob(f[root], p_level);
    if (out_nodes) *out_nodes = bdd.size();
    return 0;
}

}  // extern "C"
