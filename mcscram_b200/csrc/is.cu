// is.cu -- importance-sampling engine (include/mcg_is.h).
//
// Sampling and gate evaluation are the staged pipeline's kernels, fed with
// the proposal thresholds; a weights kernel queued after each chunk's gate
// phase turns every top-event hit into an FP64 likelihood ratio.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "engine_internal.hpp"
#include "error.hpp"
#include "mcg_is.h"
#include "smem_limit.hpp"

namespace {

#define MCG_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t err_ = (call);                                                              \
        if (err_ != cudaSuccess) {                                                              \
            return mcg::fail(err_ == cudaErrorMemoryAllocation ? MCG_ERR_OOM : MCG_ERR_CUDA,    \
                             std::string(#call) + ": " + cudaGetErrorString(err_));             \
        }                                                                                       \
    } while (0)

constexpr int kWeightThreads = 256;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xFFFFFFFFu, v, o));
    return v;
}

__device__ void atomic_max_double(double *addr, double v) {
    unsigned long long *a = reinterpret_cast<unsigned long long *>(addr);
    unsigned long long old = *a;
    while (__longlong_as_double((long long)old) < v) {
        const unsigned long long prev = atomicCAS(a, old, (unsigned long long)__double_as_longlong(v));
        if (prev == old) break;
        old = prev;
    }
}

// One warp per sample column: lane l owns samples l and l + 32 of the word.
// For samples where the top fires: log w = C + sum_i a_i x_i (FP64).
// sums = {sum w, sum w^2, hits, max log w}.  With ce != nullptr also
// ce[i] += sum over hits of w x_i.  Shared memory: a[n_be] (+ ce[n_be]).
__global__ void __launch_bounds__(kWeightThreads) k_is_weights(const uint64_t *__restrict__ buf, uint64_t W,
                                                               uint32_t n_be, uint32_t root_row,
                                                               const double *__restrict__ a, double C,
                                                               double *__restrict__ sums, double *__restrict__ ce) {
    extern __shared__ double smem_d[];
    double *s_a = smem_d;
    double *s_ce = smem_d + n_be;
    for (uint32_t i = threadIdx.x; i < n_be; i += blockDim.x) {
        s_a[i] = a[i];
        if (ce) s_ce[i] = 0.0;
    }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    double lsum = 0.0, lsum2 = 0.0, lhits = 0.0, lmax = -INFINITY;
    for (uint64_t w = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < W; w += warps) {
        const uint64_t top = buf[(uint64_t)root_row * W + w];
        if (top == 0) continue;  // uniform across the warp
        const bool f0 = (top >> lane) & 1ull, f1 = (top >> (lane + 32)) & 1ull;
        double s0 = 0.0, s1 = 0.0;
        for (uint32_t i = 0; i < n_be; ++i) {
            const uint64_t x = buf[(uint64_t)i * W + w];
            if ((x >> lane) & 1ull) s0 += s_a[i];
            if ((x >> (lane + 32)) & 1ull) s1 += s_a[i];
        }
        const double lw0 = C + s0, lw1 = C + s1;
        const double w0 = f0 ? exp(lw0) : 0.0, w1 = f1 ? exp(lw1) : 0.0;
        lsum += w0 + w1;
        lsum2 += w0 * w0 + w1 * w1;
        lhits += (double)f0 + (double)f1;
        if (f0) lmax = fmax(lmax, lw0);
        if (f1) lmax = fmax(lmax, lw1);
        if (ce) {
            for (uint32_t i = 0; i < n_be; ++i) {
                const uint64_t x = buf[(uint64_t)i * W + w];
                double c = (((x >> lane) & 1ull) ? w0 : 0.0) + (((x >> (lane + 32)) & 1ull) ? w1 : 0.0);
                c = warp_sum(c);
                if (lane == 0 && c != 0.0) atomicAdd(&s_ce[i], c);
            }
        }
    }
    lsum = warp_sum(lsum);
    lsum2 = warp_sum(lsum2);
    lhits = warp_sum(lhits);
    lmax = warp_max(lmax);
    if (lane == 0) {
        if (lsum != 0.0) atomicAdd(&sums[0], lsum);
        if (lsum2 != 0.0) atomicAdd(&sums[1], lsum2);
        if (lhits != 0.0) atomicAdd(&sums[2], lhits);
        if (lmax > -INFINITY) atomic_max_double(&sums[3], lmax);
    }
    if (ce) {
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < n_be; i += blockDim.x)
            if (s_ce[i] != 0.0) atomicAdd(&ce[i], s_ce[i]);
    }
}

// Batched form: many independent trees in one graph, tree k owning basic
// events [be_begin[k], be_begin[k + 1]) and tallied root root_row[k].
// Work items are (tree, strip of 256 words), taken from a queue (a counter
// zeroed before the launch) so that trees of very different size balance.
// One thread per word: the buffer rows are read coalesced, and because
// x_i & top is almost always zero under a proposal, the FP64 log-ratios of
// a sample are only touched where event i fired in a sample where the
// tree's top event fired.
// A pass may draw its words from several proposals (components c = 0 ..
// n_comp - 1, component 0 the main one, c taking a share pi_c of the
// words).  Every sample is then weighted by the balance heuristic of
// multiple importance sampling, whichever component drew it:
//     w = p(x) / sum_c pi_c q_c(x),
//     log w = -logsumexp_c(ln pi_c - log(p / q_c)(x)),
// which is unbiased and keeps w <= p / (pi_c q_c) for every c.
// acc[c][b] (per-thread, local memory) holds log(p / q_c) - C_c of sample
// b, acc[0][b] later its weight.
constexpr int kMaxComponents = 8;

// ---------------------------------------------------------------------------
// Cut-set component: importance sampling of a union of rare events over the
// cut sets of a tree (the "at least one event" mixture of Owen, Maximov &
// Chertkov).  For a tree of AND / OR / ATLEAST / pass-through gates without
// shared nodes, S(node) is the sum over its minimal cut sets of the product
// of their events' probabilities (event: p; AND: product; OR: sum; ATLEAST
// k: k-th elementary symmetric sum of the children's S).  A sample picks a
// cut set C with probability prod_{i in C} p_i / S(top) by descending from
// the top (OR: one child with probability S(child)/S(OR); AND: every child;
// ATLEAST: a k-subset with probability proportional to the product of its
// members' S), forces C's events to fail and draws the other events at their
// nominal probabilities.  Its density is
//     q(x) = p(x) N(x) / S(top),
// N(x) = the number of minimal cut sets contained in x (event: x_i; AND:
// product; OR: sum; ATLEAST: k-th elementary symmetric sum of the children's
// counts), so log(p/q) = log S(top) - log N(x); N(x) >= 1 wherever the top
// event fires, which bounds the weight of this component by S(top) / pi.
//
// Basic events read by several gates (gates still read by one gate each)
// are drawn first, z_i = 1 with a proposal probability r_i, and the tree is
// then one of private events with the shared ones as constants: S_z(node)
// uses z_i for a shared event's leaves (a leaf with z_i = 1 holds the empty
// cut set), and the descent and forcing above run on that conditioned tree
// (no forcing when S_z(top) = 0: z leaves no cut set).  The density is
//     q(x) = r(z) p(x_private) N(x) / S_z(top),
// with N(x) the same count (a shared leaf counts x_i), so
//     log(p/q) = log(p(z) / r(z)) + log S_z(top) - log N(x).
// S_z differs from S_0 (all z_i = 0) only above the shared leaves with
// z_i = 1, so S_z is evaluated by a descent that enters only those gates and
// takes S_0 for every other one.  In the forcing kernel a gate is entered
// when its range of shared-leaf occurrences (the leaves in depth-first
// order) holds one of the sample's z_i = 1 occurrences; in the weights
// kernel when its companion gate fired (an OR over the shared leaves below
// the gate, evaluated with the other gates).
constexpr int kCutStack = 256;     // descent stack of one sample (node ids)
constexpr int kCountDepth = 32;    // frames of the N(x) and S_z evaluations
constexpr int kCutMaxK = 8;        // ATLEAST thresholds the count frames hold
constexpr int kCutMaxN = 32;       // ATLEAST fan-in above shared leaves (suffix sums in registers)
constexpr int kZOcc = 32;          // z_i = 1 occurrences a sample keeps for pruning (more: no pruning)
constexpr uint32_t kNoNode = 0xFFFFFFFFu;

__device__ __forceinline__ uint64_t mix64(uint64_t z) {  // the SplitMix64 finaliser
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Uniform in [0, 1) number `draw` of the stream `base`.
__device__ __forceinline__ double cut_uniform(uint64_t base, uint32_t draw) {
    return (double)(mix64(base + (uint64_t)draw * 0x9E3779B97F4A7C15ull) >> 11) * 0x1.0p-53;
}

struct CutArgs {
    uint64_t *buf;
    uint64_t W, word_begin;
    uint32_t n_inst, n_be;
    const uint32_t *root_row;      // per tree
    const uint4 *gate;             // per gate: op | k << 8, in_begin, in_count, table offset
    const uint32_t *inputs;
    const double *S;               // per node: S_0
    const double *tab;             // OR: cumulative S_0(child) / S_0(OR); ATLEAST: E[j][r] = e_r(S_j..S_n-1)
    const unsigned char *tree_ok;  // per tree: drawn by the component (else its samples stay nominal)
    const unsigned char *shared;   // per basic event: read by several gates
    const uint2 *gate_occ;         // per gate: [lo, hi) of the shared-leaf occurrences below it
    const uint32_t *z_begin;       // per tree: its shared events are z_event[z_begin[k] .. z_begin[k + 1])
    const uint32_t *z_event;
    const uint64_t *z_thr;         // per shared event: z_i = 1 with probability z_thr / 2^32
    const uint32_t *z_index;       // per basic event: its entry in z_event (shared events only)
    const uint32_t *z_occ_begin;   // per shared event: its occurrences z_occ[z_occ_begin[j] .. z_occ_begin[j + 1])
    const uint32_t *z_occ;
    uint64_t seed;
    unsigned int *error;
};

// No memo: every entered gate is evaluated.
struct NoMemo {
    __device__ bool get(uint32_t, double &) { return false; }
    __device__ void put(uint32_t, double) {}
};

// Values of gates already evaluated for one sample: open addressing over
// kMemoSlots node ids with at most kMemoProbes probes, so a full table costs
// a few loads per lookup (a sample that sets many shared events evaluates
// hundreds of gates); values that find no slot are simply not kept.  The
// slots are cleared on first use, so samples that never evaluate a gate pay
// nothing.
constexpr int kMemoBits = 8;
constexpr int kMemoSlots = 1 << kMemoBits;
constexpr int kMemoProbes = 8;
struct GateMemo {
    uint32_t key[kMemoSlots];
    double val[kMemoSlots];
    bool ready = false;
    __device__ void clear() { ready = false; }
    __device__ void prepare() {
        if (ready) return;
#pragma unroll
        for (int i = 0; i < kMemoSlots; ++i) key[i] = kNoNode;
        ready = true;
    }
    __device__ bool get(uint32_t node, double &v) {
        prepare();
        uint32_t h = (node * 2654435761u) >> (32 - kMemoBits);
        for (int i = 0; i < kMemoProbes; ++i, h = (h + 1) & (kMemoSlots - 1)) {
            if (key[h] == node) {
                v = val[h];
                return true;
            }
            if (key[h] == kNoNode) return false;
        }
        return false;
    }
    __device__ void put(uint32_t node, double v) {
        prepare();
        uint32_t h = (node * 2654435761u) >> (32 - kMemoBits);
        for (int i = 0; i < kMemoProbes; ++i, h = (h + 1) & (kMemoSlots - 1)) {
            if (key[h] == kNoNode || key[h] == node) {
                key[h] = node;
                val[h] = v;
                return;
            }
        }
    }
};

// The AND / OR / ATLEAST recursion (product, sum, k-th elementary symmetric
// sum) from gate `root`: a basic event x gives leaf(x), a gate x is entered
// when enter(x) holds and gives other(x) otherwise; memo holds values of
// gates evaluated before (the same recursion gives the same value).  Returns
// -1 when the tree is deeper than the frames hold.  The frame being worked
// on (node, next input, accumulator, gate record) stays in registers; only
// the suspended ancestors and the ATLEAST k-subset sums are in local memory.
template <class Leaf, class Enter, class Other, class Memo = NoMemo>
__device__ double tree_eval(uint32_t root, const uint4 *gate, const uint32_t *inputs, uint32_t n_be, Leaf leaf,
                            Enter enter, Other other, Memo *memo = nullptr) {
    double known;
    if (memo && memo->get(root, known)) return known;
    struct Suspended {
        uint32_t node, j;
        double acc;
    };
    Suspended st[kCountDepth];
    double dp[kCountDepth][kCutMaxK + 1];  // the k-subset sums of an ATLEAST frame at each depth
    int sp = 0;                            // depth of the current frame
    uint32_t node = root, j = 0;
    uint4 g = gate[root - n_be];
    uint32_t op = g.x & 0xFFu, kk = (g.x >> 8) & 0xFFu;
    double acc = op == MCG_AND ? 1.0 : 0.0;
    auto start = [&]() {  // the k-subset sums of a new ATLEAST frame at depth sp
        if (op == MCG_ATLEAST) {
            dp[sp][0] = 1.0;
            for (uint32_t r = 1; r <= kk && r <= (uint32_t)kCutMaxK; ++r) dp[sp][r] = 0.0;
        }
    };
    auto deliver = [&](double v) {
        if (op == MCG_AND) {
            acc *= v;
        } else if (op == MCG_ATLEAST) {
            for (int r = (int)kk; r >= 1; --r) dp[sp][r] += dp[sp][r - 1] * v;
        } else {
            acc += v;
        }
    };
    start();
    for (;;) {
        if (j < g.z) {
            const uint32_t x = inputs[g.y + j++];
            if (x < n_be) {
                deliver(leaf(x));
                continue;
            }
            if (!enter(x)) {
                deliver(other(x));
                continue;
            }
            if (memo && memo->get(x, known)) {
                deliver(known);
                continue;
            }
            if (sp + 1 == kCountDepth) return -1.0;
            st[sp] = Suspended{node, j, acc};
            ++sp;
            node = x;
            j = 0;
            g = gate[x - n_be];
            op = g.x & 0xFFu;
            kk = (g.x >> 8) & 0xFFu;
            acc = op == MCG_AND ? 1.0 : 0.0;
            start();
            continue;
        }
        const double v = op == MCG_ATLEAST ? dp[sp][kk] : acc;
        if (memo) memo->put(node, v);
        if (sp == 0) return v;
        --sp;
        node = st[sp].node;
        j = st[sp].j;
        acc = st[sp].acc;
        g = gate[node - n_be];
        op = g.x & 0xFFu;
        kk = (g.x >> 8) & 0xFFu;
        deliver(v);
    }
}

// One thread per (tree, word, sample): draws the tree's shared events, then
// descends from the tree's top on the conditioned tree and ORs the sample's
// bit into the words of the chosen cut set's private events.
__global__ void __launch_bounds__(256) k_cut_force(CutArgs a) {
    const uint64_t item = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (item >= (uint64_t)a.n_inst * a.W * 64) return;
    const uint32_t b = (uint32_t)(item & 63u);
    const uint64_t wi = item >> 6;
    const uint64_t w = wi % a.W;
    const uint32_t k = (uint32_t)(wi / a.W);
    if (!a.tree_ok[k]) return;  // a tree the component cannot draw: nominal samples
    uint64_t base = mix64(a.seed ^ ((uint64_t)k << 32));
    base = mix64(base ^ (a.word_begin + w));
    base = mix64(base ^ (uint64_t)b);
    uint32_t draw = 0;
    const unsigned long long bit = 1ull << b;
    const uint32_t n_be = a.n_be;
    // z: every shared event of the tree from its own draw of the stream zbase
    const uint32_t z0 = a.z_begin[k], z1 = a.z_begin[k + 1];
    const uint64_t zbase = mix64(base ^ 0x2545F4914F6CDD1Dull);
    auto z_of = [&](uint32_t j) -> bool {  // entry j of z_event
        return (mix64(zbase + (uint64_t)(j - z0 + 1) * 0x9E3779B97F4A7C15ull) >> 32) < a.z_thr[j];
    };
    uint32_t occ[kZOcc];
    int n_occ = 0;
    bool prune = true;
    for (uint32_t j = z0; j < z1; ++j) {
        if (!z_of(j)) continue;
        atomicOr(reinterpret_cast<unsigned long long *>(a.buf + (uint64_t)a.z_event[j] * a.W + w), bit);
        for (uint32_t o = a.z_occ_begin[j]; prune && o < a.z_occ_begin[j + 1]; ++o) {
            if (n_occ == kZOcc) {
                prune = false;
                break;
            }
            const uint32_t v = a.z_occ[o];
            int q = n_occ++;
            while (q > 0 && occ[q - 1] > v) {
                occ[q] = occ[q - 1];
                --q;
            }
            occ[q] = v;
        }
    }
    // a gate whose subtree holds a z_i = 1 leaf (every gate with shared leaves
    // below when the sample has too many to keep)
    auto affected = [&](uint32_t node) -> bool {
        const uint2 r = a.gate_occ[node - n_be];
        if (r.x >= r.y) return false;
        if (!prune) return true;
        for (int q = 0; q < n_occ; ++q)
            if (occ[q] >= r.x) return occ[q] < r.y;
        return false;
    };
    auto leaf = [&](uint32_t x) -> double { return a.shared[x] ? (z_of(a.z_index[x]) ? 1.0 : 0.0) : a.S[x]; };
    auto s0 = [&](uint32_t x) -> double { return a.S[x]; };
    GateMemo memo;
    memo.clear();
    auto sz = [&](uint32_t x) -> double {  // S_z of any node
        if (x < n_be) return leaf(x);
        if (!affected(x)) return a.S[x];
        const double v = tree_eval(x, a.gate, a.inputs, n_be, leaf, affected, s0, &memo);
        if (v < 0.0) atomicOr(a.error, 4u);
        return v;
    };
    uint32_t stack[kCutStack];
    int sp = 0;
    const uint32_t root = a.root_row[k];
    if (!(sz(root) > 0.0)) return;  // z leaves no cut set: nominal private events
    stack[sp++] = root;
    while (sp) {
        const uint32_t node = stack[--sp];
        if (node < n_be) {
            if (!a.shared[node])
                atomicOr(reinterpret_cast<unsigned long long *>(a.buf + (uint64_t)node * a.W + w), bit);
            continue;
        }
        const uint4 g = a.gate[node - n_be];
        const uint32_t op = g.x & 0xFFu, kk = (g.x >> 8) & 0xFFu, n = g.z;
        const uint32_t *in = a.inputs + g.y;
        const double *tab = a.tab + g.w;
        const bool cond = affected(node);
        if (op == MCG_OR) {
            const double u = cut_uniform(base, ++draw);
            uint32_t j = 0;
            if (!cond) {
                while (j + 1 < n && u >= tab[j]) ++j;
            } else {  // shares of S_z: the children's sum, then the first child whose cumulative share passes u
                double cz[kCutMaxN];  // the children's S_z, kept from the sum (wider gates evaluate twice)
                double tot = 0.0;
                for (uint32_t c = 0; c < n; ++c) {
                    const double v = sz(in[c]);
                    if (c < (uint32_t)kCutMaxN) cz[c] = v;
                    tot += v;
                }
                double cum = 0.0;
                for (; j + 1 < n; ++j) {
                    cum += j < (uint32_t)kCutMaxN ? cz[j] : sz(in[j]);
                    if (u * tot < cum) break;
                }
            }
            if (sp == kCutStack) { atomicOr(a.error, 1u); return; }
            stack[sp++] = in[j];
        } else if (op == MCG_ATLEAST) {
            double v[kCutMaxN], E[(kCutMaxN + 1) * (kCutMaxK + 1)];
            const double *Et = tab;
            if (cond) {  // E[j][r] = e_r(S_z of children j .. n - 1)
                if (n > (uint32_t)kCutMaxN) { atomicOr(a.error, 4u); return; }
                for (uint32_t c = 0; c < n; ++c) v[c] = sz(in[c]);
                for (uint32_t r = 0; r <= kk; ++r) E[(uint64_t)n * (kk + 1) + r] = r == 0 ? 1.0 : 0.0;
                for (int c = (int)n - 1; c >= 0; --c)
                    for (uint32_t r = 0; r <= kk; ++r) {
                        double e = E[(uint64_t)(c + 1) * (kk + 1) + r];
                        if (r > 0) e += v[c] * E[(uint64_t)(c + 1) * (kk + 1) + r - 1];
                        E[(uint64_t)c * (kk + 1) + r] = e;
                    }
                Et = E;
            }
            uint32_t r = kk;
            for (uint32_t j = 0; j < n && r > 0; ++j) {
                bool take = n - j == r;
                if (!take) {  // P(take j | r still to take) = S_j E[j+1][r-1] / E[j][r]
                    const double e0 = Et[(uint64_t)j * (kk + 1) + r], e1 = Et[(uint64_t)(j + 1) * (kk + 1) + r - 1];
                    take = cut_uniform(base, ++draw) * e0 < (cond ? v[j] : a.S[in[j]]) * e1;
                }
                if (take) {
                    if (sp == kCutStack) { atomicOr(a.error, 1u); return; }
                    stack[sp++] = in[j];
                    --r;
                }
            }
        } else {  // AND and pass-through gates: every input
            for (uint32_t j = 0; j < n; ++j) {
                if (sp == kCutStack) { atomicOr(a.error, 1u); return; }
                stack[sp++] = in[j];
            }
        }
    }
}

inline uint64_t mix64_host(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// N(x) of sample b of the word whose rows start at col (row stride W), for
// the tree rooted at the fired gate `root`; only fired children are visited.
// Returns -1 when the tree is deeper than the frames hold.
__device__ double cut_count(const uint64_t *col, uint64_t W, uint32_t root, int b, const uint4 *gate,
                            const uint32_t *inputs, uint32_t n_be) {
    auto fired = [&](uint32_t x) -> bool { return (col[(uint64_t)x * W] >> b) & 1ull; };
    return tree_eval(
        root, gate, inputs, n_be, [&](uint32_t x) { return fired(x) ? 1.0 : 0.0; }, fired,
        [&](uint32_t) { return 0.0; });
}

struct IsBatchArgs {
    const uint64_t *buf;
    uint64_t W;
    uint32_t n_inst;
    uint32_t strips;               // ceil(W / (kWeightThreads / split))
    uint32_t split;                // threads per word: 1, 2, 4 or 8
    uint32_t n_comp;               // 1 .. kMaxComponents
    uint32_t n_be;                 // stride of a[] and C[] between components
    const uint32_t *be_begin;      // n_inst + 1
    const uint32_t *root_row;      // n_inst
    const double *a;               // [n_comp][n_be]
    const double *C;               // [n_comp][n_inst]
    double log_pi[kMaxComponents];
    int cut_comp;                  // component drawn by cut sets, or -1: its log(p/q) is
                                   // C + acc (the shared events' log(p(z) / r(z))) + log S_z - log N(x)
    const double *cut_logS;        // per tree: log S_0(top)
    const uint4 *cut_gate;         // per gate (see CutArgs)
    const double *cut_S;           // per node: S_0
    const unsigned char *cut_tree_ok;  // per tree: drawn by the component (else its density there is p)
    const unsigned char *shared;   // per basic event: read by several gates
    const uint32_t *companion;     // per gate: node of the OR over the shared leaves below it, or kNoNode
    const uint32_t *inputs;
    uint32_t n_be_nodes;           // basic events of the joined graph (node ids below are events)
    unsigned int *error;
    double *sums;                  // per tree: sum w, sum w^2, hits, max log w
    double *ce;                    // per event, or null
    unsigned long long *queue;
};

__global__ void __launch_bounds__(kWeightThreads) k_is_weights_batch(IsBatchArgs p) {
    __shared__ unsigned long long s_item;
    double acc[kMaxComponents][64];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t nc = p.n_comp;
    const uint64_t items = (uint64_t)p.n_inst * p.strips;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(p.queue, 1ull);
        __syncthreads();
        const uint64_t item = s_item;
        __syncthreads();
        if (item >= items) break;
        const uint32_t k = (uint32_t)(item / p.strips);
        // p.split threads share a word, thread q taking its samples [q * 64 / split, (q + 1) * 64 / split)
        const uint32_t q = threadIdx.x % p.split, per = 64u / p.split;
        const uint64_t w = (item % p.strips) * (kWeightThreads / p.split) + threadIdx.x / p.split;
        const bool valid = w < p.W;
        const uint64_t mine = per == 64u ? ~0ull : ((1ull << per) - 1ull) << (q * per);
        const uint64_t top = valid ? p.buf[(uint64_t)p.root_row[k] * p.W + w] & mine : 0ull;
        if (!__syncthreads_or(top != 0ull)) continue;
        for (uint64_t m = top; m; m &= m - 1) {
            const int b = __ffsll((long long)m) - 1;
            for (uint32_t c = 0; c < nc; ++c) acc[c][b] = 0.0;
        }
        const uint32_t b0 = p.be_begin[k], b1 = p.be_begin[k + 1];
        const uint64_t *col = p.buf + w;
        uint32_t i = b0;
        for (; i + 4 <= b1; i += 4) {
            uint64_t x[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) x[j] = valid ? col[(uint64_t)(i + j) * p.W] : 0ull;
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                for (uint64_t m = x[j] & top; m; m &= m - 1) {
                    const int b = __ffsll((long long)m) - 1;
                    for (uint32_t c = 0; c < nc; ++c) acc[c][b] += p.a[(uint64_t)c * p.n_be + i + j];
                }
            }
        }
        for (; i < b1; ++i) {
            for (uint64_t m = (valid ? col[(uint64_t)i * p.W] : 0ull) & top; m; m &= m - 1) {
                const int b = __ffsll((long long)m) - 1;
                for (uint32_t c = 0; c < nc; ++c) acc[c][b] += p.a[(uint64_t)c * p.n_be + i];
            }
        }
        double lsum = 0.0, lsum2 = 0.0, lhits = 0.0, lmax = -INFINITY;
        for (uint64_t m = top; m; m &= m - 1) {
            const int b = __ffsll((long long)m) - 1;
            double lw_cut = 0.0;
            if (p.cut_comp >= 0 && !p.cut_tree_ok[k]) {
                lw_cut = p.C[(uint64_t)p.cut_comp * p.n_inst + k] + acc[p.cut_comp][b];  // nominal: 0
            } else if (p.cut_comp >= 0) {
                const uint32_t root = p.root_row[k], nbn = p.n_be_nodes;
                const double n_cut = cut_count(col, p.W, root, b, p.cut_gate, p.inputs, nbn);
                if (!(n_cut >= 1.0)) atomicOr(p.error, 2u);  // too deep, or a failure without a cut set
                double log_sz = p.cut_logS[k];
                auto fired = [&](uint32_t x) -> bool { return (col[(uint64_t)x * p.W] >> b) & 1ull; };
                auto entered = [&](uint32_t x) -> bool {
                    const uint32_t c = p.companion[x - nbn];
                    return c != kNoNode && fired(c);
                };
                if (entered(root)) {  // a shared leaf with z_i = 1 below the top: S_z(top)
                    const double sz = tree_eval(
                        root, p.cut_gate, p.inputs, nbn,
                        [&](uint32_t x) { return p.shared[x] ? (fired(x) ? 1.0 : 0.0) : p.cut_S[x]; }, entered,
                        [&](uint32_t x) { return p.cut_S[x]; });
                    if (!(sz > 0.0)) atomicOr(p.error, 2u);
                    log_sz = log(fmax(sz, 1e-300));
                }
                lw_cut = p.C[(uint64_t)p.cut_comp * p.n_inst + k] + acc[p.cut_comp][b] + log_sz -
                         log(fmax(n_cut, 1.0));
            }
            double lw = p.cut_comp == 0 ? lw_cut : p.C[k] + acc[0][b];
            if (nc > 1) {
                // -logsumexp_c(ln pi_c - log(p/q_c))
                double u[kMaxComponents], hi = -INFINITY;
                for (uint32_t c = 0; c < nc; ++c) {
                    const double lwc = (int)c == p.cut_comp ? lw_cut : p.C[(uint64_t)c * p.n_inst + k] + acc[c][b];
                    u[c] = p.log_pi[c] - lwc;
                    hi = fmax(hi, u[c]);
                }
                double s = 0.0;
                for (uint32_t c = 0; c < nc; ++c) s += exp(u[c] - hi);
                lw = -(hi + log(s));
            }
            const double wv = exp(lw);
            acc[0][b] = wv;
            lsum += wv;
            lsum2 += wv * wv;
            lhits += 1.0;
            lmax = fmax(lmax, lw);
        }
        if (p.ce) {
            for (uint32_t e = b0; e < b1; ++e) {
                uint64_t m = (valid ? col[(uint64_t)e * p.W] : 0ull) & top;
                double c = 0.0;
                for (; m; m &= m - 1) c += acc[0][__ffsll((long long)m) - 1];
                if (__any_sync(0xFFFFFFFFu, c != 0.0)) {
                    c = warp_sum(c);
                    if (lane == 0 && c != 0.0) atomicAdd(&p.ce[e], c);
                }
            }
        }
        lsum = warp_sum(lsum);
        lsum2 = warp_sum(lsum2);
        lhits = warp_sum(lhits);
        lmax = warp_max(lmax);
        if (lane == 0 && lhits != 0.0) {
            double *out = p.sums + 4ull * k;
            atomicAdd(&out[0], lsum);
            atomicAdd(&out[1], lsum2);
            atomicAdd(&out[2], lhits);
            atomic_max_double(&out[3], lmax);
        }
    }
}

// Proposal table and log-ratio terms at the quantised probabilities, for the
// events [b0, b1): beq[i] (the sampler's layout), a[i], and the sum of the
// constant terms over the range.  Returns false with `why` set on a bad q.
bool ratio_terms(const mcg::Graph &g, const uint64_t *q_thr, uint32_t b0, uint32_t b1, uint4 *beq, double *a,
                 double &C, std::string &why) {
    const double two32 = 4294967296.0;
    C = 0.0;
    for (uint32_t i = b0; i < b1; ++i) {
        const uint64_t tp = g.be_threshold[i], tq = q_thr[i];
        const bool fixed = tp == 0 || tp >= (1ull << 32);
        if (fixed ? tq != tp : (tq == 0 || tq >= (1ull << 32))) {
            why = "proposal threshold " + std::to_string(i) +
                  " must lie in [1, 2^32 - 1] (or equal a constant nominal one)";
            return false;
        }
        beq[i] = make_uint4((uint32_t)g.be_pdag_idx[i] + 1u, g.be_event_idx[i] + 1u, (uint32_t)tq, (uint32_t)(tq >> 32));
        a[i] = 0.0;
        if (fixed) continue;
        const double p = (double)tp / two32, q = (double)tq / two32;
        const double l1 = std::log1p(-p) - std::log1p(-q);
        a[i] = std::log(p) - std::log(q) - l1;
        C += l1;
    }
    return true;
}

}  // namespace

struct mcg_is {
    mcg_engine *engine = nullptr;
    uint4 *d_be_q = nullptr;     // proposal thresholds in the sampler's table layout
    double *d_a = nullptr;       // per-event log-ratio increments
    double *d_sums = nullptr;    // 4 doubles
    double *d_ce = nullptr;      // per-event CE numerators
    uint32_t root_row = 0;
    uint32_t weight_smem = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

// Chunk size of the importance-sampling engines when the caller leaves it
// at 0: the staged engine's budget (two chunk buffers of up to 24 GB each),
// but at most 2^17 words per chunk.  A small tree would otherwise take
// 2^20-word chunks of tens of GB that its calls never fill, and these
// engines are created and destroyed as trees converge; large joined graphs
// keep their budget-sized chunks (fewer, fuller launches).
static void default_chunk(const mcg_graph_desc &graph, mcg_run_desc &run) {
    if (run.layered_max_words) return;
    const uint64_t nn = std::max<uint64_t>((uint64_t)graph.n_be + graph.n_gates, 1);
    run.layered_max_words = std::min<uint64_t>(1ull << 17, std::max<uint64_t>(256, (24ull << 30) / (nn * 8)));
}

extern "C" {

mcg_status mcg_is_create(const mcg_graph_desc *graph, const mcg_run_desc *run_in, mcg_is **out) {
    mcg::clear_error();
    if (!graph || !out) return mcg::fail(MCG_ERR_INVALID, "graph and out must not be NULL");
    *out = nullptr;
    if (graph->n_tally != 1) return mcg::fail(MCG_ERR_INVALID, "the tally list must hold exactly the top event");
    mcg_run_desc run{};
    if (run_in) run = *run_in;
    run.mode = MCG_MODE_STAGED;
    default_chunk(*graph, run);
    auto is = std::make_unique<mcg_is>();
    mcg_status st = mcg_create(graph, &run, &is->engine);
    if (st != MCG_OK) return st;
    mcg_engine *e = is->engine;
    const uint32_t nb = e->graph.n_be;
    is->root_row = e->graph.tally_nodes[0];
    is->weight_smem = (uint32_t)(2ull * std::max<uint32_t>(nb, 1) * sizeof(double));
    cudaDeviceProp prop;
    MCG_CUDA(cudaGetDeviceProperties(&prop, e->device));
    if (is->weight_smem > prop.sharedMemPerBlockOptin) {
        mcg_destroy(e);
        return mcg::fail(MCG_ERR_INVALID, "too many basic events for the weights kernel's shared memory");
    }
    st = mcg::set_smem_limit(k_is_weights, is->weight_smem);
    if (st != MCG_OK) {
        mcg_destroy(e);
        return st;
    }
    MCG_CUDA(cudaMalloc((void **)&is->d_be_q, std::max<uint32_t>(nb, 1) * sizeof(uint4)));
    MCG_CUDA(cudaMalloc((void **)&is->d_a, std::max<uint32_t>(nb, 1) * sizeof(double)));
    MCG_CUDA(cudaMalloc((void **)&is->d_ce, std::max<uint32_t>(nb, 1) * sizeof(double)));
    MCG_CUDA(cudaMalloc((void **)&is->d_sums, 4 * sizeof(double)));
    MCG_CUDA(cudaEventCreate(&is->ev0));
    MCG_CUDA(cudaEventCreate(&is->ev1));
    *out = is.release();
    return MCG_OK;
}

mcg_status mcg_is_destroy(mcg_is *is) {
    mcg::clear_error();
    if (!is) return MCG_OK;
    if (is->engine) {
        cudaSetDevice(is->engine->device);
        cudaStreamSynchronize(is->engine->stream);
    }
    cudaFree(is->d_be_q);
    cudaFree(is->d_a);
    cudaFree(is->d_ce);
    cudaFree(is->d_sums);
    if (is->ev0) cudaEventDestroy(is->ev0);
    if (is->ev1) cudaEventDestroy(is->ev1);
    if (is->engine) mcg_destroy(is->engine);
    delete is;
    return MCG_OK;
}

mcg_status mcg_is_run(mcg_is *is, const uint64_t *q_thr, uint32_t iteration, uint64_t word_begin, uint64_t word_count,
                      mcg_is_result *result, double *ce_num) {
    mcg::clear_error();
    if (!is || !q_thr || !result) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    mcg_engine *e = is->engine;
    const mcg::Graph &g = e->graph;
    const uint32_t nb = g.n_be;
    if (word_begin + word_count > (1ull << 32)) return mcg::fail(MCG_ERR_INVALID, "word range exceeds the counter");
    // Log-ratio terms at the quantised probabilities.
    std::vector<double> a(nb, 0.0);
    double C = 0.0;
    std::vector<uint4> beq(nb);
    std::string why;
    if (!ratio_terms(g, q_thr, 0, nb, beq.data(), a.data(), C, why)) return mcg::fail(MCG_ERR_INVALID, why);
    MCG_CUDA(cudaSetDevice(e->device));
    MCG_CUDA(cudaMemcpyAsync(is->d_be_q, beq.data(), nb * sizeof(uint4), cudaMemcpyHostToDevice, e->stream));
    MCG_CUDA(cudaMemcpyAsync(is->d_a, a.data(), nb * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    const double init[4] = {0.0, 0.0, 0.0, -std::numeric_limits<double>::infinity()};
    MCG_CUDA(cudaMemcpyAsync(is->d_sums, init, sizeof(init), cudaMemcpyHostToDevice, e->stream));
    MCG_CUDA(cudaMemsetAsync(is->d_ce, 0, std::max<uint32_t>(nb, 1) * sizeof(double), e->stream));
    const bool want_ce = ce_num != nullptr;
    e->d_be_sample = is->d_be_q;
    e->table_iteration = 0xFFFFFFFFu;  // the sampler table follows the proposal
    const uint32_t root_row = is->root_row;
    const uint32_t smem = want_ce ? is->weight_smem : is->weight_smem / 2;
    double *d_a = is->d_a, *d_sums = is->d_sums, *d_ce = want_ce ? is->d_ce : nullptr;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
    e->chunk_hook = [=](cudaStream_t s, const uint64_t *buf, uint64_t W) -> mcg_status {
        const uint64_t warps = (W + 0) / 1;
        const uint32_t blocks = (uint32_t)std::min<uint64_t>((warps + 7) / 8, (uint64_t)sms * 8);
        k_is_weights<<<std::max<uint32_t>(blocks, 1), kWeightThreads, smem, s>>>(buf, W, nb, root_row, d_a, C,
                                                                                 d_sums, d_ce);
        const cudaError_t err = cudaGetLastError();
        if (err != cudaSuccess) return mcg::fail(MCG_ERR_CUDA, std::string("k_is_weights: ") + cudaGetErrorString(err));
        return MCG_OK;
    };
    MCG_CUDA(cudaEventRecord(is->ev0, e->stream));
    mcg_status st = mcg::internal::run_staged(e, iteration, 1, word_begin, word_count);
    e->chunk_hook = nullptr;
    e->d_be_sample = nullptr;
    e->table_iteration = 0xFFFFFFFFu;
    if (st != MCG_OK) return st;
    MCG_CUDA(cudaEventRecord(is->ev1, e->stream));
    double sums[4];
    MCG_CUDA(cudaMemcpyAsync(sums, is->d_sums, sizeof(sums), cudaMemcpyDeviceToHost, e->stream));
    if (want_ce) MCG_CUDA(cudaMemcpyAsync(ce_num, is->d_ce, nb * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    MCG_CUDA(cudaStreamSynchronize(e->stream));
    float ms = 0;
    MCG_CUDA(cudaEventElapsedTime(&ms, is->ev0, is->ev1));
    std::memset(result, 0, sizeof(*result));
    const double n = (double)word_count * 64.0;
    result->samples = word_count * 64;
    result->hits = (uint64_t)sums[2];
    result->sum_w = sums[0];
    result->sum_w2 = sums[1];
    result->estimate = sums[0] / n;
    const double var = std::max(0.0, sums[1] / n - result->estimate * result->estimate);
    result->std_err = n > 1 ? std::sqrt(var / (n - 1.0)) : 0.0;
    result->rel_err = result->estimate > 0 ? result->std_err / result->estimate : INFINITY;
    result->ess = sums[1] > 0 ? sums[0] * sums[0] / sums[1] : 0.0;
    result->max_log_w = sums[3];
    result->kernel_ms = ms;
    return MCG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Batched importance sampling over many trees joined into one graph.

struct mcg_is_batch {
    mcg_engine *engine = nullptr;
    uint32_t n_inst = 0;
    uint32_t n_comp_cap = 0;             // components the device arrays hold
    std::vector<uint32_t> be_begin;
    uint4 *d_be_q = nullptr;             // [n_comp][n_be] sampler tables
    double *d_a = nullptr;               // [n_comp][n_be]
    double *d_C = nullptr;               // [n_comp][n_inst]
    double *d_sums = nullptr;
    double *d_ce = nullptr;
    uint32_t *d_be_begin = nullptr;
    uint32_t *d_root = nullptr;
    unsigned long long *d_queue = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<uint4> beq;
    std::vector<double> a, C, init;
    // cut-set component (built on first use)
    bool cut_ready = false;
    uint4 *d_cut_gate = nullptr;
    double *d_cut_S = nullptr, *d_cut_tab = nullptr, *d_cut_logS = nullptr;
    unsigned int *d_cut_error = nullptr;
    // shared basic events of the cut-set component: companion gates appended
    // to the graph at creation (the caller's gates are the first n_gates_in)
    uint32_t n_gates_in = 0;
    bool companions = false;
    std::vector<uint32_t> companion;     // per gate of the caller: its companion node, or kNoNode
    std::vector<unsigned char> shared;   // per basic event
    std::vector<unsigned char> tree_gates_ok;  // per tree: gates the component takes (companions built for it)
    std::vector<unsigned char> tree_ok;  // per tree: the cut-set component draws it (else its samples stay nominal)
    unsigned char *d_tree_ok = nullptr;
    std::vector<uint32_t> z_event;       // shared events, tree by tree
    std::vector<uint64_t> z_thr, cut_q;  // per run: their proposal thresholds; the component's table
    unsigned char *d_shared = nullptr;
    uint2 *d_gate_occ = nullptr;
    uint32_t *d_companion = nullptr, *d_z_begin = nullptr, *d_z_event = nullptr, *d_z_index = nullptr;
    uint32_t *d_z_occ_begin = nullptr, *d_z_occ = nullptr;
    uint64_t *d_z_thr = nullptr;
};

namespace {

// Frees everything; keeps the error message a failed create has just set.
void release_batch(mcg_is_batch *b) {
    const std::string keep = mcg::last_error();
    if (b->engine) {
        cudaSetDevice(b->engine->device);
        cudaStreamSynchronize(b->engine->stream);
    }
    cudaFree(b->d_be_q);
    cudaFree(b->d_a);
    cudaFree(b->d_C);
    cudaFree(b->d_sums);
    cudaFree(b->d_ce);
    cudaFree(b->d_be_begin);
    cudaFree(b->d_root);
    cudaFree(b->d_queue);
    cudaFree(b->d_cut_gate);
    cudaFree(b->d_cut_S);
    cudaFree(b->d_cut_tab);
    cudaFree(b->d_cut_logS);
    cudaFree(b->d_cut_error);
    for (void *q : {(void *)b->d_tree_ok, (void *)b->d_shared, (void *)b->d_gate_occ, (void *)b->d_companion, (void *)b->d_z_begin,
                    (void *)b->d_z_event, (void *)b->d_z_index, (void *)b->d_z_occ_begin, (void *)b->d_z_occ,
                    (void *)b->d_z_thr})
        cudaFree(q);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->engine) mcg_destroy(b->engine);
    mcg::last_error() = keep;
}

// Every gate must read nodes of one tree only, and root k must belong to
// tree k: the owner of each node is propagated from the event ranges.
std::string check_partition(const mcg::Graph &g, const std::vector<uint32_t> &be_begin) {
    const uint32_t n_inst = (uint32_t)be_begin.size() - 1;
    constexpr uint32_t kNone = 0xFFFFFFFFu;
    std::vector<uint32_t> owner(g.n_nodes(), kNone);
    for (uint32_t k = 0; k < n_inst; ++k)
        for (uint32_t i = be_begin[k]; i < be_begin[k + 1]; ++i) owner[i] = k;
    for (uint32_t j = 0; j < g.n_gates; ++j) {
        uint32_t o = kNone;
        for (uint32_t s = 0; s < g.gate_in_count[j]; ++s) {
            const uint32_t x = owner[g.inputs[g.gate_in_begin[j] + s]];
            if (x == kNone) continue;
            if (o != kNone && x != o) return "gate " + std::to_string(j) + " reads nodes of two trees";
            o = x;
        }
        owner[g.n_be + j] = o;
    }
    for (uint32_t k = 0; k < n_inst; ++k) {
        const uint32_t r = g.tally_nodes[k];
        if (owner[r] != k && !(owner[r] == kNone && be_begin[k] == be_begin[k + 1]))
            return "tallied node " + std::to_string(k) + " is not a node of tree " + std::to_string(k);
    }
    return std::string();
}

// Trees the cut-set component can draw: every gate AND / OR / ATLEAST /
// pass-through without complemented inputs and read by one gate at most
// (tree_ok[t]).  For those of them with basic events read by several gates,
// companion gates: for every gate with a shared event's leaf below it, an OR
// over those leaves and over its child gates' companions, appended after the
// caller's gates (the tallies stay the trees' tops).  The weights kernel
// reads a companion's word to see which gates a sample's z_i = 1 leaves
// reach.  Returns whether any companion was added.
struct Augmented {
    std::vector<uint8_t> op;
    std::vector<uint32_t> k, begin, count, neg, inputs;
    std::vector<int32_t> pdag;
    std::vector<uint32_t> companion;  // per caller's gate
    std::vector<unsigned char> tree_ok;
    mcg_graph_desc desc{};
};

bool add_companions(const mcg_graph_desc &d, uint32_t n_inst, const uint32_t *be_begin, Augmented &a) {
    const uint64_t nb = d.n_be, ng = d.n_gates, nn = nb + ng;
    std::vector<uint32_t> fanout(nn, 0), owner(nn, kNoNode);
    for (uint64_t i = 0; i < d.n_inputs; ++i)
        if (d.inputs[i] < nn) ++fanout[d.inputs[i]];
    for (uint32_t t = 0; t < n_inst; ++t)
        for (uint32_t i = be_begin[t]; i < be_begin[t + 1]; ++i) owner[i] = t;
    a.tree_ok.assign(n_inst, 1);
    for (uint64_t j = 0; j < ng; ++j) {
        uint32_t o = kNoNode;
        const bool in_range = (uint64_t)d.gate_in_begin[j] + d.gate_in_count[j] <= d.n_inputs;
        for (uint32_t c = 0; in_range && c < d.gate_in_count[j]; ++c) {
            const uint32_t x = d.inputs[d.gate_in_begin[j] + c];
            if (x < nn && owner[x] != kNoNode) o = owner[x];
        }
        owner[nb + j] = o;
        const uint8_t op = d.gate_op[j];
        if (o != kNoNode && (!in_range || fanout[nb + j] > 1 || d.gate_neg_count[j] ||
                             !(op == MCG_AND || op == MCG_OR || op == MCG_ATLEAST || op == MCG_NULL)))
            a.tree_ok[o] = 0;
    }
    bool any_shared = false;
    for (uint64_t i = 0; i < nb; ++i) any_shared |= fanout[i] > 1 && owner[i] != kNoNode && a.tree_ok[owner[i]];
    a.companion.assign(ng, kNoNode);
    if (!any_shared) return false;
    a.op.assign(d.gate_op, d.gate_op + ng);
    a.k.assign(d.gate_k, d.gate_k + ng);
    a.begin.assign(d.gate_in_begin, d.gate_in_begin + ng);
    a.count.assign(d.gate_in_count, d.gate_in_count + ng);
    a.neg.assign(d.gate_neg_count, d.gate_neg_count + ng);
    a.inputs.assign(d.inputs, d.inputs + d.n_inputs);
    if (d.gate_pdag_idx) a.pdag.assign(d.gate_pdag_idx, d.gate_pdag_idx + ng);
    for (uint64_t j = 0; j < ng; ++j) {
        if (owner[nb + j] == kNoNode || !a.tree_ok[owner[nb + j]]) continue;
        std::vector<uint32_t> in;
        for (uint32_t c = 0; c < d.gate_in_count[j]; ++c) {
            const uint32_t x = d.inputs[d.gate_in_begin[j] + c];
            if (x < nb ? fanout[x] > 1 : (x - nb < j && a.companion[x - nb] != kNoNode))
                in.push_back(x < nb ? x : a.companion[x - nb]);
        }
        if (in.empty()) continue;
        a.companion[j] = (uint32_t)(nb + a.op.size());
        a.op.push_back(MCG_OR);
        a.k.push_back(0);
        a.begin.push_back((uint32_t)a.inputs.size());
        a.count.push_back((uint32_t)in.size());
        a.neg.push_back(0);
        if (d.gate_pdag_idx) a.pdag.push_back(-1);
        a.inputs.insert(a.inputs.end(), in.begin(), in.end());
    }
    a.desc = d;
    a.desc.n_gates = (uint32_t)a.op.size();
    a.desc.gate_op = a.op.data();
    a.desc.gate_k = a.k.data();
    a.desc.gate_in_begin = a.begin.data();
    a.desc.gate_in_count = a.count.data();
    a.desc.gate_neg_count = a.neg.data();
    a.desc.inputs = a.inputs.data();
    a.desc.n_inputs = a.inputs.size();
    a.desc.gate_pdag_idx = d.gate_pdag_idx ? a.pdag.data() : nullptr;
    return true;
}

}  // namespace

extern "C" {

mcg_status mcg_is_batch_create(const mcg_graph_desc *graph, uint32_t n_inst, const uint32_t *be_begin,
                               const mcg_run_desc *run_in, mcg_is_batch **out) {
    mcg::clear_error();
    if (!graph || !be_begin || !out) return mcg::fail(MCG_ERR_INVALID, "graph, be_begin and out must not be NULL");
    *out = nullptr;
    if (n_inst == 0) return mcg::fail(MCG_ERR_INVALID, "no trees");
    if (graph->n_tally != n_inst) return mcg::fail(MCG_ERR_INVALID, "the tally list must hold one top event per tree");
    if (be_begin[0] != 0 || be_begin[n_inst] != graph->n_be)
        return mcg::fail(MCG_ERR_INVALID, "be_begin must start at 0 and end at n_be");
    for (uint32_t k = 0; k < n_inst; ++k)
        if (be_begin[k + 1] < be_begin[k]) return mcg::fail(MCG_ERR_INVALID, "be_begin must not decrease");
    mcg_run_desc run{};
    if (run_in) run = *run_in;
    run.mode = MCG_MODE_STAGED;
    default_chunk(*graph, run);
    auto b = std::unique_ptr<mcg_is_batch, void (*)(mcg_is_batch *)>(new mcg_is_batch, [](mcg_is_batch *x) {
        release_batch(x);
        delete x;
    });
    b->n_inst = n_inst;
    b->be_begin.assign(be_begin, be_begin + n_inst + 1);
    b->n_gates_in = graph->n_gates;
    Augmented aug;
    b->companions = add_companions(*graph, n_inst, be_begin, aug);
    b->companion = aug.companion;
    b->tree_gates_ok = aug.tree_ok;
    mcg_status st = mcg_create(b->companions ? &aug.desc : graph, &run, &b->engine);
    if (st != MCG_OK) return st;
    const mcg::Graph &g = b->engine->graph;
    const std::string bad = check_partition(g, b->be_begin);
    if (!bad.empty()) return mcg::fail(MCG_ERR_INVALID, bad);
    const uint32_t nb = std::max<uint32_t>(g.n_be, 1);
    MCG_CUDA(cudaSetDevice(b->engine->device));
    MCG_CUDA(cudaMalloc((void **)&b->d_ce, nb * sizeof(double)));
    MCG_CUDA(cudaMalloc((void **)&b->d_sums, 4ull * n_inst * sizeof(double)));
    MCG_CUDA(cudaMalloc((void **)&b->d_be_begin, (n_inst + 1ull) * sizeof(uint32_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_root, n_inst * sizeof(uint32_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_queue, sizeof(unsigned long long)));
    MCG_CUDA(cudaMemcpy(b->d_be_begin, be_begin, (n_inst + 1ull) * sizeof(uint32_t), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemcpy(b->d_root, g.tally_nodes.data(), n_inst * sizeof(uint32_t), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaEventCreate(&b->ev0));
    MCG_CUDA(cudaEventCreate(&b->ev1));
    b->init.resize(4ull * n_inst);
    for (uint32_t k = 0; k < n_inst; ++k) {
        b->init[4ull * k] = b->init[4ull * k + 1] = b->init[4ull * k + 2] = 0.0;
        b->init[4ull * k + 3] = -std::numeric_limits<double>::infinity();
    }
    *out = b.release();
    return MCG_OK;
}

mcg_status mcg_is_batch_destroy(mcg_is_batch *b) {
    mcg::clear_error();
    if (!b) return MCG_OK;
    release_batch(b);
    delete b;
    return MCG_OK;
}

}  // extern "C"

namespace {

// Tables of the cut-set component (see k_cut_force): every gate AND, OR,
// ATLEAST (k <= 8) or pass-through without complemented inputs and read by
// one gate at most; basic events read by several gates are the shared
// events z of their tree (the graph then carries companion gates); S(top) > 0
// for every tree.
mcg_status build_cut_tables(mcg_is_batch *b) {
    const mcg::Graph &g = b->engine->graph;
    const uint32_t nb = g.n_be, ng_all = g.n_gates, ng = b->n_gates_in, nn = g.n_nodes();
    std::vector<uint32_t> fanout(nn, 0), owner(nn, kNoNode);
    for (uint32_t j = 0; j < ng; ++j)
        for (uint32_t c = 0; c < g.gate_in_count[j]; ++c) ++fanout[g.inputs[g.gate_in_begin[j] + c]];
    for (uint32_t t = 0; t < b->n_inst; ++t)
        for (uint32_t i = b->be_begin[t]; i < b->be_begin[t + 1]; ++i) owner[i] = t;
    for (uint32_t j = 0; j < ng; ++j)
        for (uint32_t c = 0; c < g.gate_in_count[j]; ++c) {
            const uint32_t o = owner[g.inputs[g.gate_in_begin[j] + c]];
            if (o != kNoNode) owner[nb + j] = o;
        }
    // Trees the component cannot draw keep nominal samples in its words (their
    // density there is p); it fails only when it can draw none of them.
    std::vector<unsigned char> &ok = b->tree_ok;
    ok.assign(b->n_inst, 1);
    std::string why;
    auto reject = [&](uint32_t node, const std::string &msg) {
        const uint32_t t = owner[node];
        if (t == kNoNode || !ok[t]) return;
        ok[t] = 0;
        if (why.empty()) why = msg;
    };
    // a shared basic event needs its tree's companion gates (built when every gate of the tree qualified)
    for (uint32_t i = 0; i < nb + ng; ++i)
        if (fanout[i] > 1 && owner[i] != kNoNode &&
            (i >= nb || !b->companions || owner[i] >= b->tree_gates_ok.size() || !b->tree_gates_ok[owner[i]]))
            reject(i, "cut-set sampling needs trees: node " + std::to_string(i) + " is read by several gates");
    b->shared.assign(nb, 0);
    for (uint32_t i = 0; i < nb; ++i) b->shared[i] = fanout[i] > 1 && owner[i] != kNoNode && ok[owner[i]];
    // S_0 (shared events at 0) for the tables; S with every event at p for the check
    std::vector<double> S(nn, 0.0), Sp(nn, 0.0), tab;
    std::vector<uint4> gate(std::max<uint32_t>(ng_all, 1), make_uint4(0, 0, 0, 0));
    for (uint32_t i = 0; i < nb; ++i) {
        const uint64_t t = g.be_threshold[i];
        Sp[i] = t >= (1ull << 32) ? 1.0 : (double)t / 4294967296.0;
        S[i] = b->shared[i] ? 0.0 : Sp[i];
    }
    auto elementary = [](const std::vector<double> &v, uint32_t k, std::vector<double> &E) {
        const uint32_t n = (uint32_t)v.size();  // E[j][r] = e_r(v_j, ..., v_{n-1}), j = n .. 0
        E.assign((size_t)(n + 1) * (k + 1), 0.0);
        E[(size_t)n * (k + 1)] = 1.0;
        for (int c = (int)n - 1; c >= 0; --c)
            for (uint32_t r = 0; r <= k; ++r) {
                double e = E[(size_t)(c + 1) * (k + 1) + r];
                if (r > 0) e += v[c] * E[(size_t)(c + 1) * (k + 1) + r - 1];
                E[(size_t)c * (k + 1) + r] = e;
            }
    };
    std::vector<double> vals, valp, E, Ep;
    for (uint32_t j = 0; j < ng; ++j) {
        const uint32_t op = g.gate_op[j], n = g.gate_in_count[j], k = g.gate_k[j] & 0xFFu;
        const uint32_t *in = g.inputs.data() + g.gate_in_begin[j];
        if (g.gate_neg_count[j] || !(op == MCG_AND || op == MCG_OR || op == MCG_ATLEAST || op == MCG_NULL))
            reject(nb + j, "cut-set sampling needs AND/OR/ATLEAST gates without complemented inputs; gate " +
                               std::to_string(j) + " is not one");
        if (op == MCG_ATLEAST && k > (uint32_t)kCutMaxK) reject(nb + j, "cut-set sampling: ATLEAST threshold above 8");
        if (owner[nb + j] == kNoNode || !ok[owner[nb + j]]) continue;  // its tree keeps nominal samples
        gate[j] = make_uint4(op | (k << 8), g.gate_in_begin[j], n, (uint32_t)tab.size());
        vals.assign(n, 0.0);
        valp.assign(n, 0.0);
        for (uint32_t c = 0; c < n; ++c) vals[c] = S[in[c]], valp[c] = Sp[in[c]];
        double v = 0.0, vp = 0.0;
        if (op == MCG_AND) {
            v = vp = 1.0;
            for (uint32_t c = 0; c < n; ++c) v *= vals[c], vp *= valp[c];
        } else if (op == MCG_OR) {
            for (uint32_t c = 0; c < n; ++c) v += vals[c], vp += valp[c];
            double cum = 0.0;
            for (uint32_t c = 0; c < n; ++c) {
                cum += vals[c];
                tab.push_back(v > 0 ? cum / v : 1.0);
            }
        } else if (op == MCG_ATLEAST) {
            elementary(vals, k, E);
            elementary(valp, k, Ep);
            v = E[k];
            vp = Ep[k];
            tab.insert(tab.end(), E.begin(), E.end());
        } else {  // pass-through
            v = n ? vals[n - 1] : 0.0;
            vp = n ? valp[n - 1] : 0.0;
        }
        S[nb + j] = v;
        Sp[nb + j] = vp;
    }
    for (uint32_t j = ng; j < ng_all; ++j)  // companions: never entered by the descent or the evaluations
        gate[j] = make_uint4(MCG_OR, g.gate_in_begin[j], g.gate_in_count[j], 0);
    std::vector<double> logS(b->n_inst, 0.0);
    for (uint32_t t = 0; t < b->n_inst; ++t) {
        if (!ok[t]) continue;
        const double st = Sp[g.tally_nodes[t]];
        if (!(st > 0.0) || !std::isfinite(st)) {
            ok[t] = 0;
            if (why.empty()) why = "cut-set sampling: tree " + std::to_string(t) + " has no cut set";
            continue;
        }
        logS[t] = std::log(S[g.tally_nodes[t]]);  // -inf when every cut set holds a shared event
    }
    // shared-leaf occurrences in depth-first order from every top: each gate's
    // subtree holds the range [lo, hi) of them
    std::vector<uint2> occ_range(std::max<uint32_t>(ng_all, 1), make_uint2(0, 0));
    std::vector<std::vector<uint32_t>> occ_of(nb);
    uint32_t pos = 0;
    for (uint32_t t = 0; t < b->n_inst; ++t) {
        const uint32_t root = g.tally_nodes[t];
        if (root < nb || !ok[t]) continue;
        std::vector<std::pair<uint32_t, uint32_t>> st{{root, 0}};
        occ_range[root - nb].x = pos;
        while (!st.empty()) {
            auto &top = st.back();
            const uint32_t j = top.first - nb;
            if (top.second < g.gate_in_count[j]) {
                const uint32_t x = g.inputs[g.gate_in_begin[j] + top.second++];
                if (x < nb) {
                    if (b->shared[x]) occ_of[x].push_back(pos++);
                } else {
                    occ_range[x - nb].x = pos;
                    st.push_back({x, 0});
                }
            } else {
                occ_range[j].y = pos;
                const uint32_t op = g.gate_op[j];
                if (op == MCG_ATLEAST && occ_range[j].y > occ_range[j].x && g.gate_in_count[j] > (uint32_t)kCutMaxN) {
                    ok[t] = 0;
                    if (why.empty())
                        why = "cut-set sampling: ATLEAST gate " + std::to_string(j) +
                              " above shared events has more than 32 inputs";
                }
                st.pop_back();
            }
        }
    }
    bool any = false;
    for (uint32_t t = 0; t < b->n_inst; ++t) any |= ok[t] != 0;
    if (!any) return mcg::fail(MCG_ERR_INVALID, why.empty() ? std::string("cut-set sampling: no tree qualifies") : why);
    std::vector<uint32_t> z_begin(b->n_inst + 1, 0), z_index(nb, 0), z_occ_begin{0}, z_occ;
    b->z_event.clear();
    for (uint32_t t = 0; t < b->n_inst; ++t) {
        z_begin[t] = (uint32_t)b->z_event.size();
        for (uint32_t i = b->be_begin[t]; i < b->be_begin[t + 1]; ++i) {
            if (!b->shared[i] || !ok[t]) continue;
            z_index[i] = (uint32_t)b->z_event.size();
            b->z_event.push_back(i);
            z_occ.insert(z_occ.end(), occ_of[i].begin(), occ_of[i].end());
            z_occ_begin.push_back((uint32_t)z_occ.size());
        }
    }
    z_begin[b->n_inst] = (uint32_t)b->z_event.size();
    std::vector<uint32_t> comp(std::max<uint32_t>(ng, 1), kNoNode);
    if (b->companions) std::copy(b->companion.begin(), b->companion.end(), comp.begin());
    if (tab.empty()) tab.push_back(0.0);
    const uint64_t nz = std::max<uint64_t>(b->z_event.size(), 1);
    if (z_occ.empty()) z_occ.push_back(0);
    MCG_CUDA(cudaMalloc((void **)&b->d_cut_gate, gate.size() * sizeof(uint4)));
    MCG_CUDA(cudaMalloc((void **)&b->d_cut_S, nn * sizeof(double)));
    MCG_CUDA(cudaMalloc((void **)&b->d_cut_tab, tab.size() * sizeof(double)));
    MCG_CUDA(cudaMalloc((void **)&b->d_cut_logS, b->n_inst * sizeof(double)));
    MCG_CUDA(cudaMalloc((void **)&b->d_cut_error, sizeof(unsigned int)));
    MCG_CUDA(cudaMalloc((void **)&b->d_shared, std::max<uint32_t>(nb, 1)));
    MCG_CUDA(cudaMalloc((void **)&b->d_tree_ok, b->n_inst));
    MCG_CUDA(cudaMemcpy(b->d_tree_ok, ok.data(), b->n_inst, cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMalloc((void **)&b->d_gate_occ, occ_range.size() * sizeof(uint2)));
    MCG_CUDA(cudaMalloc((void **)&b->d_companion, comp.size() * sizeof(uint32_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_z_begin, z_begin.size() * sizeof(uint32_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_z_event, nz * sizeof(uint32_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_z_index, std::max<uint32_t>(nb, 1) * sizeof(uint32_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_z_occ_begin, z_occ_begin.size() * sizeof(uint32_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_z_occ, z_occ.size() * sizeof(uint32_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_z_thr, nz * sizeof(uint64_t)));
    MCG_CUDA(cudaMemcpy(b->d_cut_gate, gate.data(), gate.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemcpy(b->d_cut_S, S.data(), nn * sizeof(double), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemcpy(b->d_cut_tab, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemcpy(b->d_cut_logS, logS.data(), b->n_inst * sizeof(double), cudaMemcpyHostToDevice));
    if (nb) {
        MCG_CUDA(cudaMemcpy(b->d_shared, b->shared.data(), nb, cudaMemcpyHostToDevice));
        MCG_CUDA(cudaMemcpy(b->d_z_index, z_index.data(), nb * sizeof(uint32_t), cudaMemcpyHostToDevice));
    }
    MCG_CUDA(cudaMemcpy(b->d_gate_occ, occ_range.data(), occ_range.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemcpy(b->d_companion, comp.data(), comp.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemcpy(b->d_z_begin, z_begin.data(), z_begin.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    if (!b->z_event.empty())
        MCG_CUDA(cudaMemcpy(b->d_z_event, b->z_event.data(), b->z_event.size() * sizeof(uint32_t),
                            cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemcpy(b->d_z_occ_begin, z_occ_begin.data(), z_occ_begin.size() * sizeof(uint32_t),
                        cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMemcpy(b->d_z_occ, z_occ.data(), z_occ.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    b->cut_ready = true;
    return MCG_OK;
}

// Device arrays for n_comp components, grown on demand.
mcg_status ensure_components(mcg_is_batch *b, uint32_t n_comp) {
    if (n_comp <= b->n_comp_cap) return MCG_OK;
    const uint64_t nb = std::max<uint32_t>(b->engine->graph.n_be, 1);
    cudaFree(b->d_be_q);
    cudaFree(b->d_a);
    cudaFree(b->d_C);
    b->d_be_q = nullptr;
    b->d_a = b->d_C = nullptr;
    b->n_comp_cap = 0;
    MCG_CUDA(cudaMalloc((void **)&b->d_be_q, n_comp * nb * sizeof(uint4)));
    MCG_CUDA(cudaMalloc((void **)&b->d_a, n_comp * nb * sizeof(double)));
    MCG_CUDA(cudaMalloc((void **)&b->d_C, (uint64_t)n_comp * b->n_inst * sizeof(double)));
    b->n_comp_cap = n_comp;
    return MCG_OK;
}

}  // namespace

extern "C" {

mcg_status mcg_is_batch_run(mcg_is_batch *b, const uint64_t *q_thr, uint32_t n_def, const uint64_t *q_def,
                            const uint64_t *words_def, uint64_t words_cutset, const uint64_t *q_cutset,
                            uint32_t iteration, uint64_t word_begin, uint64_t word_count, double *tree_sums,
                            double *ce_num, double *kernel_ms) {
    mcg::clear_error();
    if (!b || !q_thr || !tree_sums) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (n_def + 1 > (uint32_t)kMaxComponents)
        return mcg::fail(MCG_ERR_INVALID, "at most " + std::to_string(kMaxComponents - 1) + " defensive proposals");
    if (n_def && (!q_def || !words_def)) return mcg::fail(MCG_ERR_INVALID, "n_defensive > 0 needs q_defensive and words");
    uint64_t def_total = words_cutset;
    for (uint32_t c = 0; c < n_def; ++c) def_total += words_def[c];
    if (def_total > word_count) return mcg::fail(MCG_ERR_INVALID, "defensive and cut-set words exceed word_count");
    if (words_cutset && n_def + 2 > (uint32_t)kMaxComponents)
        return mcg::fail(MCG_ERR_INVALID, "at most " + std::to_string(kMaxComponents - 2) +
                                              " defensive proposals next to the cut-set component");
    mcg_engine *e = b->engine;
    const mcg::Graph &g = e->graph;
    if (word_begin + word_count > (1ull << 32) || word_begin + word_count < word_begin)
        return mcg::fail(MCG_ERR_INVALID, "word range exceeds the 32-bit sample counter");
    if ((uint64_t)iteration + 2 >= (1ull << 26))
        return mcg::fail(MCG_ERR_INVALID, "iteration exceeds the 26-bit pass counter field");
    const uint32_t n_inst = b->n_inst;
    const uint64_t nb = g.n_be;
    // Components that draw words: the main proposal (if it gets any) and
    // every defensive proposal with words.  A single component needs no mixture.
    std::vector<const uint64_t *> comp_q;
    std::vector<uint64_t> comp_words;
    if (word_count - def_total > 0) {
        comp_q.push_back(q_thr);
        comp_words.push_back(word_count - def_total);
    }
    for (uint32_t c = 0; c < n_def; ++c)
        if (words_def[c]) {
            comp_q.push_back(q_def + (uint64_t)c * nb);
            comp_words.push_back(words_def[c]);
        }
    int cut_comp = -1;
    if (words_cutset) {  // shared events from q_cutset, nominal private events plus a forced cut set per sample
        if (!b->cut_ready) {
            MCG_CUDA(cudaSetDevice(e->device));
            const mcg_status cs = build_cut_tables(b);
            if (cs != MCG_OK) return cs;
        }
        b->cut_q.assign(g.be_threshold.begin(), g.be_threshold.end());
        b->z_thr.resize(b->z_event.size());
        for (size_t j = 0; j < b->z_event.size(); ++j) {
            const uint32_t i = b->z_event[j];
            const uint64_t tp = g.be_threshold[i];
            if (q_cutset && tp != 0 && tp < (1ull << 32)) b->cut_q[i] = q_cutset[i];
            b->z_thr[j] = b->cut_q[i];
        }
        cut_comp = (int)comp_q.size();
        comp_q.push_back(b->cut_q.data());
        comp_words.push_back(words_cutset);
    }
    if (comp_q.empty()) comp_q.push_back(q_thr), comp_words.push_back(0);
    const uint32_t nc = (uint32_t)comp_q.size();
    MCG_CUDA(cudaSetDevice(e->device));
    mcg_status st = ensure_components(b, nc);
    if (st != MCG_OK) return st;
    b->beq.resize(nc * std::max<uint64_t>(nb, 1));
    b->a.resize(nc * std::max<uint64_t>(nb, 1));
    b->C.resize((uint64_t)nc * n_inst);
    // log-ratio terms of every (component, tree), split over the host threads
    const uint64_t jobs = (uint64_t)nc * n_inst;
    const unsigned n_thr = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(
        std::max(1u, std::thread::hardware_concurrency()), std::min<uint64_t>(jobs, nb / 65536 + 1)));
    std::vector<std::string> why(n_thr);
    std::vector<char> bad(n_thr, 0);
    auto work = [&](unsigned t) {
        for (uint64_t j = t; j < jobs; j += n_thr) {
            const uint32_t c = (uint32_t)(j / n_inst), k = (uint32_t)(j % n_inst);
            if (!ratio_terms(g, comp_q[c], b->be_begin[k], b->be_begin[k + 1], b->beq.data() + c * nb,
                             b->a.data() + c * nb, b->C[(uint64_t)c * n_inst + k], why[t])) {
                bad[t] = 1;
                return;
            }
        }
    };
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < n_thr; ++t) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    for (unsigned t = 0; t < n_thr; ++t)
        if (bad[t]) return mcg::fail(MCG_ERR_INVALID, why[t]);
    if (cut_comp >= 0) {  // the forcing kernel draws the shared events itself: the sampler leaves them 0
        uint4 *cq = b->beq.data() + (uint64_t)cut_comp * nb;
        for (uint32_t i : b->z_event) cq[i].z = cq[i].w = 0u;
        if (!b->z_thr.empty())
            MCG_CUDA(cudaMemcpyAsync(b->d_z_thr, b->z_thr.data(), b->z_thr.size() * sizeof(uint64_t),
                                     cudaMemcpyHostToDevice, e->stream));
    }
    if (nb) {
        MCG_CUDA(cudaMemcpyAsync(b->d_be_q, b->beq.data(), nc * nb * sizeof(uint4), cudaMemcpyHostToDevice, e->stream));
        MCG_CUDA(cudaMemcpyAsync(b->d_a, b->a.data(), nc * nb * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        MCG_CUDA(cudaMemsetAsync(b->d_ce, 0, nb * sizeof(double), e->stream));
    }
    MCG_CUDA(cudaMemcpyAsync(b->d_C, b->C.data(), (uint64_t)nc * n_inst * sizeof(double), cudaMemcpyHostToDevice,
                             e->stream));
    MCG_CUDA(cudaMemcpyAsync(b->d_sums, b->init.data(), 4ull * n_inst * sizeof(double), cudaMemcpyHostToDevice,
                             e->stream));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
    IsBatchArgs args{};
    args.n_inst = n_inst;
    args.n_comp = nc;
    args.n_be = (uint32_t)nb;
    args.be_begin = b->d_be_begin;
    args.root_row = b->d_root;
    args.a = b->d_a;
    args.C = b->d_C;
    for (uint32_t c = 0; c < nc; ++c)
        args.log_pi[c] = nc > 1 ? std::log((double)comp_words[c] / (double)word_count) : 0.0;
    args.sums = b->d_sums;
    args.ce = ce_num ? b->d_ce : nullptr;
    args.queue = b->d_queue;
    args.cut_comp = cut_comp;
    args.cut_logS = b->d_cut_logS;
    args.cut_gate = b->d_cut_gate;
    args.cut_S = b->d_cut_S;
    args.cut_tree_ok = b->d_tree_ok;
    args.shared = b->d_shared;
    args.companion = b->d_companion;
    args.inputs = e->d_inputs;
    args.n_be_nodes = g.n_be;
    args.error = b->d_cut_error;
    if (cut_comp >= 0) MCG_CUDA(cudaMemsetAsync(b->d_cut_error, 0, sizeof(unsigned int), e->stream));
    e->chunk_hook = [=](cudaStream_t s, const uint64_t *buf, uint64_t W) -> mcg_status {
        IsBatchArgs p = args;
        p.buf = buf;
        p.W = W;
        // one thread per word, or more where that leaves most SMs idle (a
        // few trees in a short pass: each sample's cut-set terms are costly)
        p.split = 1;
        while (p.split < 8 && (uint64_t)n_inst * ((W * p.split + kWeightThreads - 1) / kWeightThreads) < 4ull * sms)
            p.split *= 2;
        p.strips = (uint32_t)((W * p.split + kWeightThreads - 1) / kWeightThreads);
        const uint64_t items = (uint64_t)n_inst * p.strips;
        const uint32_t blocks = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(items, (uint64_t)sms * 8));
        cudaError_t err = cudaMemsetAsync(p.queue, 0, sizeof(unsigned long long), s);
        if (err == cudaSuccess) {
            k_is_weights_batch<<<blocks, kWeightThreads, 0, s>>>(p);
            err = cudaGetLastError();
        }
        if (err != cudaSuccess)
            return mcg::fail(MCG_ERR_CUDA, std::string("k_is_weights_batch: ") + cudaGetErrorString(err));
        return MCG_OK;
    };
    MCG_CUDA(cudaEventRecord(b->ev0, e->stream));
    // component c draws the next comp_words[c] words with its own sampler table
    uint64_t off = 0;
    for (uint32_t c = 0; c < nc && st == MCG_OK; ++c) {
        if (!comp_words[c]) continue;
        e->d_be_sample = b->d_be_q + c * nb;
        e->table_iteration = 0xFFFFFFFFu;  // the sampler table follows the component
        if ((int)c == cut_comp) {
            CutArgs ca{};
            ca.n_inst = n_inst;
            ca.n_be = g.n_be;
            ca.root_row = b->d_root;
            ca.gate = b->d_cut_gate;
            ca.inputs = e->d_inputs;
            ca.S = b->d_cut_S;
            ca.tab = b->d_cut_tab;
            ca.tree_ok = b->d_tree_ok;
            ca.shared = b->d_shared;
            ca.gate_occ = b->d_gate_occ;
            ca.z_begin = b->d_z_begin;
            ca.z_event = b->d_z_event;
            ca.z_thr = b->d_z_thr;
            ca.z_index = b->d_z_index;
            ca.z_occ_begin = b->d_z_occ_begin;
            ca.z_occ = b->d_z_occ;
            ca.seed = mix64_host(((uint64_t)iteration << 32) ^ 0x5bd1e995u);
            ca.error = b->d_cut_error;
            e->sample_hook = [=](cudaStream_t s, uint64_t *buf, uint64_t W, uint64_t wb) -> mcg_status {
                CutArgs x = ca;
                x.buf = buf;
                x.W = W;
                x.word_begin = wb;
                const uint64_t threads = (uint64_t)x.n_inst * W * 64;
                k_cut_force<<<(uint32_t)((threads + 255) / 256), 256, 0, s>>>(x);
                const cudaError_t err = cudaGetLastError();
                if (err != cudaSuccess) return mcg::fail(MCG_ERR_CUDA, std::string("k_cut_force: ") + cudaGetErrorString(err));
                return MCG_OK;
            };
        }
        st = mcg::internal::run_staged(e, iteration, 1, word_begin + off, comp_words[c]);
        e->sample_hook = nullptr;
        off += comp_words[c];
    }
    e->chunk_hook = nullptr;
    e->sample_hook = nullptr;
    e->d_be_sample = nullptr;
    e->table_iteration = 0xFFFFFFFFu;
    if (st != MCG_OK) return st;
    MCG_CUDA(cudaEventRecord(b->ev1, e->stream));
    MCG_CUDA(cudaMemcpyAsync(tree_sums, b->d_sums, 4ull * n_inst * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    if (ce_num && nb)
        MCG_CUDA(cudaMemcpyAsync(ce_num, b->d_ce, nb * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    unsigned int cut_error = 0;
    if (cut_comp >= 0)
        MCG_CUDA(cudaMemcpyAsync(&cut_error, b->d_cut_error, sizeof(unsigned int), cudaMemcpyDeviceToHost, e->stream));
    MCG_CUDA(cudaStreamSynchronize(e->stream));
    if (cut_error & 1u) return mcg::fail(MCG_ERR_STATE, "cut-set descent deeper than its stack (256 nodes)");
    if (cut_error & 2u)
        return mcg::fail(MCG_ERR_STATE, "cut-set count failed (tree deeper than 32 levels, or a failure without "
                                        "a cut set)");
    if (cut_error & 4u)
        return mcg::fail(MCG_ERR_STATE, "cut-set descent above shared events failed (tree deeper than 32 levels)");
    if (kernel_ms) {
        float ms = 0.f;
        MCG_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
        *kernel_ms = ms;
    }
    return MCG_OK;
}

}  // extern "C"
