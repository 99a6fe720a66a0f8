// kernels.cuh -- sm_100a kernels of the Monte Carlo engine.
//
//  k_fused       persistent interpreter: each thread owns one sample word per
//                slab and walks the compiled node program (program_format.h):
//                Philox sampling in registers, gates in an accumulator,
//                shared-memory value slots, popcount tallies reduced per warp
//                into shared-memory counters and flushed once per CTA.
//  k_layer_be    reference dataflow, basic events: one word per thread
//                (src/mc/kernel/basic_event.h:125-142)
//  k_layer_gates reference dataflow, one layer of gates
//                (src/mc/kernel/gate.h:299-362, ATLEAST 506-555)
//  k_layer_tally reference dataflow, tallies (src/mc/kernel/tally.h:322-361)
//  k_sampler_peak register-only sampler: the fused kernel's speed of light.
#pragma once
#include <cstdint>

#include "mcg.h"
#include "philox.cuh"
#include "program_format.h"

namespace mcg {
namespace dev {

constexpr uint64_t kAllOnes = ~0ull;

// Bit-sliced 8-bit counters (mod 256, like the reference's uint8 count).
// Bit-sliced count of up to 15 inputs (4 slices); count >= k for k <= 15.
struct SlicedCount4 {
    uint64_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
    __device__ __forceinline__ void add(uint64_t v) {
        const uint64_t t = c0 & v;
        c0 ^= v;
        const uint64_t t1 = c1 & t;
        c1 ^= t;
        const uint64_t t2 = c2 & t1;
        c2 ^= t1;
        c3 ^= t2;
    }
    __device__ __forceinline__ uint64_t ge(uint32_t k) const {
        const uint64_t c[4] = {c0, c1, c2, c3};
        uint64_t gt = 0, eq = kAllOnes;
#pragma unroll
        for (int b = 3; b >= 0; --b) {
            if ((k >> b) & 1u) {
                eq &= c[b];
            } else {
                gt |= eq & c[b];
                eq &= ~c[b];
            }
        }
        return gt | eq;
    }
};

struct SlicedCount {
    uint64_t c[8];
    __device__ __forceinline__ void clear() {
#pragma unroll
        for (int b = 0; b < 8; ++b) c[b] = 0;
    }
    __device__ __forceinline__ void add(uint64_t v, uint32_t nbits) {
        uint64_t carry = v;
#pragma unroll
        for (int b = 0; b < 8; ++b) {
            if ((uint32_t)b < nbits) {
                const uint64_t t = c[b] & carry;
                c[b] ^= carry;
                carry = t;
            }
        }
    }
    // Per-lane (count >= k) for an 8-bit k.
    __device__ __forceinline__ uint64_t ge(uint32_t k) const {
        uint64_t gt = 0, eq = kAllOnes;
#pragma unroll
        for (int b = 7; b >= 0; --b) {
            if ((k >> b) & 1u) {
                eq &= c[b];
            } else {
                gt |= eq & c[b];
                eq &= ~c[b];
            }
        }
        return gt | eq;
    }
};

__device__ __forceinline__ uint64_t load_slot(uint32_t ref, const uint64_t *my_slots, const uint64_t *my_scratch,
                                              uint32_t nt, uint64_t stride) {
    if (ref & kSlotGlobal) return my_scratch[(uint64_t)(ref & kSlotIndexMask) * stride];
    return my_slots[(uint32_t)ref * nt];
}

__device__ __forceinline__ void store_slot(uint32_t ref, uint64_t v, uint64_t *my_slots, uint64_t *my_scratch,
                                           uint32_t nt, uint64_t stride) {
    if (ref == kNoSlot) return;
    if (ref & kSlotGlobal) my_scratch[(uint64_t)(ref & kSlotIndexMask) * stride] = v;
    else my_slots[(uint32_t)ref * nt] = v;
}

// Walks one node program for this thread's sample word.  With THR_TABLE the
// basic-event ops carry an index into thr (a per-instance uint64 threshold
// table) instead of the threshold itself.  tally(index, count) is called by
// lane 0 of each warp with the warp's popcount sum for a TALLY op.
template <int NT, int MF, int PF, bool THR_TABLE, class Tally>
__device__ __forceinline__ void interpret(const uint4 *__restrict__ ops, const WordCtx &ctx, uint32_t t3, bool valid,
                                          uint64_t *my_slots, uint64_t *my_scratch, uint64_t stride,
                                          const uint64_t *__restrict__ thr, Tally &&tally) {
    const uint32_t lane = threadIdx.x & 31u;
    uint64_t acc = 0, last = 0;
    uint32_t conn = 0, kk = 0, nbits = 0;
    SlicedCount cnt;
    cnt.clear();
    const uint4 *p = ops;
    uint4 op = __ldg(p);
    while (true) {
        const uint4 nxt = __ldg(p + 1);
        const uint32_t code = op.x & kOpMask;
        if (code == kOpHalt) break;
        // Value of the op: one sampler call site keeps the unrolled Philox
        // body in the instruction cache once.
        uint64_t v = 0;
        if (code == kOpInBe || code == kOpBeDef) {
            if constexpr (THR_TABLE) {
                const uint64_t t = thr[op.z];
                if (t >= (1ull << 32)) v = kAllOnes;
                else if (t == 0) v = 0;
                else v = be_word<MF, PF>(op.y, op.w, ctx, t3, (uint32_t)t);
            } else {
                v = be_word<MF, PF>(op.y, op.w, ctx, t3, op.z);
            }
        } else if (code == kOpInSlot) {
            v = load_slot(op.y, my_slots, my_scratch, NT, stride);
        } else if (code == kOpInConst || code == kOpConstDef) {
            v = ((uint64_t)op.z << 32) | op.y;
        }
        if (code == kOpInBe || code == kOpInSlot || code == kOpInConst) {
            if (op.x & kNegBit) v = ~v;
            switch (conn) {
                case MCG_AND: case MCG_NAND: acc &= v; break;
                case MCG_OR: case MCG_NOR: acc |= v; break;
                case MCG_XOR: acc ^= v; break;
                case MCG_ATLEAST: cnt.add(v, nbits); break;
                default: acc = v; break;  // NOT, NULL: the last input wins
            }
        } else if (code == kOpBeDef || code == kOpConstDef) {
            last = v;
            store_slot(op.x >> 8, last, my_slots, my_scratch, NT, stride);
        } else if (code == kOpBegin) {
            conn = (op.x >> 8) & 0xFFu;
            kk = (op.x >> 16) & 0xFFu;
            nbits = (op.x >> 24) & 0xFu;
            acc = (conn == MCG_AND || conn == MCG_NAND) ? kAllOnes : 0ull;
            if (conn == MCG_ATLEAST) cnt.clear();
        } else if (code == kOpEnd) {
            if (conn == MCG_ATLEAST) last = cnt.ge(kk);
            else if (conn == MCG_NAND || conn == MCG_NOR || conn == MCG_NOT) last = ~acc;
            else last = acc;
            store_slot(op.y, last, my_slots, my_scratch, NT, stride);
        } else if (code == kOpTally) {
            uint32_t c = valid ? (uint32_t)__popcll(last) : 0u;
            c = __reduce_add_sync(0xFFFFFFFFu, c);
            if (lane == 0) tally(op.y, c);
        }
        op = nxt;
        ++p;
    }
}

struct FusedArgs {
    const uint4 *ops;
    uint32_t smem_slots;
    uint64_t *scratch;        // [global_slots][grid * NT]
    uint64_t scratch_stride;  // grid * NT of the allocation
    unsigned long long *tally;
    uint32_t n_tally;
    uint32_t tally_in_smem;
    uint32_t iteration_first;
    uint32_t n_iterations;
    uint64_t word_begin;
    uint64_t word_count;
};

template <int NT, int MINB, int MF, int PF>
__global__ void __launch_bounds__(NT, MINB) k_fused(FusedArgs a) {
    extern __shared__ __align__(16) uint64_t smem[];
    const uint32_t tid = threadIdx.x;
    unsigned long long *s_tally = reinterpret_cast<unsigned long long *>(smem + (size_t)a.smem_slots * NT);
    if (a.tally_in_smem) {
        for (uint32_t i = tid; i < a.n_tally; i += NT) s_tally[i] = 0ull;
        __syncthreads();
    }
    unsigned long long *tally = a.tally_in_smem ? s_tally : a.tally;
    const uint64_t gtid = (uint64_t)blockIdx.x * NT + tid;
    const uint64_t total_threads = (uint64_t)gridDim.x * NT;
    uint64_t *my_slots = smem + tid;
    uint64_t *my_scratch = a.scratch + gtid;
    auto add = [tally](uint32_t idx, uint32_t c) { atomicAdd(&tally[idx], (unsigned long long)c); };

    for (uint32_t it = 0; it < a.n_iterations; ++it) {
        const uint32_t t3 = (a.iteration_first + it + 1u) << 6;
        for (uint64_t base = 0; base < a.word_count; base += total_threads) {
            const uint64_t j = base + gtid;
            const WordCtx ctx = make_word_ctx<MF>((uint32_t)(a.word_begin + j));
            interpret<NT, MF, PF, false>(a.ops, ctx, t3, j < a.word_count, my_slots, my_scratch, a.scratch_stride,
                                         nullptr, add);
        }
    }
    if (a.tally_in_smem) {
        __syncthreads();
        for (uint32_t i = tid; i < a.n_tally; i += NT) {
            const unsigned long long c = s_tally[i];
            if (c) atomicAdd(&a.tally[i], c);
        }
    }
}

// Batched instances (uncertainty analysis): a persistent work queue over
// (instance, slab) items; an instance runs its tree's program with its own
// threshold table over words [0, words_per_instance) of pass `iteration`
// and counts the ones of every TALLY op into inst_ones[instance].
struct BatchArgs {
    const uint4 *ops;                  // all tree programs, concatenated
    const uint32_t *tree_op_offset;    // first op of each tree's program
    const uint32_t *inst_tree;         // tree of each instance
    const uint64_t *inst_thr_offset;   // first threshold of each instance
    const uint64_t *thr;               // thresholds (uint64, 0 .. 2^32)
    uint32_t n_instances;
    uint32_t slabs_per_instance;
    uint64_t words_per_instance;
    uint32_t iteration;
    uint32_t smem_slots;
    uint64_t *scratch;
    uint64_t scratch_stride;
    unsigned int *queue;               // next item; zero before the launch
    unsigned long long *inst_ones;
    // k_fused_batch_k: groups of up to K consecutive instances of one tree
    const uint32_t *group_first;
    const uint32_t *group_size;
    uint32_t n_groups;
};

template <int NT, int MINB, int MF, int PF>
__global__ void __launch_bounds__(NT, MINB) k_fused_batch(BatchArgs a) {
    extern __shared__ __align__(16) uint64_t smem[];
    __shared__ unsigned int s_item;
    const uint32_t tid = threadIdx.x;
    const uint64_t gtid = (uint64_t)blockIdx.x * NT + tid;
    uint64_t *my_slots = smem + tid;
    uint64_t *my_scratch = a.scratch + gtid;
    const uint32_t t3 = (a.iteration + 1u) << 6;
    const unsigned int n_items = a.n_instances * a.slabs_per_instance;
    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(a.queue, 1u);
        __syncthreads();
        const unsigned int item = s_item;
        if (item >= n_items) break;
        const uint32_t inst = item / a.slabs_per_instance;
        const uint64_t j = (uint64_t)(item % a.slabs_per_instance) * NT + tid;
        const WordCtx ctx = make_word_ctx<MF>((uint32_t)j);
        unsigned long long *ones = a.inst_ones + inst;
        auto add = [ones](uint32_t, uint32_t c) { atomicAdd(ones, (unsigned long long)c); };
        interpret<NT, MF, PF, true>(a.ops + a.tree_op_offset[a.inst_tree[inst]], ctx, t3, j < a.words_per_instance,
                                    my_slots, my_scratch, a.scratch_stride, a.thr + a.inst_thr_offset[inst], add);
    }
}

// Slot planes of the K-wide interpreter: slot s of instance k at [s * K + k].
template <int K>
__device__ __forceinline__ uint64_t load_slot_k(uint32_t ref, int k, const uint64_t *my_slots,
                                                const uint64_t *my_scratch, uint32_t nt, uint64_t stride) {
    if (ref & kSlotGlobal) return my_scratch[((uint64_t)(ref & kSlotIndexMask) * K + k) * stride];
    return my_slots[((uint32_t)ref * K + k) * nt];
}

template <int K>
__device__ __forceinline__ void store_slot_k(uint32_t ref, int k, uint64_t v, uint64_t *my_slots,
                                             uint64_t *my_scratch, uint32_t nt, uint64_t stride) {
    if (ref == kNoSlot) return;
    if (ref & kSlotGlobal) my_scratch[((uint64_t)(ref & kSlotIndexMask) * K + k) * stride] = v;
    else my_slots[((uint32_t)ref * K + k) * nt] = v;
}

// The interpreter over K instances of one tree that differ only in their
// thresholds (draws of an uncertainty analysis): every op acts on K words, a
// basic event's 16 Philox calls run once and are compared with the K
// instances' thresholds (thr[k][op.z]), so word k equals what interpret gives
// instance k.  With ATL, ATLEAST gates of at most 15 inputs count in four
// bit slices per instance; without it the program must have no ATLEAST gate
// (the batch runs wider ones one instance at a time).  tally(k, count) is
// called by lane 0 with instance k's warp popcount sum.
template <int NT, int MF, int PF, int K, bool ATL, class Tally>
__device__ __forceinline__ void interpret_k(const uint4 *__restrict__ ops, const WordCtx &ctx, uint32_t t3,
                                            bool valid, uint64_t *my_slots, uint64_t *my_scratch, uint64_t stride,
                                            const uint64_t *const *thr, Tally &&tally) {
    const uint32_t lane = threadIdx.x & 31u;
    uint64_t acc[K], last[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = last[k] = 0ull;
    SlicedCount4 cnt[K];
    uint32_t conn = 0, kk = 0;
    const uint4 *p = ops;
    uint4 op = __ldg(p);
    while (true) {
        const uint4 nxt = __ldg(p + 1);
        const uint32_t code = op.x & kOpMask;
        if (code == kOpHalt) break;
        uint64_t v[K];
#pragma unroll
        for (int k = 0; k < K; ++k) v[k] = 0ull;
        if (code == kOpInBe || code == kOpBeDef) {
            uint32_t t32[K];
            uint32_t ones = 0, zeros = 0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const uint64_t t = thr[k][op.z];
                t32[k] = (uint32_t)t;
                if (t >= (1ull << 32)) {
                    ones |= 1u << k;
                    t32[k] = 1u;
                } else if (t == 0) {
                    zeros |= 1u << k;
                    t32[k] = 1u;
                }
            }
            if ((ones | zeros) != (1u << K) - 1u) be_words<MF, PF, K>(op.y, op.w, ctx, t3, t32, v);
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if ((ones >> k) & 1u) v[k] = kAllOnes;
                else if ((zeros >> k) & 1u) v[k] = 0ull;
            }
        } else if (code == kOpInSlot) {
#pragma unroll
            for (int k = 0; k < K; ++k) v[k] = load_slot_k<K>(op.y, k, my_slots, my_scratch, NT, stride);
        } else if (code == kOpInConst || code == kOpConstDef) {
#pragma unroll
            for (int k = 0; k < K; ++k) v[k] = ((uint64_t)op.z << 32) | op.y;
        }
        if (code == kOpInBe || code == kOpInSlot || code == kOpInConst) {
            if (op.x & kNegBit) {
#pragma unroll
                for (int k = 0; k < K; ++k) v[k] = ~v[k];
            }
            switch (conn) {
                case MCG_AND: case MCG_NAND:
#pragma unroll
                    for (int k = 0; k < K; ++k) acc[k] &= v[k];
                    break;
                case MCG_OR: case MCG_NOR:
#pragma unroll
                    for (int k = 0; k < K; ++k) acc[k] |= v[k];
                    break;
                case MCG_XOR:
#pragma unroll
                    for (int k = 0; k < K; ++k) acc[k] ^= v[k];
                    break;
                case MCG_ATLEAST:
                    if constexpr (ATL) {
#pragma unroll
                        for (int k = 0; k < K; ++k) cnt[k].add(v[k]);
                    }
                    break;
                default:  // NOT, NULL: the last input wins
#pragma unroll
                    for (int k = 0; k < K; ++k) acc[k] = v[k];
                    break;
            }
        } else if (code == kOpBeDef || code == kOpConstDef) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                last[k] = v[k];
                store_slot_k<K>(op.x >> 8, k, last[k], my_slots, my_scratch, NT, stride);
            }
        } else if (code == kOpBegin) {
            conn = (op.x >> 8) & 0xFFu;
            kk = (op.x >> 16) & 0xFFu;
            const uint64_t init = (conn == MCG_AND || conn == MCG_NAND) ? kAllOnes : 0ull;
#pragma unroll
            for (int k = 0; k < K; ++k) acc[k] = init;
            if constexpr (ATL) {
                if (conn == MCG_ATLEAST) {
#pragma unroll
                    for (int k = 0; k < K; ++k) cnt[k] = SlicedCount4{};
                }
            }
        } else if (code == kOpEnd) {
            const bool inv = conn == MCG_NAND || conn == MCG_NOR || conn == MCG_NOT;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (ATL && conn == MCG_ATLEAST) last[k] = kk > 15 ? 0ull : cnt[k].ge(kk);  // at most 15 inputs
                else last[k] = inv ? ~acc[k] : acc[k];
                store_slot_k<K>(op.y, k, last[k], my_slots, my_scratch, NT, stride);
            }
        } else if (code == kOpTally) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, valid ? (uint32_t)__popcll(last[k]) : 0u);
                if (lane == 0) tally((uint32_t)k, c);
            }
        }
        op = nxt;
        ++p;
    }
}

// Batched instances K at a time: a work item is (group, slab), a group up to
// K consecutive instances of one tree; missing members of a short group
// repeat its first instance's thresholds and add nothing to any tally.
template <int NT, int MINB, int MF, int PF, int K, bool ATL>
__global__ void __launch_bounds__(NT, MINB) k_fused_batch_k(BatchArgs a) {
    extern __shared__ __align__(16) uint64_t smem[];
    __shared__ unsigned int s_item;
    const uint32_t tid = threadIdx.x;
    const uint64_t gtid = (uint64_t)blockIdx.x * NT + tid;
    uint64_t *my_slots = smem + tid;
    uint64_t *my_scratch = a.scratch + gtid;
    const uint32_t t3 = (a.iteration + 1u) << 6;
    const unsigned int n_items = a.n_groups * a.slabs_per_instance;
    while (true) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(a.queue, 1u);
        __syncthreads();
        const unsigned int item = s_item;
        if (item >= n_items) break;
        const uint32_t grp = item / a.slabs_per_instance;
        const uint64_t j = (uint64_t)(item % a.slabs_per_instance) * NT + tid;
        const uint32_t first = a.group_first[grp], n = a.group_size[grp];
        const uint64_t *thr[K];
#pragma unroll
        for (int k = 0; k < K; ++k) thr[k] = a.thr + a.inst_thr_offset[first + ((uint32_t)k < n ? (uint32_t)k : 0u)];
        const WordCtx ctx = make_word_ctx<MF>((uint32_t)j);
        unsigned long long *ones = a.inst_ones + first;
        auto add = [ones, n](uint32_t k, uint32_t c) {
            if (k < n) atomicAdd(ones + k, (unsigned long long)c);
        };
        interpret_k<NT, MF, PF, K, ATL>(a.ops + a.tree_op_offset[a.inst_tree[first]], ctx, t3, j < a.words_per_instance,
                                   my_slots, my_scratch, a.scratch_stride, thr, add);
    }
}

// ---------------------------------------------------------------------------
// Reference dataflow (layered).  Node words live in buf[node * W + w].

// Basic events: be[e] = {pdag_idx+1, event_idx+1, thr_lo, thr_hi}.
template <int MF, int PF>
__global__ void __launch_bounds__(256) k_layer_be(const uint4 *__restrict__ be, uint32_t n_be, uint64_t W,
                                                  uint64_t word_begin, uint32_t t3, uint64_t *__restrict__ buf) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t e = blockIdx.y + gridDim.y * blockIdx.z;
    if (w >= W || e >= n_be) return;
    const uint4 r = be[e];
    const uint64_t thr = ((uint64_t)r.w << 32) | r.z;
    uint64_t v;
    if (thr == 0) v = 0;
    else if (thr >= (1ull << 32)) v = kAllOnes;
    else v = be_word<MF, PF>(r.x, r.y, make_word_ctx<MF>((uint32_t)(word_begin + w)), t3, (uint32_t)thr);
    buf[(uint64_t)e * W + w] = v;
}

// One layer of gates; gate ids listed in layer_gates.  meta[g] = {op | k<<8, in_begin, in_count, neg_count}.
// ATLEAST counts each bit lane with a uint8 counter, as the reference kernel does.
static __global__ void __launch_bounds__(256) k_layer_gates(const uint4 *__restrict__ meta, const uint32_t *__restrict__ inputs,
                                                     const uint32_t *__restrict__ layer_gates, uint32_t n_layer,
                                                     uint32_t n_be, uint64_t W, uint64_t *__restrict__ buf) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t li = blockIdx.y + gridDim.y * blockIdx.z;
    if (w >= W || li >= n_layer) return;
    const uint32_t gi = layer_gates[li];
    const uint4 m = meta[gi];
    const uint32_t op = m.x & 0xFFu;
    const uint32_t n = m.z;
    const uint32_t off = n - m.w;
    const uint32_t *in = inputs + m.y;
    uint64_t r;
    if (op == MCG_ATLEAST) {
        const uint8_t k = (uint8_t)(m.x >> 8);
        r = 0;
        for (uint32_t lane = 0; lane < 64; ++lane) {
            const uint64_t mask = 1ull << lane;
            uint8_t cnt = 0;
            for (uint32_t i = 0; i < n; ++i) {
                const uint64_t v = buf[(uint64_t)in[i] * W + w];
                cnt += (uint8_t)((((i < off) ? v : ~v) & mask) ? 1 : 0);
            }
            if (cnt >= k) r |= mask;
        }
    } else {
        r = (op == MCG_AND || op == MCG_NAND) ? kAllOnes : 0ull;
        for (uint32_t i = 0; i < n; ++i) {
            uint64_t v = buf[(uint64_t)in[i] * W + w];
            if (i >= off) v = ~v;
            if (op == MCG_OR || op == MCG_NOR) r |= v;
            else if (op == MCG_AND || op == MCG_NAND) r &= v;
            else if (op == MCG_XOR) r ^= v;
            else r = v;
        }
        if (op == MCG_NAND || op == MCG_NOR || op == MCG_NOT) r = ~r;
    }
    buf[(uint64_t)(n_be + gi) * W + w] = r;
}

// Tallies: popcount, block reduction, one atomic per block and node.
// tally_idx (optional) maps row t of tally_nodes to its counter.
static __global__ void __launch_bounds__(256) k_layer_tally(const uint32_t *__restrict__ tally_nodes, uint32_t n_tally,
                                                     uint64_t W, const uint64_t *__restrict__ buf,
                                                     unsigned long long *__restrict__ ones,
                                                     const uint32_t *__restrict__ tally_idx) {
    __shared__ uint32_t warp_sums[8];
    const uint32_t t = blockIdx.y + gridDim.y * blockIdx.z;
    if (t >= n_tally) return;
    uint32_t c = 0;
    const uint64_t *row = buf + (uint64_t)tally_nodes[t] * W;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < W; w += (uint64_t)gridDim.x * blockDim.x)
        c += (uint32_t)__popcll(row[w]);
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31u) == 0) warp_sums[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (uint32_t i = 0; i < (blockDim.x >> 5); ++i) s += warp_sums[i];
        if (s) atomicAdd(&ones[tally_idx ? tally_idx[t] : t], s);
    }
}

// ---------------------------------------------------------------------------
// Staged pipeline.  Phase A samples basic-event words into buf rows
// [0, n_be); phase B evaluates one layer of gates per launch into rows
// n_be + g, with tallies fused.

// Per-pass event table (philox.cuh): thread (e, g) fills entry g of event e.
template <int MF>
__global__ void __launch_bounds__(256) k_event_table(const uint4 *__restrict__ be, uint32_t n_be, uint32_t t3,
                                                     uint2 *__restrict__ table) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)n_be * kEventTableStride) return;
    const uint32_t e = (uint32_t)(i / kEventTableStride);
    const int g = (int)(i % kEventTableStride);
    event_table_entry<MF>(be[e].x, t3, g, table[i]);
}

// Phase A: thread (w, group) samples word w of events [group * EPT, +EPT)
// using the pass's event table.  Launched with dynamic shared memory that
// only caps the blocks per SM, leaving room for gate-phase blocks.
template <int MF, int PF, int EPT>
__global__ void __launch_bounds__(256, 6) k_stage_be(const uint4 *__restrict__ be, const uint2 *__restrict__ table,
                                                  uint32_t n_be, uint64_t W, uint64_t word_begin,
                                                  uint64_t *__restrict__ buf) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t e0 = (blockIdx.y + gridDim.y * blockIdx.z) * EPT;
    if (w >= W || e0 >= n_be) return;
    const WordCtx ctx = make_word_ctx<MF>((uint32_t)(word_begin + w));
#pragma unroll 1
    for (uint32_t i = 0; i < EPT; ++i) {
        const uint32_t e = e0 + i;
        if (e >= n_be) break;
        const uint4 r = be[e];
        uint64_t v;
        if (r.w != 0) v = kAllOnes;           // threshold 2^32
        else if (r.z == 0) v = 0;             // threshold 0
        else v = be_word_tab<MF, PF>(r.y, ctx, table + (uint64_t)e * kEventTableStride, r.z);
        buf[(uint64_t)e * W + w] = v;
    }
}

// Phase B: gate layer_gates[blockIdx.y] for words [blockIdx.x * NT * WPT, ...),
// WPT words per thread at stride NT (coalesced).  meta[g] = {op | k << 8 |
// nbits << 16, in_begin, in_count, neg_count}; gate_tally[g] = {offset, count}
// into tally_list.  Each block adds its popcount once per tally entry.
template <int NT, int WPT>
__global__ void __launch_bounds__(NT) k_stage_gates(const uint4 *__restrict__ meta, const uint32_t *__restrict__ inputs,
                                                     const uint32_t *__restrict__ layer_gates, uint32_t n_layer,
                                                     uint32_t n_be, uint64_t W, uint64_t *__restrict__ buf,
                                                     const uint2 *__restrict__ gate_tally,
                                                     const uint32_t *__restrict__ tally_list,
                                                     unsigned long long *__restrict__ ones) {
    constexpr uint32_t kMaxIn = 8;  // inputs loaded up front (memory-level parallelism)
    __shared__ uint32_t warp_sums[NT / 32];
    const uint32_t li = blockIdx.y + gridDim.y * blockIdx.z;
    if (li >= n_layer) return;
    const uint32_t gi = layer_gates[li];
    const uint4 m = meta[gi];
    const uint32_t op = m.x & 0xFFu;
    const uint32_t kk = (m.x >> 8) & 0xFFu;
    const uint32_t nbits = (m.x >> 16) & 0xFu;
    const uint32_t n = m.z;
    const uint32_t off = n - m.w;
    const uint32_t *in = inputs + m.y;
    uint64_t *out = buf + (uint64_t)(n_be + gi) * W;
    const uint64_t base = (uint64_t)blockIdx.x * NT * WPT + threadIdx.x;
    uint64_t r[WPT];
    if (n <= kMaxIn) {
        uint64_t v[kMaxIn][WPT];
#pragma unroll
        for (uint32_t i = 0; i < kMaxIn; ++i) {
            if (i < n) {
                const uint64_t *row = buf + (uint64_t)in[i] * W;
#pragma unroll
                for (int k = 0; k < WPT; ++k) {
                    const uint64_t w = base + (uint64_t)k * NT;
                    v[i][k] = (w < W) ? row[w] : 0ull;
                }
            }
        }
#pragma unroll
        for (int k = 0; k < WPT; ++k) {
            if (op == MCG_ATLEAST) {
                SlicedCount cnt;
                cnt.clear();
#pragma unroll
                for (uint32_t i = 0; i < kMaxIn; ++i)
                    if (i < n) cnt.add(i >= off ? ~v[i][k] : v[i][k], nbits);
                r[k] = cnt.ge(kk);
            } else {
                uint64_t a = (op == MCG_AND || op == MCG_NAND) ? kAllOnes : 0ull;
#pragma unroll
                for (uint32_t i = 0; i < kMaxIn; ++i) {
                    if (i < n) {
                        const uint64_t x = i >= off ? ~v[i][k] : v[i][k];
                        if (op == MCG_OR || op == MCG_NOR) a |= x;
                        else if (op == MCG_AND || op == MCG_NAND) a &= x;
                        else if (op == MCG_XOR) a ^= x;
                        else a = x;
                    }
                }
                r[k] = (op == MCG_NAND || op == MCG_NOR || op == MCG_NOT) ? ~a : a;
            }
        }
    } else {
#pragma unroll
        for (int k = 0; k < WPT; ++k) {
            const uint64_t w = base + (uint64_t)k * NT;
            r[k] = 0;
            if (w >= W) continue;
            if (op == MCG_ATLEAST) {
                SlicedCount cnt;
                cnt.clear();
                for (uint32_t i = 0; i < n; ++i) {
                    const uint64_t x = buf[(uint64_t)in[i] * W + w];
                    cnt.add(i >= off ? ~x : x, nbits);
                }
                r[k] = cnt.ge(kk);
            } else {
                uint64_t a = (op == MCG_AND || op == MCG_NAND) ? kAllOnes : 0ull;
                for (uint32_t i = 0; i < n; ++i) {
                    uint64_t x = buf[(uint64_t)in[i] * W + w];
                    if (i >= off) x = ~x;
                    if (op == MCG_OR || op == MCG_NOR) a |= x;
                    else if (op == MCG_AND || op == MCG_NAND) a &= x;
                    else if (op == MCG_XOR) a ^= x;
                    else a = x;
                }
                r[k] = (op == MCG_NAND || op == MCG_NOR || op == MCG_NOT) ? ~a : a;
            }
        }
    }
    uint32_t count = 0;
#pragma unroll
    for (int k = 0; k < WPT; ++k) {
        const uint64_t w = base + (uint64_t)k * NT;
        if (w < W) {
            out[w] = r[k];
            count += (uint32_t)__popcll(r[k]);
        }
    }
    const uint2 t = gate_tally[gi];
    if (t.y == 0) return;  // uniform per block
    count = __reduce_add_sync(0xFFFFFFFFu, count);
    if ((threadIdx.x & 31u) == 0) warp_sums[threadIdx.x >> 5] = count;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (uint32_t i = 0; i < NT / 32; ++i) s += warp_sums[i];
        if (s)
            for (uint32_t j = 0; j < t.y; ++j) atomicAdd(&ones[tally_list[t.x + j]], s);
    }
}

// Strip mode: one persistent kernel per pass.  A block takes strips of 256
// consecutive words from a queue; warp w owns words [32 w, 32 w + 32) of
// the strip and a private scratch block of n_nodes rows x 32 words.  Lane l
// first samples its word of every basic event (one Philox word per event,
// event table of the pass), then evaluates every gate in layer order for the
// same word, and adds the popcounts of tallied nodes into the block's
// shared-memory counters.  A lane only reads the column it wrote, so the
// only barrier is the strip hand-out: the eight warps of a block walk the
// events together (the table rows they read stay in L1), while the blocks
// on an SM drift apart, so the memory-bound gate work of some blocks runs
// under the multiply-bound sampling of the others.
constexpr int kStripLanes = 32;
constexpr int kStripThreads = 256;

struct StripArgs {
    const uint4 *be;              // {pdag + 1, event + 1, thr lo, thr hi}
    const uint2 *table;           // event table of the pass
    uint32_t n_be, n_nodes;
    const uint4 *smeta;           // per gate: op | k << 8 | nbits << 16, in_begin, in_count, neg_count
    const uint32_t *inputs;
    const uint4 *groups;          // per group two records: {count | fan-in << 8 | single << 24, gin offset,
                                  // ginfo offset, outinv} and the output nodes of its gates
    uint32_t n_groups;
    const uint32_t *gin;          // group inputs, slot-major, kStripGroup records per slot: node << 1 | flip
    const uint4 *ginfo;           // per grouped gate: {output node, tally offset, tally count, gate id}
    const uint32_t *tally_list;
    const uint32_t *be_tally_nodes, *be_tally_idx;
    uint32_t n_be_tally;
    uint32_t n_tally;
    uint32_t tally_in_smem;
    unsigned long long *ones;
    uint64_t *scratch;            // per warp: n_nodes x 32 words
    uint64_t word_begin, word_count;
    unsigned long long *queue;
};

__device__ __forceinline__ void strip_tally(const StripArgs &a, unsigned long long *s_ones, uint32_t idx,
                                            uint32_t c) {
    if (a.tally_in_smem) atomicAdd(&s_ones[idx], (unsigned long long)c);
    else atomicAdd(&a.ones[idx], (unsigned long long)c);
}

// Gate groups of the strip kernel: up to kStripGroup gates of one layer
// evaluated together in the OR form r = outinv ^ OR_i (x_i ^ flip_i); an
// input record is node << 1 | flip, kStripNoInput an empty slot.
constexpr uint32_t kStripGroup = 4;
constexpr uint32_t kStripGroupMaxIn = 8;
constexpr uint32_t kStripNoInput = 0xFFFFFFFFu;
static_assert(kStripGroup == 4, "k_strip's group loop packs four gates' tallies into two reductions");

__device__ __forceinline__ uint64_t strip_in(const uint64_t *col, uint32_t rec) {
    uint64_t x = 0;
    if (rec != kStripNoInput) {
        x = col[(uint64_t)(rec >> 1) * kStripLanes];
        if (rec & 1u) x = ~x;
    }
    return x;
}

// Tally of one gate word column: warp sum of the valid lanes' popcounts,
// added by lane 0 to every tally slot of the node.
__device__ __forceinline__ void strip_gate_tally(const StripArgs &a, unsigned long long *s_ones, const uint4 &f,
                                                 uint64_t r, bool valid, uint32_t lane) {
    if (f.z) {
        const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, valid ? (uint32_t)__popcll(r) : 0u);
        if (lane == 0 && c)
            for (uint32_t j = 0; j < f.z; ++j) strip_tally(a, s_ones, a.tally_list[f.y + j], c);
    }
}


// Not inlined: the one-gate path (ATLEAST counters, wide fan-in loops) then
// keeps its registers to itself, and k_strip's sampler and gate groups spill
// 36 bytes instead of 376 at 40 registers.
static __device__ __noinline__ uint64_t strip_gate(const StripArgs &a, const uint64_t *col, uint32_t gi) {
    constexpr uint32_t kMaxIn = 8;
    const uint4 m = a.smeta[gi];
    const uint32_t op = m.x & 0xFFu, kk = (m.x >> 8) & 0xFFu, nbits = (m.x >> 16) & 0xFu;
    const uint32_t n = m.z, off = n - m.w;
    const uint32_t *in = a.inputs + m.y;
    if (op == MCG_ATLEAST) {
        if (n <= kMaxIn) {
            // counts of at most 8 fit 4 slices; k > 8 can never be reached
            SlicedCount4 cnt;
#pragma unroll
            for (uint32_t i0 = 0; i0 < kMaxIn; i0 += 4) {
                uint64_t v[4];
#pragma unroll
                for (uint32_t j = 0; j < 4; ++j)
                    if (i0 + j < n) v[j] = col[(uint64_t)in[i0 + j] * kStripLanes];
#pragma unroll
                for (uint32_t j = 0; j < 4; ++j)
                    if (i0 + j < n) cnt.add(i0 + j >= off ? ~v[j] : v[j]);
            }
            return kk > 8 ? 0ull : cnt.ge(kk);
        }
        SlicedCount cnt;
        cnt.clear();
        for (uint32_t i = 0; i < n; ++i) {
            const uint64_t x = col[(uint64_t)in[i] * kStripLanes];
            cnt.add(i >= off ? ~x : x, nbits);
        }
        return cnt.ge(kk);
    }
    uint64_t acc = (op == MCG_AND || op == MCG_NAND) ? kAllOnes : 0ull;
    if (n <= kMaxIn) {
#pragma unroll
        for (uint32_t i0 = 0; i0 < kMaxIn; i0 += 4) {
            uint64_t v[4];
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j)
                if (i0 + j < n) v[j] = col[(uint64_t)in[i0 + j] * kStripLanes];
#pragma unroll
            for (uint32_t j = 0; j < 4; ++j) {
                if (i0 + j < n) {
                    const uint64_t x = i0 + j >= off ? ~v[j] : v[j];
                    if (op == MCG_OR || op == MCG_NOR) acc |= x;
                    else if (op == MCG_AND || op == MCG_NAND) acc &= x;
                    else if (op == MCG_XOR) acc ^= x;
                    else acc = x;
                }
            }
        }
    } else {
        for (uint32_t i = 0; i < n; ++i) {
            uint64_t x = col[(uint64_t)in[i] * kStripLanes];
            if (i >= off) x = ~x;
            if (op == MCG_OR || op == MCG_NOR) acc |= x;
            else if (op == MCG_AND || op == MCG_NAND) acc &= x;
            else if (op == MCG_XOR) acc ^= x;
            else acc = x;
        }
    }
    return (op == MCG_NAND || op == MCG_NOR || op == MCG_NOT) ? ~acc : acc;
}

template <int MF, int PF, int MINB>
__global__ void __launch_bounds__(kStripThreads, MINB) k_strip(StripArgs a) {
    extern __shared__ unsigned long long s_ones[];
    __shared__ unsigned long long s_strip;
    const uint32_t lane = threadIdx.x & 31u;
    if (a.tally_in_smem)
        for (uint32_t i = threadIdx.x; i < a.n_tally; i += blockDim.x) s_ones[i] = 0;
    const uint64_t gwarp = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    uint64_t *col = a.scratch + gwarp * (uint64_t)a.n_nodes * kStripLanes + lane;
    const uint64_t n_strips = (a.word_count + kStripThreads - 1) / kStripThreads;
    for (;;) {
        __syncthreads();  // s_strip is free again (and the tally counters are zeroed)
        if (threadIdx.x == 0) s_strip = atomicAdd(a.queue, 1ull);
        __syncthreads();
        const unsigned long long strip = s_strip;
        if (strip >= n_strips) break;
        const uint64_t wl = strip * kStripThreads + threadIdx.x;
        const bool valid = wl < a.word_count;
        const WordCtx ctx = make_word_ctx<MF>((uint32_t)(a.word_begin + wl));
#pragma unroll 1
        for (uint32_t e = 0; e < a.n_be; ++e) {
            const uint4 r = a.be[e];
            uint64_t v;
            if (r.w != 0) v = kAllOnes;
            else if (r.z == 0) v = 0;
            else v = be_word_tab<MF, PF>(r.y, ctx, a.table + (uint64_t)e * kEventTableStride, r.z);
            col[(uint64_t)e * kStripLanes] = v;
        }
        for (uint32_t j = 0; j < a.n_be_tally; ++j) {
            const uint64_t v = col[(uint64_t)a.be_tally_nodes[j] * kStripLanes];
            const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, valid ? (uint32_t)__popcll(v) : 0u);
            if (lane == 0 && c) strip_tally(a, s_ones, a.be_tally_idx[j], c);
        }
        // gates, layer by layer, a group at a time: no gate of a group reads
        // another, so the loads of a whole group are in flight together and
        // its outputs are stored after them
#pragma unroll 1
        for (uint32_t gq = 0; gq < a.n_groups; ++gq) {
            const uint4 h = a.groups[2 * gq];
            if (h.x >> 24) {
                const uint4 f = a.ginfo[h.z];
                const uint64_t r = strip_gate(a, col, f.w);
                col[(uint64_t)f.x * kStripLanes] = r;
                strip_gate_tally(a, s_ones, f, r, valid, lane);
                continue;
            }
            const uint32_t cnt = h.x & 0xFFu, maxn = (h.x >> 8) & 0xFFFFu;
            const uint4 *rec = reinterpret_cast<const uint4 *>(a.gin + h.y);
            uint64_t acc[kStripGroup] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll 2
            for (uint32_t sl = 0; sl < maxn; ++sl) {
                const uint4 rr = rec[sl];
                acc[0] |= strip_in(col, rr.x);
                acc[1] |= strip_in(col, rr.y);
                acc[2] |= strip_in(col, rr.z);
                acc[3] |= strip_in(col, rr.w);
            }
            const uint4 out = a.groups[2 * gq + 1];
            uint32_t pc[kStripGroup];
#pragma unroll
            for (uint32_t j = 0; j < kStripGroup; ++j) {
                const uint64_t r = ((h.w >> j) & 1u) ? ~acc[j] : acc[j];
                pc[j] = valid && j < cnt ? (uint32_t)__popcll(r) : 0u;
                const uint32_t node = j == 0 ? out.x : j == 1 ? out.y : j == 2 ? out.z : out.w;
                if (j < cnt) col[(uint64_t)node * kStripLanes] = r;
            }
            // tallies: two gates' warp sums (at most 32 x 64 each) per 32-bit
            // reduction, then lane j adds gate j's sum to its tally slots
            const uint32_t s01 = __reduce_add_sync(0xFFFFFFFFu, pc[0] | (pc[1] << 16));
            const uint32_t s23 = __reduce_add_sync(0xFFFFFFFFu, pc[2] | (pc[3] << 16));
            if (lane < cnt) {
                const uint4 f = a.ginfo[h.z + lane];
                const uint32_t c = ((lane < 2 ? s01 : s23) >> (16 * (lane & 1u))) & 0xFFFFu;
                if (f.z && c)
                    for (uint32_t t = 0; t < f.z; ++t) strip_tally(a, s_ones, a.tally_list[f.y + t], c);
            }
        }
    }
    __syncthreads();
    if (a.tally_in_smem)
        for (uint32_t i = threadIdx.x; i < a.n_tally; i += blockDim.x)
            if (s_ones[i]) atomicAdd(&a.ones[i], s_ones[i]);
}

// Register-only sampler: thread w generates words (e, w) for n_events events
// (event e: pdag_idx + 1 = e + 3, event_idx + 1 = e + 1, table row e) and
// xors them together; one store per thread keeps the work alive.  Same
// sampler code as the product's sampling kernel.
template <int MF, int PF>
__global__ void __launch_bounds__(256) k_sampler_peak(uint32_t n_events, uint64_t n_words,
                                                      const uint2 *__restrict__ table, uint64_t *__restrict__ sink) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_words) return;
    const WordCtx ctx = make_word_ctx<MF>((uint32_t)w);
    uint64_t x = 0;
    for (uint32_t e = 0; e < n_events; ++e) {
        const uint32_t thr = 0x01000000u + (e * 0x9E3779B9u >> 8);  // spread of probabilities
        x ^= be_word_tab<MF, PF>(e + 1u, ctx, table + (uint64_t)e * kEventTableStride, thr);
    }
    sink[w] = x;
}

// Register-only sampler of the shared batch path: thread w generates words
// (e, w) of K instances per Philox evaluation (be_words, the sampler the
// batch interpreters call) and xors them together.
template <int MF, int PF, int K>
__global__ void __launch_bounds__(256) k_sampler_peak_shared(uint32_t n_events, uint64_t n_words,
                                                             uint64_t *__restrict__ sink) {
    const uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= n_words) return;
    const WordCtx ctx = make_word_ctx<MF>((uint32_t)w);
    uint64_t x = 0;
    for (uint32_t e = 0; e < n_events; ++e) {
        uint32_t thr[K];
        uint64_t out[K];
#pragma unroll
        for (int k = 0; k < K; ++k) thr[k] = 0x01000000u + ((e * 0x9E3779B9u + (uint32_t)k * 0x7F4A7C15u) >> 8);
        be_words<MF, PF, K>(e + 3u, e + 1u, ctx, 2u << 6, thr, out);
#pragma unroll
        for (int k = 0; k < K; ++k) x ^= out[k];
    }
    sink[w] = x;
}

// Event table for k_sampler_peak's synthetic events.
template <int MF>
__global__ void __launch_bounds__(256) k_peak_table(uint32_t n_events, uint32_t t3, uint2 *__restrict__ table) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (uint64_t)n_events * kEventTableStride) return;
    const uint32_t e = (uint32_t)(i / kEventTableStride);
    event_table_entry<MF>(e + 3u, t3, (int)(i % kEventTableStride), table[i]);
}

}  // namespace dev
}  // namespace mcg
