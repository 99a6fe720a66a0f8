// engine.cu -- the mcg_* engine entry points of include/mcg.h.
//
// One engine = one flattened PDAG on one device and stream.  It owns the
// device copies of the compiled fused program, the layered-mode tables, the
// tally counters and the fused kernel's scratch.  Replaces the device-memory
// ownership and pass submission of the reference's layer_manager
// (src/mc/queue/layer_manager.tpp:203-301) and its queueables
// (src/mc/queue/queueable.h:206-273, 725-731).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "engine_internal.hpp"
#include "error.hpp"
#include "graph.hpp"
#include "kernels.cuh"
#include "mcg.h"
#include "mcg_tune.h"
#include "program.hpp"
#include "smem_limit.hpp"

namespace {

// Sampler code form: separate high/low multiplies and the carry-chain bit
// packing measured fastest of the four forms on B200 (register-only sampler).
constexpr int kMulForm = 1;
constexpr int kPackForm = 1;
using mcg::internal::kDefaultChunkWords;
using mcg::internal::kFusedThreads;

#define MCG_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t err_ = (call);                                                              \
        if (err_ != cudaSuccess) {                                                              \
            return mcg::fail(err_ == cudaErrorMemoryAllocation ? MCG_ERR_OOM : MCG_ERR_CUDA,    \
                             std::string(#call) + ": " + cudaGetErrorString(err_));             \
        }                                                                                       \
    } while (0)

template <typename T>
cudaError_t upload(T **dptr, const std::vector<T> &v) {
    *dptr = nullptr;
    if (v.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc((void **)dptr, v.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// The engines' large work buffers (strip and fused scratch, staged chunk
// buffers: gigabytes for a large tree) are kept per device when an engine is
// destroyed (it has synchronised its streams by then), and the next engine
// takes the smallest kept buffer that fits instead of allocating.  What does
// not fit comes from cudaMalloc; at most kKeptBuffers buffers and
// kKeptBytes bytes are kept per device, and a failed allocation first
// frees the kept ones.  mcg_trim_memory frees them all.
constexpr size_t kKeptBuffers = 2;
constexpr size_t kKeptBytes = 32ull << 30;

struct KeptBuffer {
    void *ptr;
    size_t bytes;
};
std::mutex g_kept_mutex;
std::vector<std::vector<KeptBuffer>> g_kept;  // per device

std::vector<KeptBuffer> &kept_on(int device) {
    if (g_kept.size() <= (size_t)device) g_kept.resize((size_t)device + 1);
    return g_kept[device];
}

void free_kept(int device) {
    std::vector<KeptBuffer> drop;
    {
        std::lock_guard<std::mutex> lock(g_kept_mutex);
        drop.swap(kept_on(device));
    }
    for (const KeptBuffer &b : drop) cudaFree(b.ptr);
}

cudaError_t work_alloc(mcg_engine *e, void **ptr, size_t bytes) {
    *ptr = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_kept_mutex);
        std::vector<KeptBuffer> &kept = kept_on(e->device);
        size_t best = kept.size();
        for (size_t i = 0; i < kept.size(); ++i)
            if (kept[i].bytes >= bytes && (best == kept.size() || kept[i].bytes < kept[best].bytes)) best = i;
        if (best < kept.size()) {
            *ptr = kept[best].ptr;
            e->work_bytes[*ptr] = kept[best].bytes;
            kept.erase(kept.begin() + (std::ptrdiff_t)best);
            return cudaSuccess;
        }
    }
    cudaError_t err = cudaMalloc(ptr, bytes);
    if (err == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        free_kept(e->device);
        err = cudaMalloc(ptr, bytes);
    }
    if (err == cudaSuccess) e->work_bytes[*ptr] = bytes;
    return err;
}

void work_free(mcg_engine *e, void *ptr) {
    if (!ptr) return;
    const size_t bytes = e->work_bytes[ptr];
    std::vector<KeptBuffer> drop;
    {
        std::lock_guard<std::mutex> lock(g_kept_mutex);
        std::vector<KeptBuffer> &kept = kept_on(e->device);
        kept.push_back({ptr, bytes});
        size_t total = 0;
        for (const KeptBuffer &b : kept) total += b.bytes;
        while (!kept.empty() && (kept.size() > kKeptBuffers || total > kKeptBytes)) {
            auto smallest = std::min_element(kept.begin(), kept.end(),
                                             [](const KeptBuffer &a, const KeptBuffer &b) { return a.bytes < b.bytes; });
            total -= smallest->bytes;
            drop.push_back(*smallest);
            kept.erase(smallest);
        }
    }
    for (const KeptBuffer &b : drop) cudaFree(b.ptr);
}

}  // namespace

extern "C" mcg_status mcg_trim_memory(int device) {
    mcg::clear_error();
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || device < 0 || device >= n_dev) {
        cudaGetLastError();
        return mcg::fail(MCG_ERR_INVALID, "mcg_trim_memory: device ordinal out of range");
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    free_kept(device);
    cudaSetDevice(prev);
    return MCG_OK;
}

namespace {

// Strip mode's gate program: the gates of each layer in groups of up to
// kStripGroup that the kernel evaluates together (no gate of a group reads
// another, so all their input loads can be in flight at once).  AND, OR,
// NAND and NOR gates of at most kStripGroupMaxIn inputs and one-input NOT and
// NULL gates take the OR form r = outinv ^ OR_i (x_i ^ flip_i) (De Morgan:
// AND = ~OR(~x), NAND = OR(~x)); flip_i also carries the input's negation.
// Within a layer they are sorted by fan-in so a group's slots are mostly
// full.  Every other gate (XOR, ATLEAST, NOT/NULL of other fan-in, wider
// gates) is a group of one evaluated by strip_gate.  Each group is two
// uint4 records: its header and the output nodes of its gates.
mcg_status build_strip_groups(mcg_engine *e, const std::vector<uint32_t> &order,
                              const std::vector<uint2> &gate_tally) {
    using mcg::dev::kStripGroup;
    using mcg::dev::kStripGroupMaxIn;
    using mcg::dev::kStripNoInput;
    const mcg::Graph &g = e->graph;
    if ((uint64_t)g.n_nodes() >= 0x7FFFFFFFull) return mcg::fail(MCG_ERR_INVALID, "strip mode: too many nodes");
    std::vector<uint4> groups, ginfo;
    std::vector<uint32_t> gin;
    auto info = [&](uint32_t gi) { return make_uint4(g.n_be + gi, gate_tally[gi].x, gate_tally[gi].y, gi); };
    auto or_form = [&](uint32_t gi) {
        const uint8_t op = g.gate_op[gi];
        const uint32_t n = g.gate_in_count[gi];
        if (op == MCG_AND || op == MCG_OR || op == MCG_NAND || op == MCG_NOR) return n <= kStripGroupMaxIn;
        return (op == MCG_NOT || op == MCG_NULL) && n == 1;
    };
    std::vector<uint32_t> eligible;
    for (size_t l = 0; l + 1 < e->layer_offsets.size(); ++l) {
        eligible.clear();
        for (uint32_t q = e->layer_offsets[l]; q < e->layer_offsets[l + 1]; ++q) {
            const uint32_t gi = order[q];
            if (or_form(gi)) {
                eligible.push_back(gi);
            } else {
                groups.push_back(make_uint4(1u | (1u << 24), 0u, (uint32_t)ginfo.size(), 0u));
                groups.push_back(make_uint4(g.n_be + gi, 0u, 0u, 0u));
                ginfo.push_back(info(gi));
            }
        }
        std::stable_sort(eligible.begin(), eligible.end(),
                         [&](uint32_t x, uint32_t y) { return g.gate_in_count[x] < g.gate_in_count[y]; });
        for (size_t b = 0; b < eligible.size(); b += kStripGroup) {
            const uint32_t cnt = (uint32_t)std::min<size_t>(kStripGroup, eligible.size() - b);
            uint32_t maxn = 0, outinv = 0;
            for (uint32_t j = 0; j < cnt; ++j) {
                const uint32_t gi = eligible[b + j];
                const uint8_t op = g.gate_op[gi];
                maxn = std::max(maxn, g.gate_in_count[gi]);
                if (op == MCG_AND || op == MCG_NOR || op == MCG_NOT) outinv |= 1u << j;
            }
            groups.push_back(make_uint4(cnt | (maxn << 8), (uint32_t)gin.size(), (uint32_t)ginfo.size(), outinv));
            uint32_t outs[kStripGroup] = {0u, 0u, 0u, 0u};
            for (uint32_t j = 0; j < cnt; ++j) outs[j] = g.n_be + eligible[b + j];
            groups.push_back(make_uint4(outs[0], outs[1], outs[2], outs[3]));
            for (uint32_t s = 0; s < maxn; ++s) {
                for (uint32_t j = 0; j < kStripGroup; ++j) {
                    uint32_t rec = kStripNoInput;
                    if (j < cnt) {
                        const uint32_t gi = eligible[b + j];
                        const uint32_t n = g.gate_in_count[gi];
                        if (s < n) {
                            const bool negated = s >= n - g.gate_neg_count[gi];
                            const bool and_type = g.gate_op[gi] == MCG_AND || g.gate_op[gi] == MCG_NAND;
                            rec = (g.inputs[g.gate_in_begin[gi] + s] << 1) | (uint32_t)(negated != and_type);
                        }
                    }
                    gin.push_back(rec);
                }
            }
            for (uint32_t j = 0; j < cnt; ++j) ginfo.push_back(info(eligible[b + j]));
        }
    }
    e->n_strip_groups = (uint32_t)(groups.size() / 2);
    MCG_CUDA(upload(&e->d_strip_groups, groups));
    MCG_CUDA(upload(&e->d_strip_gin, gin));
    MCG_CUDA(upload(&e->d_strip_ginfo, ginfo));
    return MCG_OK;
}

mcg_status build_layered_tables(mcg_engine *e) {
    const mcg::Graph &g = e->graph;
    std::vector<uint4> be(g.n_be);
    for (uint32_t i = 0; i < g.n_be; ++i) {
        be[i] = make_uint4((uint32_t)g.be_pdag_idx[i] + 1u, g.be_event_idx[i] + 1u, (uint32_t)g.be_threshold[i],
                           (uint32_t)(g.be_threshold[i] >> 32));
    }
    std::vector<uint4> meta(g.n_gates);
    std::vector<uint32_t> layer(g.n_gates, 1);
    uint32_t n_layers = 0;
    for (uint32_t i = 0; i < g.n_gates; ++i) {
        meta[i] = make_uint4((uint32_t)g.gate_op[i] | ((g.gate_k[i] & 0xFFu) << 8), g.gate_in_begin[i],
                             g.gate_in_count[i], g.gate_neg_count[i]);
        uint32_t l = 1;
        for (uint32_t j = 0; j < g.gate_in_count[i]; ++j) {
            const uint32_t c = g.inputs[g.gate_in_begin[i] + j];
            if (c >= g.n_be) l = std::max(l, layer[c - g.n_be] + 1);
        }
        layer[i] = l;
        n_layers = std::max(n_layers, l);
    }
    // Gate ids grouped by layer (layer 1 .. n_layers), like the reference's
    // LayeredTopologicalOrder depth (src/preprocessor.cc:130-171).
    std::vector<uint32_t> counts(n_layers + 2, 0);
    for (uint32_t i = 0; i < g.n_gates; ++i) counts[layer[i]]++;
    e->layer_offsets.assign(n_layers + 1, 0);
    for (uint32_t l = 1; l <= n_layers; ++l) e->layer_offsets[l] = e->layer_offsets[l - 1] + counts[l];
    std::vector<uint32_t> cursor(e->layer_offsets.begin(), e->layer_offsets.end());
    std::vector<uint32_t> order(g.n_gates);
    for (uint32_t i = 0; i < g.n_gates; ++i) order[cursor[layer[i] - 1]++] = i;

    // staged-mode tables
    std::vector<uint4> smeta(g.n_gates);
    for (uint32_t i = 0; i < g.n_gates; ++i) {
        uint32_t nbits = 0;
        while (nbits < 8 && (g.gate_in_count[i] >> nbits) != 0) ++nbits;
        if (nbits == 0) nbits = 1;
        smeta[i] = make_uint4((uint32_t)g.gate_op[i] | ((g.gate_k[i] & 0xFFu) << 8) | (nbits << 16),
                              g.gate_in_begin[i], g.gate_in_count[i], g.gate_neg_count[i]);
    }
    std::vector<std::vector<uint32_t>> per_gate(g.n_gates);
    std::vector<uint32_t> be_nodes, be_idx;
    for (uint32_t t = 0; t < (uint32_t)g.tally_nodes.size(); ++t) {
        const uint32_t v = g.tally_nodes[t];
        if (v < g.n_be) {
            be_nodes.push_back(v);
            be_idx.push_back(t);
        } else {
            per_gate[v - g.n_be].push_back(t);
        }
    }
    std::vector<uint2> gate_tally(g.n_gates);
    std::vector<uint32_t> gate_tally_list;
    for (uint32_t i = 0; i < g.n_gates; ++i) {
        gate_tally[i] = make_uint2((uint32_t)gate_tally_list.size(), (uint32_t)per_gate[i].size());
        gate_tally_list.insert(gate_tally_list.end(), per_gate[i].begin(), per_gate[i].end());
    }
    e->n_be_tally = (uint32_t)be_nodes.size();
    if (e->mode == MCG_MODE_STRIP) {
        mcg_status st = build_strip_groups(e, order, gate_tally);
        if (st != MCG_OK) return st;
    }
    MCG_CUDA(upload(&e->d_smeta, smeta));
    MCG_CUDA(upload(&e->d_gate_tally, gate_tally));
    MCG_CUDA(upload(&e->d_gate_tally_list, gate_tally_list));
    MCG_CUDA(upload(&e->d_be_tally_nodes, be_nodes));
    MCG_CUDA(upload(&e->d_be_tally_idx, be_idx));

    MCG_CUDA(upload(&e->d_be, be));
    MCG_CUDA(upload(&e->d_meta, meta));
    MCG_CUDA(upload(&e->d_inputs, g.inputs));
    MCG_CUDA(upload(&e->d_tally_nodes, g.tally_nodes));
    MCG_CUDA(upload(&e->d_layer_gates, order));
    return MCG_OK;
}

dim3 rows_grid(uint64_t words, uint32_t rows, uint32_t threads) {
    const uint32_t bx = (uint32_t)((words + threads - 1) / threads);
    uint32_t by = rows, bz = 1;
    while (by > 65535u) {
        bz *= 2;
        by = (rows + bz - 1) / bz;
    }
    return dim3(bx, by, bz);
}

// Materialises every node's words for one pass over [word_begin, word_begin + W)
// into d_buf (reference dataflow).
mcg_status layered_eval(mcg_engine *e, uint32_t iteration, uint64_t word_begin, uint64_t W) {
    const mcg::Graph &g = e->graph;
    const uint64_t need = (uint64_t)g.n_nodes() * W;
    if (need > e->buf_words) {
        if (e->d_buf) cudaFree(e->d_buf);
        e->d_buf = nullptr;
        e->buf_words = 0;
        MCG_CUDA(cudaMalloc((void **)&e->d_buf, std::max<uint64_t>(need, 1) * sizeof(uint64_t)));
        e->buf_words = need;
    }
    const uint32_t t3 = (iteration + 1u) << 6;
    if (g.n_be > 0) {
        mcg::dev::k_layer_be<kMulForm, kPackForm><<<rows_grid(W, g.n_be, 256), 256, 0, e->stream>>>(
            e->d_be, g.n_be, W, word_begin, t3, e->d_buf);
        ++e->launches;
    }
    for (size_t l = 0; l + 1 < e->layer_offsets.size(); ++l) {
        const uint32_t n = e->layer_offsets[l + 1] - e->layer_offsets[l];
        if (n == 0) continue;
        mcg::dev::k_layer_gates<<<rows_grid(W, n, 256), 256, 0, e->stream>>>(
            e->d_meta, e->d_inputs, e->d_layer_gates + e->layer_offsets[l], n, g.n_be, W, e->d_buf);
        ++e->launches;
    }
    MCG_CUDA(cudaGetLastError());
    return MCG_OK;
}

using FusedKernel = void (*)(mcg::dev::FusedArgs);

// Register budget follows the CTAs wanted per SM (65536 / (256 * n) per thread).
FusedKernel fused_kernel(uint32_t ctas_per_sm) {
    switch (ctas_per_sm) {
        case 1: return mcg::dev::k_fused<kFusedThreads, 1, kMulForm, kPackForm>;
        case 3: return mcg::dev::k_fused<kFusedThreads, 3, kMulForm, kPackForm>;
        case 4: return mcg::dev::k_fused<kFusedThreads, 4, kMulForm, kPackForm>;
        default: return mcg::dev::k_fused<kFusedThreads, 2, kMulForm, kPackForm>;
    }
}

// Host-only compilation of the fused program (launch shape from the options).
mcg_status compile_fused(mcg_engine *e, const mcg_run_desc &run) {
    cudaDeviceProp prop;
    MCG_CUDA(cudaGetDeviceProperties(&prop, e->device));
    if (run.block_threads != 0 && run.block_threads != kFusedThreads)
        return mcg::fail(MCG_ERR_INVALID, "block_threads must be 0 or 256");
    e->nt = kFusedThreads;
    // 4 CTAs per SM measured fastest on the 200- and the 5,000-event trees
    const uint32_t ctas_per_sm = run.ctas_per_sm ? run.ctas_per_sm : 4u;
    if (ctas_per_sm < 1 || ctas_per_sm > 4) return mcg::fail(MCG_ERR_INVALID, "ctas_per_sm must be 1..4");
    e->ctas_per_sm = ctas_per_sm;
    const size_t smem_cap = std::min<size_t>(prop.sharedMemPerBlockOptin, prop.sharedMemPerMultiprocessor / ctas_per_sm) -
                            1024;  // per-CTA reserve
    const uint64_t n_tally = e->graph.tally_nodes.size();
    size_t tally_bytes = n_tally * sizeof(unsigned long long);
    e->tally_in_smem = tally_bytes <= smem_cap / 2;
    if (!e->tally_in_smem) tally_bytes = 0;
    const size_t slot_bytes = (size_t)e->nt * sizeof(uint64_t);
    uint32_t budget = (uint32_t)((smem_cap - tally_bytes) / slot_bytes);
    if (run.smem_slots == MCG_SMEM_SLOTS_NONE) budget = 0;
    else if (run.smem_slots) budget = std::min(budget, run.smem_slots);
    const std::string err = mcg::compile_program(e->graph, budget, e->prog);
    if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, err);
    e->smem_bytes = (uint32_t)(e->prog.smem_slots * slot_bytes + tally_bytes);
    e->grid = (uint32_t)prop.multiProcessorCount * ctas_per_sm;
    e->scratch_stride = (uint64_t)e->grid * e->nt;
    e->chunk_words = run.chunk_words ? run.chunk_words : kDefaultChunkWords;
    e->prog_compiled = true;
    return MCG_OK;
}

mcg_status setup_fused(mcg_engine *e, const mcg_run_desc &run) {
    mcg_status st = compile_fused(e, run);
    if (st != MCG_OK) return st;
    st = mcg::set_smem_limit(fused_kernel(e->ctas_per_sm), e->smem_bytes);
    if (st != MCG_OK) return st;
    MCG_CUDA(upload(reinterpret_cast<mcg::Op **>(&e->d_ops), e->prog.ops));
    if (e->prog.global_slots && e->mode == MCG_MODE_FUSED) {
        MCG_CUDA(work_alloc(e, (void **)&e->d_scratch,
                            (size_t)e->prog.global_slots * e->scratch_stride * sizeof(uint64_t)));
    }
    return MCG_OK;
}

constexpr uint32_t kStageEventsPerThread = 4;
constexpr uint32_t kStripBlocksPerSm = 6;
// Gate-phase blocks are small (128 threads, 2 words each) so that they fit in
// the registers and threads left next to the capped sampler blocks.
constexpr int kStageGateThreads = 128;
constexpr int kStageWordsPerThread = 2;

mcg_status setup_staged(mcg_engine *e, const mcg_run_desc &run) {
    const uint64_t nn = std::max<uint64_t>(e->graph.n_nodes(), 1);
    // two chunk buffers, together at most ~48 GB by default
    uint64_t words = run.layered_max_words ? run.layered_max_words : (24ull << 30) / (nn * sizeof(uint64_t));
    words = std::max<uint64_t>(256, std::min<uint64_t>(words, 1ull << 20));
    words = (words + 255) / 256 * 256;
    e->stage_words = words;
    for (int i = 0; i < 2; ++i) MCG_CUDA(work_alloc(e, (void **)&e->d_stage[i], nn * words * sizeof(uint64_t)));
    MCG_CUDA(cudaMalloc((void **)&e->d_event_table,
                        std::max<uint64_t>(e->graph.n_be, 1) * mcg::dev::kEventTableStride * sizeof(uint2)));
    // Cap the resident sampler blocks per SM through their shared-memory
    // footprint, so gate-phase blocks (memory bound) can run next to them.
    cudaDeviceProp prop;
    MCG_CUDA(cudaGetDeviceProperties(&prop, e->device));
    const uint32_t blocks = run.sampler_blocks_per_sm ? run.sampler_blocks_per_sm : 8u;
    if (blocks < 1 || blocks > 8) return mcg::fail(MCG_ERR_INVALID, "sampler_blocks_per_sm must be 1..8");
    e->sampler_smem = blocks >= 8 ? 0u : (uint32_t)(prop.sharedMemPerMultiprocessor / blocks - 2048);
    const mcg_status lim = mcg::set_smem_limit(mcg::dev::k_stage_be<kMulForm, kPackForm, kStageEventsPerThread>,
                                               e->sampler_smem);
    if (lim != MCG_OK) return lim;
    // The gate phase of chunk k runs while chunk k+1 is sampled: giving its
    // stream the higher priority lets its (memory-bound) blocks be scheduled
    // in between the sampler's blocks instead of after all of them.
    int prio_low = 0, prio_high = 0;
    MCG_CUDA(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
    MCG_CUDA(cudaStreamCreateWithPriority(&e->s_a, cudaStreamNonBlocking, prio_low));
    MCG_CUDA(cudaStreamCreateWithPriority(&e->s_b, cudaStreamNonBlocking, prio_high));
    for (cudaEvent_t *ev : {&e->ev_fork, &e->ev_a[0], &e->ev_a[1], &e->ev_b[0], &e->ev_b[1], &e->ev_join_a,
                            &e->ev_join_b})
        MCG_CUDA(cudaEventCreateWithFlags(ev, cudaEventDisableTiming));
    return MCG_OK;
}

// Strip kernel for a residency target: fewer blocks per SM give each thread
// more registers (6: 40, 5: 48, 4: 64).
using StripKernel = void (*)(mcg::dev::StripArgs);
StripKernel strip_kernel(uint32_t blocks_per_sm) {
    switch (blocks_per_sm) {
        case 4: return mcg::dev::k_strip<kMulForm, kPackForm, 4>;
        case 5: return mcg::dev::k_strip<kMulForm, kPackForm, 5>;
        default: return mcg::dev::k_strip<kMulForm, kPackForm, 6>;
    }
}

mcg_status setup_strip(mcg_engine *e, const mcg_run_desc &run) {
    const mcg::Graph &g = e->graph;
    cudaDeviceProp prop;
    MCG_CUDA(cudaGetDeviceProperties(&prop, e->device));
    const uint32_t target = run.ctas_per_sm ? run.ctas_per_sm : kStripBlocksPerSm;
    if (target < 4 || target > 6) return mcg::fail(MCG_ERR_INVALID, "strip mode: ctas_per_sm must be 0 or 4..6");
    e->strip_blocks = target;
    const uint64_t n_tally = g.tally_nodes.size();
    // tally counters in shared memory while the target residency still fits
    const uint64_t tally_bytes = n_tally * sizeof(unsigned long long);
    const uint64_t per_block = prop.sharedMemPerMultiprocessor / target - 2048;
    e->strip_smem = tally_bytes <= per_block ? (uint32_t)tally_bytes : 0u;
    const StripKernel kern = strip_kernel(target);
    const mcg_status lim = mcg::set_smem_limit(kern, e->strip_smem);
    if (lim != MCG_OK) return lim;
    int per_sm = 0;
    MCG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, mcg::dev::kStripThreads, e->strip_smem));
    if (per_sm < 1) return mcg::fail(MCG_ERR_INVALID, "strip kernel does not fit on an SM");
    e->strip_grid = (uint32_t)(prop.multiProcessorCount * per_sm);
    const uint64_t warps = (uint64_t)e->strip_grid * (mcg::dev::kStripThreads / 32);
    const uint64_t bytes = warps * std::max<uint64_t>(g.n_nodes(), 1) * mcg::dev::kStripLanes * sizeof(uint64_t);
    MCG_CUDA(work_alloc(e, (void **)&e->d_strip_scratch, bytes));
    MCG_CUDA(cudaMalloc((void **)&e->d_queue, sizeof(unsigned long long)));
    MCG_CUDA(cudaMalloc((void **)&e->d_event_table,
                        std::max<uint64_t>(g.n_be, 1) * mcg::dev::kEventTableStride * sizeof(uint2)));
    return MCG_OK;
}

// One persistent launch per pass on the engine stream.
mcg_status run_strip(mcg_engine *e, uint32_t it_first, uint32_t n_it, uint64_t word_begin, uint64_t count) {
    const mcg::Graph &g = e->graph;
    mcg::dev::StripArgs a{};
    a.be = e->d_be;
    a.table = e->d_event_table;
    a.n_be = g.n_be;
    a.n_nodes = g.n_nodes();
    a.smeta = e->d_smeta;
    a.inputs = e->d_inputs;
    a.groups = e->d_strip_groups;
    a.n_groups = e->n_strip_groups;
    a.gin = e->d_strip_gin;
    a.ginfo = e->d_strip_ginfo;
    a.tally_list = e->d_gate_tally_list;
    a.be_tally_nodes = e->d_be_tally_nodes;
    a.be_tally_idx = e->d_be_tally_idx;
    a.n_be_tally = e->n_be_tally;
    a.n_tally = (uint32_t)g.tally_nodes.size();
    a.tally_in_smem = e->strip_smem ? 1u : 0u;
    a.ones = e->d_tally;
    a.scratch = e->d_strip_scratch;
    a.word_begin = word_begin;
    a.word_count = count;
    a.queue = e->d_queue;
    for (uint32_t it = 0; it < n_it; ++it) {
        const uint32_t iteration = it_first + it;
        if (g.n_be > 0 && e->table_iteration != iteration) {
            const uint64_t n = (uint64_t)g.n_be * mcg::dev::kEventTableStride;
            mcg::dev::k_event_table<kMulForm><<<(uint32_t)((n + 255) / 256), 256, 0, e->stream>>>(
                e->d_be, g.n_be, (iteration + 1u) << 6, e->d_event_table);
            ++e->launches;
            e->table_iteration = iteration;
        }
        MCG_CUDA(cudaMemsetAsync(e->d_queue, 0, sizeof(unsigned long long), e->stream));
        cudaEvent_t p0 = nullptr, p1 = nullptr;
        if (e->profile_a) {
            if (e->prof_used == e->prof_events.size()) {
                cudaEvent_t x, y;
                MCG_CUDA(cudaEventCreate(&x));
                MCG_CUDA(cudaEventCreate(&y));
                e->prof_events.push_back({x, y});
            }
            p0 = e->prof_events[e->prof_used].first;
            p1 = e->prof_events[e->prof_used].second;
            ++e->prof_used;
            MCG_CUDA(cudaEventRecord(p0, e->stream));
        }
        strip_kernel(e->strip_blocks)<<<e->strip_grid, mcg::dev::kStripThreads, e->strip_smem, e->stream>>>(a);
        ++e->launches;
        if (p1) MCG_CUDA(cudaEventRecord(p1, e->stream));
        MCG_CUDA(cudaGetLastError());
    }
    return MCG_OK;
}

// One chunk: phase A (sampling) on s_a into buffer `set`, phase B (gate layers
// and tallies) on s_b once A is done.  A reuses a buffer only after the B that
// read it (two chunks earlier) has finished.
mcg_status staged_chunk(mcg_engine *e, uint64_t k, uint32_t iteration, uint64_t word_begin, uint64_t W) {
    const mcg::Graph &g = e->graph;
    const int set = (int)(k & 1);
    uint64_t *buf = e->d_stage[set];
    if (k >= 2) MCG_CUDA(cudaStreamWaitEvent(e->s_a, e->ev_b[set], 0));
    const uint32_t t3 = (iteration + 1u) << 6;
    const uint4 *be_tab = e->d_be_sample ? e->d_be_sample : e->d_be;
    if (g.n_be > 0 && e->table_iteration != iteration) {
        // s_a is in order: earlier sampler launches finish before the table changes
        const uint64_t n = (uint64_t)g.n_be * mcg::dev::kEventTableStride;
        mcg::dev::k_event_table<kMulForm><<<(uint32_t)((n + 255) / 256), 256, 0, e->s_a>>>(be_tab, g.n_be, t3,
                                                                                           e->d_event_table);
        ++e->launches;
        e->table_iteration = iteration;
    }
    if (g.n_be > 0) {
        const uint32_t groups = (g.n_be + kStageEventsPerThread - 1) / kStageEventsPerThread;
        cudaEvent_t p0 = nullptr, p1 = nullptr;
        if (e->profile_a) {
            if (e->prof_used == e->prof_events.size()) {
                cudaEvent_t a, b;
                MCG_CUDA(cudaEventCreate(&a));
                MCG_CUDA(cudaEventCreate(&b));
                e->prof_events.push_back({a, b});
            }
            p0 = e->prof_events[e->prof_used].first;
            p1 = e->prof_events[e->prof_used].second;
            ++e->prof_used;
            MCG_CUDA(cudaEventRecord(p0, e->s_a));
        }
        mcg::dev::k_stage_be<kMulForm, kPackForm, kStageEventsPerThread>
            <<<rows_grid(W, groups, 256), 256, e->sampler_smem, e->s_a>>>(be_tab, e->d_event_table, g.n_be, W,
                                                                          word_begin, buf);
        ++e->launches;
        if (p1) MCG_CUDA(cudaEventRecord(p1, e->s_a));
    }
    if (e->sample_hook) {
        const mcg_status st = e->sample_hook(e->s_a, buf, W, word_begin);
        if (st != MCG_OK) return st;
    }
    MCG_CUDA(cudaEventRecord(e->ev_a[set], e->s_a));
    MCG_CUDA(cudaStreamWaitEvent(e->s_b, e->ev_a[set], 0));
    const uint64_t words_per_block = (uint64_t)kStageGateThreads * kStageWordsPerThread;
    for (size_t l = 0; l + 1 < e->layer_offsets.size(); ++l) {
        const uint32_t n = e->layer_offsets[l + 1] - e->layer_offsets[l];
        if (n == 0) continue;
        dim3 grid = rows_grid(1, n, 256);
        grid.x = (uint32_t)((W + words_per_block - 1) / words_per_block);
        mcg::dev::k_stage_gates<kStageGateThreads, kStageWordsPerThread><<<grid, kStageGateThreads, 0, e->s_b>>>(
            e->d_smeta, e->d_inputs, e->d_layer_gates + e->layer_offsets[l], n, g.n_be, W, buf, e->d_gate_tally,
            e->d_gate_tally_list, e->d_tally);
        ++e->launches;
    }
    if (e->n_be_tally) {
        dim3 grid = rows_grid(1, e->n_be_tally, 256);
        grid.x = (uint32_t)std::min<uint64_t>((W + 255) / 256, 64);
        mcg::dev::k_layer_tally<<<grid, 256, 0, e->s_b>>>(e->d_be_tally_nodes, e->n_be_tally, W, buf, e->d_tally,
                                                          e->d_be_tally_idx);
        ++e->launches;
    }
    if (e->chunk_hook) {
        const mcg_status st = e->chunk_hook(e->s_b, buf, W);
        if (st != MCG_OK) return st;
    }
    MCG_CUDA(cudaEventRecord(e->ev_b[set], e->s_b));
    MCG_CUDA(cudaGetLastError());
    return MCG_OK;
}

mcg_status run_staged_impl(mcg_engine *e, uint32_t it_first, uint32_t n_it, uint64_t word_begin, uint64_t count) {
    // fork from the engine stream so the chunks follow earlier work on it
    MCG_CUDA(cudaEventRecord(e->ev_fork, e->stream));
    MCG_CUDA(cudaStreamWaitEvent(e->s_a, e->ev_fork, 0));
    MCG_CUDA(cudaStreamWaitEvent(e->s_b, e->ev_fork, 0));
    uint64_t k = 0;
    for (uint32_t it = 0; it < n_it; ++it) {
        for (uint64_t off = 0; off < count; off += e->stage_words, ++k) {
            const uint64_t n = std::min<uint64_t>(e->stage_words, count - off);
            const mcg_status st = staged_chunk(e, k, it_first + it, word_begin + off, n);
            if (st != MCG_OK) return st;
        }
    }
    // join back into the engine stream
    MCG_CUDA(cudaEventRecord(e->ev_join_a, e->s_a));
    MCG_CUDA(cudaEventRecord(e->ev_join_b, e->s_b));
    MCG_CUDA(cudaStreamWaitEvent(e->stream, e->ev_join_a, 0));
    MCG_CUDA(cudaStreamWaitEvent(e->stream, e->ev_join_b, 0));
    return MCG_OK;
}

mcg_status launch_fused(mcg_engine *e, uint32_t it_first, uint32_t n_it, uint64_t word_begin, uint64_t count) {
    mcg::dev::FusedArgs a;
    a.ops = e->d_ops;
    a.smem_slots = e->prog.smem_slots;
    a.scratch = e->d_scratch;
    a.scratch_stride = e->scratch_stride;
    a.tally = e->d_tally;
    a.n_tally = (uint32_t)e->graph.tally_nodes.size();
    a.tally_in_smem = e->tally_in_smem ? 1u : 0u;
    a.iteration_first = it_first;
    a.n_iterations = n_it;
    a.word_begin = word_begin;
    a.word_count = count;
    const uint64_t want = (count + e->nt - 1) / e->nt;
    const uint32_t grid = (uint32_t)std::min<uint64_t>(e->grid, std::max<uint64_t>(want, 1));
    fused_kernel(e->ctas_per_sm)<<<grid, e->nt, e->smem_bytes, e->stream>>>(a);
    ++e->launches;
    MCG_CUDA(cudaGetLastError());
    return MCG_OK;
}

void release(mcg_engine *e) {
    // the side streams' work ends before their buffers go back to the pool
    if (e->s_a) cudaStreamSynchronize(e->s_a);
    if (e->s_b) cudaStreamSynchronize(e->s_b);
    if (e->stream) cudaStreamSynchronize(e->stream);
    work_free(e, e->d_scratch);
    work_free(e, e->d_stage[0]);
    work_free(e, e->d_stage[1]);
    work_free(e, e->d_strip_scratch);
    cudaFree(e->d_ops);
    cudaFree(e->d_tally);
    cudaFree(e->d_be);
    cudaFree(e->d_meta);
    cudaFree(e->d_inputs);
    cudaFree(e->d_tally_nodes);
    cudaFree(e->d_layer_gates);
    cudaFree(e->d_buf);
    cudaFree(e->d_smeta);
    cudaFree(e->d_gate_tally);
    cudaFree(e->d_gate_tally_list);
    cudaFree(e->d_be_tally_nodes);
    cudaFree(e->d_be_tally_idx);
    cudaFree(e->d_event_table);
    cudaFree(e->d_queue);
    cudaFree(e->d_strip_groups);
    cudaFree(e->d_strip_gin);
    cudaFree(e->d_strip_ginfo);
    for (int i = 0; i < 2; ++i) {
        if (e->ev_snap[i]) cudaEventDestroy(e->ev_snap[i]);
    }
    for (cudaEvent_t ev : {e->ev_fork, e->ev_a[0], e->ev_a[1], e->ev_b[0], e->ev_b[1], e->ev_join_a, e->ev_join_b})
        if (ev) cudaEventDestroy(ev);
    for (auto &pe : e->prof_events) {
        cudaEventDestroy(pe.first);
        cudaEventDestroy(pe.second);
    }
    if (e->s_a) cudaStreamDestroy(e->s_a);
    if (e->s_b) cudaStreamDestroy(e->s_b);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
}

}  // namespace

namespace mcg {
namespace internal {
mcg_status run_staged(mcg_engine *e, uint32_t it_first, uint32_t n_it, uint64_t word_begin, uint64_t count) {
    return run_staged_impl(e, it_first, n_it, word_begin, count);
}
}  // namespace internal
}  // namespace mcg

extern "C" {

mcg_status mcg_create(const mcg_graph_desc *graph, const mcg_run_desc *run_in, mcg_engine **out) {
    mcg::clear_error();
    if (!graph || !out) return mcg::fail(MCG_ERR_INVALID, "graph and out must not be NULL");
    *out = nullptr;
    mcg_run_desc run{};
    if (run_in) run = *run_in;
    if (run.mode > MCG_MODE_FUSED) return mcg::fail(MCG_ERR_INVALID, "unknown mode");
    auto *e = new (std::nothrow) mcg_engine();
    if (!e) return mcg::fail(MCG_ERR_OOM, "host allocation failed");
    const std::string err = mcg::Graph::from_desc(*graph, e->graph);
    if (!err.empty()) {
        delete e;
        return mcg::fail(MCG_ERR_INVALID, err);
    }
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
        cudaGetLastError();
        delete e;
        return mcg::fail(MCG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    if (run.device < 0 || run.device >= n_dev) {
        delete e;
        return mcg::fail(MCG_ERR_INVALID, "device ordinal out of range");
    }
    if (run.mode == MCG_MODE_AUTO) {
        // the launch shape tuned (or cached) for this tree shape on this device
        mcg_tune_choice ch{};
        const mcg_status ts = mcg_tune(graph, &run, run.tune_pass_words, nullptr, nullptr, &ch);
        if (ts != MCG_OK) {
            delete e;
            return ts;
        }
        run.mode = ch.mode;
        run.ctas_per_sm = ch.ctas_per_sm;
        run.layered_max_words = ch.layered_max_words;
        run.smem_slots = 0;
        run.chunk_words = 0;
        run.sampler_blocks_per_sm = 0;
        mcg::clear_error();
    }
    e->device = run.device;
    e->mode = run.mode;
    e->run_desc = run;
    e->layered_max_words = run.layered_max_words;
    mcg_status st = MCG_OK;
    do {
        if (cudaSetDevice(e->device) != cudaSuccess) {
            st = mcg::fail(MCG_ERR_CUDA, "cudaSetDevice failed");
            break;
        }
        if (run.stream) {
            e->stream = (cudaStream_t)run.stream;
        } else {
            if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
                st = mcg::fail(MCG_ERR_CUDA, "cudaStreamCreate failed");
                break;
            }
            e->own_stream = true;
        }
        const size_t nt = std::max<size_t>(e->graph.tally_nodes.size(), 1);
        // the counters and, behind them, two snapshot slots (mcg_snapshot_tallies)
        if (cudaMalloc((void **)&e->d_tally, 3 * nt * sizeof(unsigned long long)) != cudaSuccess ||
            cudaMemset(e->d_tally, 0, nt * sizeof(unsigned long long)) != cudaSuccess) {
            st = mcg::fail(MCG_ERR_OOM, "tally allocation failed");
            break;
        }
        st = build_layered_tables(e);
        if (st != MCG_OK) break;
        // the fused program is compiled here only for the fused mode (on request otherwise)
        if (e->mode == MCG_MODE_FUSED) st = setup_fused(e, run);
        else if (e->mode == MCG_MODE_STAGED) st = setup_staged(e, run);
        else if (e->mode == MCG_MODE_STRIP) st = setup_strip(e, run);
    } while (false);
    if (st != MCG_OK) {
        release(e);
        delete e;
        return st;
    }
    *out = e;
    return MCG_OK;
}

mcg_status mcg_engine_launch_shape(mcg_engine *e, uint32_t *mode, uint32_t *ctas_per_sm) {
    mcg::clear_error();
    if (!e) return mcg::fail(MCG_ERR_INVALID, "engine is NULL");
    if (mode) *mode = e->mode;
    if (ctas_per_sm)
        *ctas_per_sm = e->mode == MCG_MODE_STRIP ? e->strip_blocks : e->mode == MCG_MODE_FUSED ? e->ctas_per_sm : 0u;
    return MCG_OK;
}

mcg_status mcg_destroy(mcg_engine *e) {
    mcg::clear_error();
    if (!e) return MCG_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    release(e);
    delete e;
    return MCG_OK;
}

mcg_status mcg_run(mcg_engine *e, uint32_t iteration_first, uint32_t n_iterations, uint64_t word_begin,
                   uint64_t word_count) {
    mcg::clear_error();
    if (!e) return mcg::fail(MCG_ERR_INVALID, "engine is NULL");
    if (word_begin + word_count > (1ull << 32) || word_begin + word_count < word_begin)
        return mcg::fail(MCG_ERR_INVALID, "word range exceeds the 32-bit sample counter");
    if ((uint64_t)iteration_first + n_iterations + 1 >= (1ull << 26))
        return mcg::fail(MCG_ERR_INVALID, "iteration exceeds the 26-bit pass counter field");
    if (n_iterations == 0 || word_count == 0) return MCG_OK;
    MCG_CUDA(cudaSetDevice(e->device));
    if (e->mode == MCG_MODE_STAGED) {
        const mcg_status st = run_staged_impl(e, iteration_first, n_iterations, word_begin, word_count);
        if (st != MCG_OK) return st;
    } else if (e->mode == MCG_MODE_STRIP) {
        const mcg_status st = run_strip(e, iteration_first, n_iterations, word_begin, word_count);
        if (st != MCG_OK) return st;
    } else if (e->mode == MCG_MODE_FUSED) {
        for (uint64_t off = 0; off < word_count; off += e->chunk_words) {
            const uint64_t n = std::min<uint64_t>(e->chunk_words, word_count - off);
            const mcg_status st = launch_fused(e, iteration_first, n_iterations, word_begin + off, n);
            if (st != MCG_OK) return st;
        }
    } else {
        const uint64_t nn = std::max<uint64_t>(e->graph.n_nodes(), 1);
        uint64_t W = e->layered_max_words ? e->layered_max_words : std::max<uint64_t>((8ull << 30) / (nn * 8), 1024);
        W = std::min<uint64_t>(W, word_count);
        const uint32_t n_tally = (uint32_t)e->graph.tally_nodes.size();
        for (uint32_t it = 0; it < n_iterations; ++it) {
            for (uint64_t off = 0; off < word_count; off += W) {
                const uint64_t n = std::min<uint64_t>(W, word_count - off);
                mcg_status st = layered_eval(e, iteration_first + it, word_begin + off, n);
                if (st != MCG_OK) return st;
                if (n_tally) {
                    const uint32_t bx = (uint32_t)std::min<uint64_t>((n + 255) / 256, 64);
                    dim3 grid = rows_grid(1, n_tally, 256);
                    grid.x = bx;
                    mcg::dev::k_layer_tally<<<grid, 256, 0, e->stream>>>(e->d_tally_nodes, n_tally, n, e->d_buf,
                                                                         e->d_tally, nullptr);
                    ++e->launches;
                    MCG_CUDA(cudaGetLastError());
                }
            }
        }
    }
    e->total_bits += (uint64_t)n_iterations * word_count * 64ull;
    return MCG_OK;
}

mcg_status mcg_synchronize(mcg_engine *e) {
    mcg::clear_error();
    if (!e) return mcg::fail(MCG_ERR_INVALID, "engine is NULL");
    MCG_CUDA(cudaSetDevice(e->device));
    MCG_CUDA(cudaStreamSynchronize(e->stream));
    return MCG_OK;
}

mcg_status mcg_read_tallies(mcg_engine *e, uint64_t *ones, uint64_t *total_bits) {
    mcg::clear_error();
    if (!e) return mcg::fail(MCG_ERR_INVALID, "engine is NULL");
    MCG_CUDA(cudaSetDevice(e->device));
    MCG_CUDA(cudaStreamSynchronize(e->stream));
    if (ones && !e->graph.tally_nodes.empty()) {
        MCG_CUDA(cudaMemcpy(ones, e->d_tally, e->graph.tally_nodes.size() * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    }
    if (total_bits) *total_bits = e->total_bits;
    return MCG_OK;
}

mcg_status mcg_tally_device_ptr(mcg_engine *e, uint64_t **ones_dev) {
    mcg::clear_error();
    if (!e || !ones_dev) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    *ones_dev = reinterpret_cast<uint64_t *>(e->d_tally);
    return MCG_OK;
}

mcg_status mcg_set_tallies(mcg_engine *e, const uint64_t *ones, uint64_t total_bits) {
    mcg::clear_error();
    if (!e || !ones) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    MCG_CUDA(cudaSetDevice(e->device));
    MCG_CUDA(cudaStreamSynchronize(e->stream));
    if (!e->graph.tally_nodes.empty())
        MCG_CUDA(cudaMemcpy(e->d_tally, ones, e->graph.tally_nodes.size() * sizeof(uint64_t), cudaMemcpyHostToDevice));
    e->total_bits = total_bits;
    return MCG_OK;
}

mcg_status mcg_snapshot_tallies(mcg_engine *e, uint32_t slot) {
    mcg::clear_error();
    if (!e) return mcg::fail(MCG_ERR_INVALID, "engine is NULL");
    if (slot > 1) return mcg::fail(MCG_ERR_INVALID, "slot must be 0 or 1");
    MCG_CUDA(cudaSetDevice(e->device));
    const size_t n = std::max<size_t>(e->graph.tally_nodes.size(), 1);
    if (!e->ev_snap[slot]) MCG_CUDA(cudaEventCreateWithFlags(&e->ev_snap[slot], cudaEventDisableTiming));
    // device-side copy into the slot behind the counters: no host buffer to pin
    MCG_CUDA(cudaMemcpyAsync(e->d_tally + (1 + slot) * n, e->d_tally, n * sizeof(uint64_t), cudaMemcpyDeviceToDevice,
                             e->stream));
    MCG_CUDA(cudaEventRecord(e->ev_snap[slot], e->stream));
    e->snap_total[slot] = e->total_bits;
    return MCG_OK;
}

mcg_status mcg_snapshot_read(mcg_engine *e, uint32_t slot, uint64_t *ones, uint64_t *total_bits) {
    mcg::clear_error();
    if (!e || !ones || !total_bits) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (slot > 1 || !e->ev_snap[slot]) return mcg::fail(MCG_ERR_STATE, "no snapshot in this slot");
    MCG_CUDA(cudaSetDevice(e->device));
    MCG_CUDA(cudaEventSynchronize(e->ev_snap[slot]));
    // the slot is not written by the passes behind the snapshot: this copy does not wait for them
    const size_t n = std::max<size_t>(e->graph.tally_nodes.size(), 1);
    if (!e->graph.tally_nodes.empty())
        MCG_CUDA(cudaMemcpy(ones, e->d_tally + (1 + slot) * n, e->graph.tally_nodes.size() * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost));
    *total_bits = e->snap_total[slot];
    return MCG_OK;
}

mcg_status mcg_reset_tallies(mcg_engine *e) {
    mcg::clear_error();
    if (!e) return mcg::fail(MCG_ERR_INVALID, "engine is NULL");
    MCG_CUDA(cudaSetDevice(e->device));
    MCG_CUDA(cudaMemsetAsync(e->d_tally, 0, std::max<size_t>(e->graph.tally_nodes.size(), 1) * sizeof(uint64_t),
                             e->stream));
    e->total_bits = 0;
    return MCG_OK;
}

mcg_status mcg_dump_words(mcg_engine *e, uint32_t iteration, uint64_t word_begin, uint64_t n_words, uint64_t *out) {
    mcg::clear_error();
    if (!e || !out) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (word_begin + n_words > (1ull << 32)) return mcg::fail(MCG_ERR_INVALID, "word range exceeds the sample counter");
    if (n_words == 0) return MCG_OK;
    MCG_CUDA(cudaSetDevice(e->device));
    mcg_status st = layered_eval(e, iteration, word_begin, n_words);
    if (st != MCG_OK) return st;
    MCG_CUDA(cudaStreamSynchronize(e->stream));
    MCG_CUDA(cudaMemcpy(out, e->d_buf, (size_t)e->graph.n_nodes() * n_words * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    return MCG_OK;
}

mcg_status mcg_program_info_get(mcg_engine *e, mcg_program_info *info) {
    mcg::clear_error();
    if (!e || !info) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (!e->prog_compiled) {
        MCG_CUDA(cudaSetDevice(e->device));
        mcg_run_desc rd = e->run_desc;
        rd.ctas_per_sm = 0;  // the other modes' value means something else
        const mcg_status st = compile_fused(e, rd);
        if (st != MCG_OK) return st;
    }
    info->n_ops = e->prog.ops.size();
    info->smem_slots = e->prog.smem_slots;
    info->global_slots = e->prog.global_slots;
    info->max_live = e->prog.max_live;
    info->block_threads = e->nt;
    info->grid_ctas = e->grid;
    info->scratch_bytes = (uint64_t)e->prog.global_slots * e->scratch_stride * sizeof(uint64_t);
    info->smem_bytes = e->smem_bytes;
    info->n_inline_be = e->prog.n_inline_be;
    return MCG_OK;
}

mcg_status mcg_launch_count(mcg_engine *e, uint64_t *launches) {
    mcg::clear_error();
    if (!e || !launches) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    *launches = e->launches;
    return MCG_OK;
}

mcg_status mcg_time_runs(mcg_engine *e, uint32_t iteration_first, uint64_t word_begin, uint64_t word_count,
                         uint32_t repeats, double *ms_per_run) {
    mcg::clear_error();
    if (!e || !ms_per_run || repeats == 0) return mcg::fail(MCG_ERR_INVALID, "bad argument");
    MCG_CUDA(cudaSetDevice(e->device));
    cudaEvent_t a, b;
    MCG_CUDA(cudaEventCreate(&a));
    MCG_CUDA(cudaEventCreate(&b));
    MCG_CUDA(cudaEventRecord(a, e->stream));
    for (uint32_t r = 0; r < repeats; ++r) {
        const mcg_status st = mcg_run(e, iteration_first + r, 1, word_begin, word_count);
        if (st != MCG_OK) {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            return st;
        }
    }
    MCG_CUDA(cudaEventRecord(b, e->stream));
    MCG_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    MCG_CUDA(cudaEventElapsedTime(&ms, a, b));
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    *ms_per_run = (double)ms / repeats;
    return MCG_OK;
}

mcg_status mcg_sampler_peak(int32_t device, uint64_t n_events, uint64_t n_words, uint32_t repeats,
                            double *words_per_second) {
    mcg::clear_error();
    if (!words_per_second || n_events == 0 || n_words == 0 || repeats == 0 || n_events > 0xFFFFFFFFull ||
        n_words > 0xFFFFFFFFull)
        return mcg::fail(MCG_ERR_INVALID, "bad argument");
    MCG_CUDA(cudaSetDevice(device));
    uint64_t *sink = nullptr;
    uint2 *table = nullptr;
    MCG_CUDA(cudaMalloc((void **)&sink, n_words * sizeof(uint64_t)));
    if (cudaMalloc((void **)&table, n_events * mcg::dev::kEventTableStride * sizeof(uint2)) != cudaSuccess) {
        cudaFree(sink);
        return mcg::fail(MCG_ERR_OOM, "sampler table allocation failed");
    }
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const uint64_t nt = n_events * mcg::dev::kEventTableStride;
    mcg::dev::k_peak_table<kMulForm><<<(uint32_t)((nt + 255) / 256), 256>>>((uint32_t)n_events, 2u << 6, table);
    const uint32_t blocks = (uint32_t)((n_words + 255) / 256);
    // warm-up
    mcg::dev::k_sampler_peak<kMulForm, kPackForm><<<blocks, 256>>>((uint32_t)n_events, n_words, table, sink);
    cudaEventRecord(a);
    for (uint32_t r = 0; r < repeats; ++r)
        mcg::dev::k_sampler_peak<kMulForm, kPackForm><<<blocks, 256>>>((uint32_t)n_events, n_words, table, sink);
    cudaEventRecord(b);
    cudaError_t err = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(table);
    cudaFree(sink);
    if (err != cudaSuccess) return mcg::fail(MCG_ERR_CUDA, cudaGetErrorString(err));
    *words_per_second = (double)n_events * (double)n_words * repeats / (ms * 1e-3);
    return MCG_OK;
}

mcg_status mcg_sampler_peak_shared(int32_t device, uint64_t n_events, uint64_t n_words, uint32_t repeats,
                                   uint32_t instances, double *instance_words_per_second) {
    mcg::clear_error();
    if (!instance_words_per_second || n_events == 0 || n_words == 0 || repeats == 0 || n_events > 0xFFFFFFFFull ||
        n_words > 0xFFFFFFFFull || (instances != 1 && instances != 4))
        return mcg::fail(MCG_ERR_INVALID, "bad argument");
    MCG_CUDA(cudaSetDevice(device));
    uint64_t *sink = nullptr;
    MCG_CUDA(cudaMalloc((void **)&sink, n_words * sizeof(uint64_t)));
    auto launch = [&] {
        const uint32_t blocks = (uint32_t)((n_words + 255) / 256);
        if (instances == 4)
            mcg::dev::k_sampler_peak_shared<kMulForm, kPackForm, 4><<<blocks, 256>>>((uint32_t)n_events, n_words, sink);
        else
            mcg::dev::k_sampler_peak_shared<kMulForm, kPackForm, 1><<<blocks, 256>>>((uint32_t)n_events, n_words, sink);
    };
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    launch();  // warm-up
    cudaEventRecord(a);
    for (uint32_t r = 0; r < repeats; ++r) launch();
    cudaEventRecord(b);
    cudaError_t err = cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    if (err != cudaSuccess) return mcg::fail(MCG_ERR_CUDA, cudaGetErrorString(err));
    *instance_words_per_second = (double)n_events * (double)n_words * instances * repeats / (ms * 1e-3);
    return MCG_OK;
}

mcg_status mcg_profile_sampler(mcg_engine *e, int32_t enable) {
    mcg::clear_error();
    if (!e) return mcg::fail(MCG_ERR_INVALID, "engine is NULL");
    e->profile_a = enable != 0;
    e->prof_used = 0;
    return MCG_OK;
}

mcg_status mcg_profile_sampler_read(mcg_engine *e, uint64_t *launches, double *total_ms) {
    mcg::clear_error();
    if (!e || !launches || !total_ms) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    MCG_CUDA(cudaSetDevice(e->device));
    MCG_CUDA(cudaStreamSynchronize(e->stream));
    double sum = 0;
    for (size_t i = 0; i < e->prof_used; ++i) {
        float ms = 0;
        MCG_CUDA(cudaEventElapsedTime(&ms, e->prof_events[i].first, e->prof_events[i].second));
        sum += ms;
    }
    *launches = e->prof_used;
    *total_ms = sum;
    return MCG_OK;
}

const char *mcg_version(void) { return "mcg 0.1 (sm_100a)"; }

}  // extern "C"
