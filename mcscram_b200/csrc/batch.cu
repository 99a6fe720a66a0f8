// batch.cu -- batched instances in one persistent, graph-captured launch
// (include/mcg_batch.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "error.hpp"
#include "graph.hpp"
#include "kernels.cuh"
#include "mcg_batch.h"
#include "program.hpp"
#include "smem_limit.hpp"

namespace {

constexpr int kThreads = 256;
constexpr int kMulForm = 1;
constexpr int kPackForm = 1;
// Instances of one tree that differ only in thresholds (uncertainty draws)
// share their Philox calls kShare at a time (k_fused_batch_k) unless a tree
// has an ATLEAST gate of more than kShareAtleastMaxIn inputs (the four-wide
// interpreter counts ATLEAST inputs in four bit slices per instance).
constexpr uint32_t kShare = 4;
constexpr uint32_t kShareAtleastMaxIn = 15;

#define MCG_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t err_ = (call);                                                              \
        if (err_ != cudaSuccess) {                                                              \
            return mcg::fail(err_ == cudaErrorMemoryAllocation ? MCG_ERR_OOM : MCG_ERR_CUDA,    \
                             std::string(#call) + ": " + cudaGetErrorString(err_));             \
        }                                                                                       \
    } while (0)

using BatchKernel = void (*)(mcg::dev::BatchArgs);

BatchKernel batch_kernel(uint32_t ctas_per_sm, uint32_t share, bool atleast) {
    if (share == kShare && atleast) {
        switch (ctas_per_sm) {
            case 2: return mcg::dev::k_fused_batch_k<kThreads, 2, kMulForm, kPackForm, kShare, true>;
            case 3: return mcg::dev::k_fused_batch_k<kThreads, 3, kMulForm, kPackForm, kShare, true>;
            default: return mcg::dev::k_fused_batch_k<kThreads, 4, kMulForm, kPackForm, kShare, true>;
        }
    }
    if (share == kShare) {
        switch (ctas_per_sm) {
            case 2: return mcg::dev::k_fused_batch_k<kThreads, 2, kMulForm, kPackForm, kShare, false>;
            case 3: return mcg::dev::k_fused_batch_k<kThreads, 3, kMulForm, kPackForm, kShare, false>;
            default: return mcg::dev::k_fused_batch_k<kThreads, 4, kMulForm, kPackForm, kShare, false>;
        }
    }
    switch (ctas_per_sm) {
        case 2: return mcg::dev::k_fused_batch<kThreads, 2, kMulForm, kPackForm>;
        case 3: return mcg::dev::k_fused_batch<kThreads, 3, kMulForm, kPackForm>;
        default: return mcg::dev::k_fused_batch<kThreads, 4, kMulForm, kPackForm>;
    }
}

template <typename T>
cudaError_t ensure(T **p, uint64_t &cap, uint64_t n) {
    if (n <= cap && *p) return cudaSuccess;
    if (*p) cudaFree(*p);
    *p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void **)p, std::max<uint64_t>(n, 1) * sizeof(T));
    if (e == cudaSuccess) cap = std::max<uint64_t>(n, 1);
    return e;
}

}  // namespace

struct mcg_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    uint32_t ctas_per_sm = 4;
    uint32_t share = 1;  // instances per work item (kShare or 1)
    bool atleast = false; // the shared kernel needs its ATLEAST counters
    std::vector<mcg::Graph> trees;
    std::vector<uint32_t> tree_op_offset;
    uint32_t smem_slots = 0, max_global = 0, grid = 0, smem_bytes = 0;
    uint64_t total_ops = 0;
    uint4 *d_ops = nullptr;
    uint32_t *d_tree_off = nullptr;
    uint64_t *d_scratch = nullptr;
    uint64_t scratch_stride = 0;
    unsigned int *d_queue = nullptr;
    // per-run buffers
    uint32_t *d_inst_tree = nullptr;
    uint64_t cap_inst = 0, cap_inst2 = 0, cap_thr = 0, cap_ones = 0;
    uint64_t *d_thr_off = nullptr;
    uint64_t *d_thr = nullptr;
    unsigned long long *d_ones = nullptr;
    uint32_t *d_group_first = nullptr, *d_group_size = nullptr;
    uint64_t cap_grp = 0, cap_grp2 = 0;
    uint32_t n_groups = 0;
    // graph
    cudaGraphExec_t graph = nullptr;
    uint32_t g_instances = 0, g_iteration = 0;
    uint64_t g_words = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    uint64_t launches = 0;
    double last_ms = 0.0;
};

namespace {

void release(mcg_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    cudaFree(b->d_ops);
    cudaFree(b->d_tree_off);
    cudaFree(b->d_scratch);
    cudaFree(b->d_queue);
    cudaFree(b->d_inst_tree);
    cudaFree(b->d_thr_off);
    cudaFree(b->d_thr);
    cudaFree(b->d_ones);
    cudaFree(b->d_group_first);
    cudaFree(b->d_group_size);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
}

mcg_status setup(mcg_batch *b, const mcg_run_desc &run) {
    MCG_CUDA(cudaSetDevice(b->device));
    cudaDeviceProp prop;
    MCG_CUDA(cudaGetDeviceProperties(&prop, b->device));
    b->ctas_per_sm = run.ctas_per_sm ? run.ctas_per_sm : 4u;
    if (b->ctas_per_sm < 2 || b->ctas_per_sm > 4) return mcg::fail(MCG_ERR_INVALID, "ctas_per_sm must be 2..4");
    b->share = kShare;
    for (const auto &g : b->trees)
        for (size_t i = 0; i < g.gate_op.size(); ++i)
            if (g.gate_op[i] == MCG_ATLEAST) {
                if (g.gate_in_count[i] <= kShareAtleastMaxIn) b->atleast = true;
                else b->share = 1;
            }
    // What one of ctas_per_sm resident CTAs may take: the SM's shared memory
    // shared out, less the per-block reservation and the kernel's static
    // shared memory (its work-item slot), so that all of them stay resident.
    cudaFuncAttributes fa{};
    MCG_CUDA(cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(batch_kernel(b->ctas_per_sm, b->share,
                                                                                     b->atleast))));
    const size_t cap = std::min<size_t>(prop.sharedMemPerBlockOptin,
                                        prop.sharedMemPerMultiprocessor / b->ctas_per_sm -
                                            prop.reservedSharedMemPerBlock) -
                       fa.sharedSizeBytes;
    // a slot holds one word per instance of a work item
    uint32_t budget = (uint32_t)(cap / (kThreads * sizeof(uint64_t) * b->share));
    if (run.smem_slots == MCG_SMEM_SLOTS_NONE) budget = 0;
    else if (run.smem_slots) budget = std::min(budget, run.smem_slots);
    std::vector<mcg::Op> all;
    for (const auto &g : b->trees) {
        mcg::Program prog;
        const std::string err = mcg::compile_program(g, budget, prog, true);
        if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, err);
        b->tree_op_offset.push_back((uint32_t)all.size());
        all.insert(all.end(), prog.ops.begin(), prog.ops.end());
        b->smem_slots = std::max(b->smem_slots, prog.smem_slots);
        b->max_global = std::max(b->max_global, prog.global_slots);
    }
    if (all.size() >= 0xFFFFFFFFull) return mcg::fail(MCG_ERR_INVALID, "programs too large");
    b->total_ops = all.size();
    b->smem_bytes = b->smem_slots * b->share * kThreads * (uint32_t)sizeof(uint64_t);
    b->grid = (uint32_t)prop.multiProcessorCount * b->ctas_per_sm;
    b->scratch_stride = (uint64_t)b->grid * kThreads;
    MCG_CUDA(cudaMalloc((void **)&b->d_ops, all.size() * sizeof(mcg::Op)));
    MCG_CUDA(cudaMemcpy(b->d_ops, all.data(), all.size() * sizeof(mcg::Op), cudaMemcpyHostToDevice));
    MCG_CUDA(cudaMalloc((void **)&b->d_tree_off, b->tree_op_offset.size() * sizeof(uint32_t)));
    MCG_CUDA(cudaMemcpy(b->d_tree_off, b->tree_op_offset.data(), b->tree_op_offset.size() * sizeof(uint32_t),
                        cudaMemcpyHostToDevice));
    if (b->max_global)
        MCG_CUDA(cudaMalloc((void **)&b->d_scratch,
                            (size_t)b->max_global * b->share * b->scratch_stride * sizeof(uint64_t)));
    MCG_CUDA(cudaMalloc((void **)&b->d_queue, sizeof(unsigned int)));
    const mcg_status lim = mcg::set_smem_limit(batch_kernel(b->ctas_per_sm, b->share, b->atleast), b->smem_bytes);
    if (lim != MCG_OK) return lim;
    if (run.stream) {
        b->stream = (cudaStream_t)run.stream;
    } else {
        MCG_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->own_stream = true;
    }
    MCG_CUDA(cudaEventCreate(&b->ev0));
    MCG_CUDA(cudaEventCreate(&b->ev1));
    return MCG_OK;
}

// Captures [zero queue, zero ones, persistent launch] for the current shapes.
mcg_status capture(mcg_batch *b, uint32_t n_inst, uint32_t iteration, uint64_t words) {
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    mcg::dev::BatchArgs a;
    a.ops = b->d_ops;
    a.tree_op_offset = b->d_tree_off;
    a.inst_tree = b->d_inst_tree;
    a.inst_thr_offset = b->d_thr_off;
    a.thr = b->d_thr;
    a.n_instances = n_inst;
    a.slabs_per_instance = (uint32_t)((words + kThreads - 1) / kThreads);
    a.words_per_instance = words;
    a.iteration = iteration;
    a.smem_slots = b->smem_slots;
    a.scratch = b->d_scratch;
    a.scratch_stride = b->scratch_stride;
    a.queue = b->d_queue;
    a.inst_ones = b->d_ones;
    a.group_first = b->d_group_first;
    a.group_size = b->d_group_size;
    a.n_groups = b->n_groups;
    cudaGraph_t g = nullptr;
    MCG_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(b->d_queue, 0, sizeof(unsigned int), b->stream);
    cudaMemsetAsync(b->d_ones, 0, (size_t)n_inst * sizeof(unsigned long long), b->stream);
    batch_kernel(b->ctas_per_sm, b->share, b->atleast)<<<b->grid, kThreads, b->smem_bytes, b->stream>>>(a);
    const cudaError_t launch_err = cudaGetLastError();
    const cudaError_t end_err = cudaStreamEndCapture(b->stream, &g);
    if (launch_err != cudaSuccess || end_err != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return mcg::fail(MCG_ERR_CUDA, std::string("batch capture: ") +
                                           cudaGetErrorString(launch_err != cudaSuccess ? launch_err : end_err));
    }
    const cudaError_t inst_err = cudaGraphInstantiate(&b->graph, g, 0);
    cudaGraphDestroy(g);
    if (inst_err != cudaSuccess) return mcg::fail(MCG_ERR_CUDA, cudaGetErrorString(inst_err));
    b->g_instances = n_inst;
    b->g_iteration = iteration;
    b->g_words = words;
    return MCG_OK;
}

}  // namespace

extern "C" {

mcg_status mcg_batch_create(const mcg_graph_desc *trees, uint32_t n_trees, const mcg_run_desc *run_in,
                            mcg_batch **out) {
    mcg::clear_error();
    if (!trees || !out || n_trees == 0) return mcg::fail(MCG_ERR_INVALID, "trees and out must be given");
    *out = nullptr;
    mcg_run_desc run{};
    if (run_in) run = *run_in;
    auto b = std::make_unique<mcg_batch>();
    for (uint32_t t = 0; t < n_trees; ++t) {
        mcg::Graph g;
        const std::string err = mcg::Graph::from_desc(trees[t], g);
        if (!err.empty()) return mcg::fail(MCG_ERR_INVALID, "tree " + std::to_string(t) + ": " + err);
        if (g.tally_nodes.empty()) return mcg::fail(MCG_ERR_INVALID, "tree " + std::to_string(t) + ": no tally node");
        b->trees.push_back(std::move(g));
    }
    int n_dev = 0;
    if (cudaGetDeviceCount(&n_dev) != cudaSuccess || n_dev == 0) {
        cudaGetLastError();
        return mcg::fail(MCG_ERR_NO_DEVICE, "no CUDA device visible");
    }
    b->device = run.device;
    const mcg_status st = setup(b.get(), run);
    if (st != MCG_OK) {
        release(b.get());
        return st;
    }
    *out = b.release();
    return MCG_OK;
}

mcg_status mcg_batch_destroy(mcg_batch *b) {
    mcg::clear_error();
    if (!b) return MCG_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    release(b);
    delete b;
    return MCG_OK;
}

mcg_status mcg_batch_run(mcg_batch *b, uint32_t n_inst, const uint32_t *inst_tree, const uint64_t *thr_offset,
                         const uint64_t *thresholds, uint64_t n_thr, uint32_t iteration, uint64_t words,
                         uint64_t *ones) {
    mcg::clear_error();
    if (!b || !inst_tree || !thr_offset || !thresholds || !ones) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    if (n_inst == 0 || words == 0) return MCG_OK;
    if (words > 0xFFFFFFFFull) return mcg::fail(MCG_ERR_INVALID, "words_per_instance exceeds the sample counter");
    const uint64_t slabs = (words + kThreads - 1) / kThreads;
    if ((uint64_t)n_inst * slabs >= 0xFFFFFFFFull) return mcg::fail(MCG_ERR_INVALID, "too many work items");
    if ((uint64_t)iteration + 2 >= (1ull << 26)) return mcg::fail(MCG_ERR_INVALID, "iteration out of range");
    for (uint32_t i = 0; i < n_inst; ++i) {
        if (inst_tree[i] >= b->trees.size()) return mcg::fail(MCG_ERR_INVALID, "instance tree out of range");
        if (thr_offset[i] + b->trees[inst_tree[i]].n_be > n_thr)
            return mcg::fail(MCG_ERR_INVALID, "instance thresholds out of range");
    }
    for (uint64_t k = 0; k < n_thr; ++k)
        if (thresholds[k] > (1ull << 32)) return mcg::fail(MCG_ERR_INVALID, "threshold above 2^32");
    // groups of up to `share` consecutive instances of one tree
    std::vector<uint32_t> gfirst, gsize;
    for (uint32_t i = 0; i < n_inst;) {
        uint32_t n = 1;
        while (n < b->share && i + n < n_inst && inst_tree[i + n] == inst_tree[i]) ++n;
        gfirst.push_back(i);
        gsize.push_back(n);
        i += n;
    }
    if ((uint64_t)gfirst.size() * slabs >= 0xFFFFFFFFull) return mcg::fail(MCG_ERR_INVALID, "too many work items");
    MCG_CUDA(cudaSetDevice(b->device));
    const uint32_t *old_tree = b->d_inst_tree, *old_gf = b->d_group_first, *old_gs = b->d_group_size;
    const uint64_t *old_off = b->d_thr_off, *old_thr = b->d_thr;
    const unsigned long long *old_ones = b->d_ones;
    MCG_CUDA(ensure(&b->d_inst_tree, b->cap_inst, n_inst));
    MCG_CUDA(ensure(&b->d_thr_off, b->cap_inst2, n_inst));
    MCG_CUDA(ensure(&b->d_thr, b->cap_thr, n_thr));
    MCG_CUDA(ensure(&b->d_ones, b->cap_ones, n_inst));
    MCG_CUDA(ensure(&b->d_group_first, b->cap_grp, gfirst.size()));
    MCG_CUDA(ensure(&b->d_group_size, b->cap_grp2, gsize.size()));
    const bool moved = old_tree != b->d_inst_tree || old_off != b->d_thr_off || old_thr != b->d_thr ||
                       old_ones != b->d_ones || old_gf != b->d_group_first || old_gs != b->d_group_size ||
                       b->n_groups != (uint32_t)gfirst.size();
    b->n_groups = (uint32_t)gfirst.size();
    MCG_CUDA(cudaMemcpyAsync(b->d_group_first, gfirst.data(), gfirst.size() * sizeof(uint32_t),
                             cudaMemcpyHostToDevice, b->stream));
    MCG_CUDA(cudaMemcpyAsync(b->d_group_size, gsize.data(), gsize.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             b->stream));
    MCG_CUDA(cudaMemcpyAsync(b->d_inst_tree, inst_tree, n_inst * sizeof(uint32_t), cudaMemcpyHostToDevice, b->stream));
    MCG_CUDA(cudaMemcpyAsync(b->d_thr_off, thr_offset, n_inst * sizeof(uint64_t), cudaMemcpyHostToDevice, b->stream));
    MCG_CUDA(cudaMemcpyAsync(b->d_thr, thresholds, n_thr * sizeof(uint64_t), cudaMemcpyHostToDevice, b->stream));
    if (!b->graph || moved || b->g_instances != n_inst || b->g_iteration != iteration || b->g_words != words) {
        const mcg_status st = capture(b, n_inst, iteration, words);
        if (st != MCG_OK) return st;
    }
    MCG_CUDA(cudaEventRecord(b->ev0, b->stream));
    MCG_CUDA(cudaGraphLaunch(b->graph, b->stream));
    MCG_CUDA(cudaEventRecord(b->ev1, b->stream));
    ++b->launches;
    MCG_CUDA(cudaMemcpyAsync(ones, b->d_ones, n_inst * sizeof(uint64_t), cudaMemcpyDeviceToHost, b->stream));
    MCG_CUDA(cudaStreamSynchronize(b->stream));
    float ms = 0;
    MCG_CUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    b->last_ms = ms;
    return MCG_OK;
}

mcg_status mcg_batch_info_get(mcg_batch *b, mcg_batch_info *info) {
    mcg::clear_error();
    if (!b || !info) return mcg::fail(MCG_ERR_INVALID, "NULL argument");
    info->n_trees = (uint32_t)b->trees.size();
    info->smem_slots = b->smem_slots;
    info->max_global_slots = b->max_global;
    info->grid_ctas = b->grid;
    info->total_ops = b->total_ops;
    info->launches = b->launches;
    info->last_kernel_ms = b->last_ms;
    info->instances_per_item = b->share;
    return MCG_OK;
}

}  // extern "C"

// Tree sizes for the uncertainty driver (ua.cpp).
uint32_t mcg_batch_tree_count(const mcg_batch *b) { return (uint32_t)b->trees.size(); }
uint32_t mcg_batch_tree_n_be(const mcg_batch *b, uint32_t t) { return b->trees[t].n_be; }
