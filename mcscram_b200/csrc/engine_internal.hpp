// engine_internal.hpp -- the engine object shared by engine.cu and is.cu.
#pragma once
#include <cuda_runtime.h>

#include <functional>
#include <utility>
#include <unordered_map>
#include <vector>

#include "graph.hpp"
#include "mcg.h"
#include "program.hpp"

namespace mcg {
namespace internal {
constexpr int kFusedThreads = 256;
constexpr uint64_t kDefaultChunkWords = 1ull << 21;
}  // namespace internal
}  // namespace mcg

struct mcg_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::unordered_map<void *, size_t> work_bytes;  // sizes of the kept-buffer cache's allocations
    uint32_t mode = MCG_MODE_FUSED;
    mcg::Graph graph;
    mcg::Program prog;

    // fused
    uint4 *d_ops = nullptr;
    uint64_t *d_scratch = nullptr;
    uint64_t scratch_stride = 0;
    uint32_t nt = mcg::internal::kFusedThreads;
    uint32_t ctas_per_sm = 2;
    uint32_t grid = 0;
    uint32_t smem_bytes = 0;
    bool tally_in_smem = false;
    uint64_t chunk_words = mcg::internal::kDefaultChunkWords;

    // tallies
    unsigned long long *d_tally = nullptr;
    uint64_t total_bits = 0;

    // layered
    uint4 *d_be = nullptr;
    uint4 *d_meta = nullptr;
    uint32_t *d_inputs = nullptr;
    uint32_t *d_tally_nodes = nullptr;
    uint32_t *d_layer_gates = nullptr;
    std::vector<uint32_t> layer_offsets;  // into d_layer_gates, size n_layers + 1
    uint64_t *d_buf = nullptr;
    uint64_t buf_words = 0;
    uint64_t layered_max_words = 0;

    // staged
    uint4 *d_smeta = nullptr;           // gate meta with counter bits for the bit-sliced ATLEAST
    uint2 *d_gate_tally = nullptr;      // per gate {offset, count} into d_gate_tally_list
    uint32_t *d_gate_tally_list = nullptr;
    uint32_t *d_be_tally_nodes = nullptr;  // tallied basic events
    uint32_t *d_be_tally_idx = nullptr;
    uint32_t n_be_tally = 0;
    uint64_t *d_stage[2] = {nullptr, nullptr};
    uint2 *d_event_table = nullptr;     // per-pass sampler table, n_be x kEventTableStride
    uint32_t table_iteration = 0xFFFFFFFFu;
    const uint4 *d_be_sample = nullptr;  // basic-event table the sampler phase reads (d_be unless overridden)
    // optional work queued on the gate stream after each chunk's gate phase
    std::function<mcg_status(cudaStream_t, const uint64_t *, uint64_t)> chunk_hook;
    // optional work queued on the sampler stream after a chunk's basic-event
    // words are written and before its gates read them (buffer, W, word_begin)
    std::function<mcg_status(cudaStream_t, uint64_t *, uint64_t, uint64_t)> sample_hook;
    uint32_t sampler_smem = 0;          // dynamic smem that caps sampler blocks per SM
    uint64_t stage_words = 0;           // words per chunk the stage buffers hold
    cudaStream_t s_a = nullptr, s_b = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_a[2] = {nullptr, nullptr}, ev_b[2] = {nullptr, nullptr};
    cudaEvent_t ev_join_a = nullptr, ev_join_b = nullptr;
    // strip
    uint64_t *d_strip_scratch = nullptr;   // per warp n_nodes x 32 words
    unsigned long long *d_queue = nullptr; // strip counter
    uint4 *d_strip_groups = nullptr;       // strip mode: gate groups, one layer at a time
    uint32_t *d_strip_gin = nullptr;       // their inputs, slot-major, four records per slot
    uint4 *d_strip_ginfo = nullptr;        // per grouped gate: output node, tally offset / count, gate id
    uint32_t n_strip_groups = 0;
    uint32_t strip_grid = 0;
    uint32_t strip_smem = 0;               // tally counters in shared memory (0: global atomics)
    uint32_t strip_blocks = 6;             // resident blocks per SM the kernel is built for

    cudaEvent_t ev_snap[2] = {nullptr, nullptr};  // tally snapshots (slots behind d_tally)
    uint64_t snap_total[2] = {0, 0};

    mcg_run_desc run_desc{};                  // options the engine was created with
    bool prog_compiled = false;               // fused program compiled (fused mode, or on request)
    bool profile_a = false;                   // time every sampler-phase launch
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> prof_events;
    size_t prof_used = 0;

    uint64_t launches = 0;
};


namespace mcg {
namespace internal {

// Staged pass over [word_begin, word_begin + count) for n_it passes (engine.cu).
mcg_status run_staged(mcg_engine *e, uint32_t it_first, uint32_t n_it, uint64_t word_begin, uint64_t count);

}  // namespace internal
}  // namespace mcg
