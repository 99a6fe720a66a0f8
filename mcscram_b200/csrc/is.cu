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
#include <vector>

#include "engine_internal.hpp"
#include "error.hpp"
#include "mcg_is.h"

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

extern "C" {

mcg_status mcg_is_create(const mcg_graph_desc *graph, const mcg_run_desc *run_in, mcg_is **out) {
    mcg::clear_error();
    if (!graph || !out) return mcg::fail(MCG_ERR_INVALID, "graph and out must not be NULL");
    *out = nullptr;
    if (graph->n_tally != 1) return mcg::fail(MCG_ERR_INVALID, "the tally list must hold exactly the top event");
    mcg_run_desc run{};
    if (run_in) run = *run_in;
    run.mode = MCG_MODE_STAGED;
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
    MCG_CUDA(cudaFuncSetAttribute(k_is_weights, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)is->weight_smem));
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
    const double two32 = 4294967296.0;
    for (uint32_t i = 0; i < nb; ++i) {
        const uint64_t tp = g.be_threshold[i], tq = q_thr[i];
        const bool fixed = tp == 0 || tp >= (1ull << 32);
        if (fixed ? tq != tp : (tq == 0 || tq >= (1ull << 32)))
            return mcg::fail(MCG_ERR_INVALID, "proposal threshold " + std::to_string(i) +
                                                  " must lie in [1, 2^32 - 1] (or equal a constant nominal one)");
        beq[i] = make_uint4((uint32_t)g.be_pdag_idx[i] + 1u, g.be_event_idx[i] + 1u, (uint32_t)tq, (uint32_t)(tq >> 32));
        if (fixed) continue;
        const double p = (double)tp / two32, q = (double)tq / two32;
        const double l1 = std::log1p(-p) - std::log1p(-q);
        a[i] = std::log(p) - std::log(q) - l1;
        C += l1;
    }
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
