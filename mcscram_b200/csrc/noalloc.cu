// noalloc.cu -- the fused kernel for callers that cannot allocate device memory
// (mcg_run_fused_noalloc in include/mcg.h).
//
// Some callers of the engine must not call cudaMalloc: code that enqueues
// work while a CUDA graph is being captured, processes whose device memory is
// owned by their own pool or held to a fixed budget, and latency-bound
// services where cudaMalloc/cudaFree would add implicit synchronisation.
// They compile a program with mcg_compile, place it in device memory they
// already own, and call this entry point.  The values the program keeps
// outside shared memory go to the fixed array below instead of an engine's
// scratch allocation.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "error.hpp"
#include "kernels.cuh"
#include "mcg.h"
#include "smem_limit.hpp"

// Global-scratch slots of the fused kernel, one array per device that loads
// the library, held until the process exits.  Every call shares it; no call
// needs it cleared, because the program writes each slot before reading it.
static __device__ __align__(256) uint64_t g_noalloc_scratch[MCG_NOALLOC_SCRATCH_BYTES / sizeof(uint64_t)];

namespace {

constexpr int kThreads = 256;
constexpr int kCtasPerSm = 2;
constexpr uint64_t kChunkWords = 1ull << 21;
constexpr int kMaxDevices = 64;

struct DeviceSetup {
    bool done = false;
    uint64_t *scratch = nullptr;  // device address of g_noalloc_scratch on this device
    int sms = 0;
    size_t smem_cap = 0;
};

std::mutex g_setup_mutex;
DeviceSetup g_setup[kMaxDevices];

// Once per device, with that device current: resolve the array's device
// address (the host-side symbol is only a stand-in), read the SM count and
// raise the kernel's dynamic shared-memory limit.  Nothing is allocated.
// The result is kept for the life of the process: a caller that resets the
// device (cudaDeviceReset) drops the module that holds the array, and this
// entry point must not be called again in that process.
mcg_status setup_device(int dev, DeviceSetup *&out) {
    if (dev < 0 || dev >= kMaxDevices) return mcg::fail(MCG_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    DeviceSetup &s = g_setup[dev];
    if (!s.done) {
        void *p = nullptr;
        cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (err != cudaSuccess) return mcg::fail(MCG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(err));
        int sms = 0, optin = 0, per_sm = 0;
        if ((err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
            (err = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess ||
            (err = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess)
            return mcg::fail(MCG_ERR_CUDA, std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(err));
        // what one of the two CTAs per SM may use; the kernel's limit itself
        // is the device maximum, as engines with this kernel set it too
        const size_t cap = std::min<size_t>((size_t)optin, (size_t)per_sm / kCtasPerSm) - 1024;
        const mcg_status lim = mcg::set_smem_limit(mcg::dev::k_fused<kThreads, kCtasPerSm, 1, 1>, cap);
        if (lim != MCG_OK) return lim;
        s.scratch = static_cast<uint64_t *>(p);
        s.sms = sms;
        s.smem_cap = cap;
        s.done = true;
    }
    out = &s;
    return MCG_OK;
}

}  // namespace

extern "C" mcg_status mcg_run_fused_noalloc(const void *d_ops, uint64_t n_ops, uint32_t smem_slots,
                                            uint32_t global_slots, uint64_t *d_ones, uint32_t n_tally,
                                            uint32_t iteration_first, uint32_t n_iterations, uint64_t word_begin,
                                            uint64_t word_count, void *stream) {
    mcg::clear_error();
    if (!d_ops || n_ops < 2) return mcg::fail(MCG_ERR_INVALID, "d_ops must hold a whole program from mcg_compile");
    if (n_tally > 0 && !d_ones) return mcg::fail(MCG_ERR_INVALID, "d_ones is NULL");
    if (word_begin + word_count > (1ull << 32) || word_begin + word_count < word_begin)
        return mcg::fail(MCG_ERR_INVALID, "word range exceeds the 32-bit sample counter");
    if ((uint64_t)iteration_first + n_iterations + 1 >= (1ull << 26))
        return mcg::fail(MCG_ERR_INVALID, "iteration exceeds the 26-bit pass counter field");
    if (n_iterations == 0 || word_count == 0) return MCG_OK;
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return mcg::fail(MCG_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(err));
    DeviceSetup *s = nullptr;
    mcg_status st = setup_device(dev, s);
    if (st != MCG_OK) return st;

    const size_t slot_bytes = (size_t)kThreads * sizeof(uint64_t);
    const size_t slots_bytes = (size_t)smem_slots * slot_bytes;
    if (slots_bytes > s->smem_cap)
        return mcg::fail(MCG_ERR_INVALID, "smem_slots exceeds the shared memory of one CTA; compile with a smaller budget");
    const size_t tally_bytes = (size_t)n_tally * sizeof(unsigned long long);
    const bool tally_in_smem = tally_bytes <= s->smem_cap - slots_bytes;
    const uint64_t grid_max = (uint64_t)s->sms * kCtasPerSm;
    // Scratch at the largest grid a call uses, checked before any launch.
    const uint64_t need = (uint64_t)global_slots * grid_max * kThreads * sizeof(uint64_t);
    if (need > MCG_NOALLOC_SCRATCH_BYTES)
        return mcg::fail(MCG_ERR_INVALID, "the program needs " + std::to_string(need) +
                                              " bytes of global scratch at full occupancy; the static scratch holds " +
                                              std::to_string((uint64_t)MCG_NOALLOC_SCRATCH_BYTES) +
                                              " (compile with a larger shared-memory budget or use mcg_create/mcg_run)");
    const uint32_t smem = (uint32_t)(slots_bytes + (tally_in_smem ? tally_bytes : 0));
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    for (uint64_t off = 0; off < word_count; off += kChunkWords) {
        const uint64_t count = std::min<uint64_t>(kChunkWords, word_count - off);
        const uint32_t grid = (uint32_t)std::min<uint64_t>(grid_max, std::max<uint64_t>((count + kThreads - 1) / kThreads, 1));
        mcg::dev::FusedArgs a;
        a.ops = static_cast<const uint4 *>(d_ops);
        a.smem_slots = smem_slots;
        a.scratch = s->scratch;
        a.scratch_stride = (uint64_t)grid * kThreads;
        a.tally = reinterpret_cast<unsigned long long *>(d_ones);
        a.n_tally = n_tally;
        a.tally_in_smem = tally_in_smem ? 1u : 0u;
        a.iteration_first = iteration_first;
        a.n_iterations = n_iterations;
        a.word_begin = word_begin + off;
        a.word_count = count;
        mcg::dev::k_fused<kThreads, kCtasPerSm, 1, 1><<<grid, kThreads, smem, cs>>>(a);
        err = cudaGetLastError();
        if (err != cudaSuccess) return mcg::fail(MCG_ERR_CUDA, std::string("k_fused launch: ") + cudaGetErrorString(err));
    }
    return MCG_OK;
}
