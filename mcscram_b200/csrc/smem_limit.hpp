// smem_limit.hpp -- dynamic shared-memory limits of the library's kernels.
//
// cudaFuncAttributeMaxDynamicSharedMemorySize belongs to a kernel
// instantiation in one device context, not to an engine: every engine,
// batch or no-allocation call that launches the same instantiation on the
// same device sees the value the last caller set.  Setting it to one
// program's own need would let an engine created later with a smaller
// program lower it under a live engine with a larger one, whose next launch
// then fails with cudaErrorInvalidValue.  The limit is therefore always set
// to the most the device allows the kernel (its opt-in maximum per block less
// the kernel's static shared memory): the same value for every caller, so
// the order in which engines are created does not matter.  The attribute only
// bounds what a launch may ask for; residency still follows each launch's
// own dynamic shared memory.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "error.hpp"

namespace mcg {

// Raises `func`'s dynamic shared-memory limit on the current device to the
// device maximum; fails when `need` bytes exceed it.
template <typename F>
inline mcg_status set_smem_limit(F func, size_t need) {
    int dev = 0, optin = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    cudaFuncAttributes fa{};
    if (err == cudaSuccess) err = cudaFuncGetAttributes(&fa, reinterpret_cast<const void *>(func));
    if (err != cudaSuccess) return fail(MCG_ERR_CUDA, std::string("kernel attributes: ") + cudaGetErrorString(err));
    const size_t cap = (size_t)optin > fa.sharedSizeBytes ? (size_t)optin - fa.sharedSizeBytes : 0;
    if (need > cap)
        return fail(MCG_ERR_INVALID, "a launch needs " + std::to_string(need) +
                                         " bytes of dynamic shared memory; the device allows " + std::to_string(cap));
    err = cudaFuncSetAttribute(reinterpret_cast<const void *>(func), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)cap);
    if (err != cudaSuccess) return fail(MCG_ERR_CUDA, std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(err));
    return MCG_OK;
}

}  // namespace mcg
