// claw2_devattr.h -- per-device kernel set-up shared by the launchers.
//
// cudaFuncSetAttribute acts on the device that is current when it is called,
// so a kernel that needs more than 48 KB of dynamic shared memory must opt in
// once on every device it runs on; a process that steps on several GPUs
// reaches each of them through the same launcher.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

namespace claw2 {

constexpr int kDevAttrSlots = 64;   // device ordinals remembered per kernel

// Opt `kern` in to `bytes` of dynamic shared memory on the current device.
// `mask` (one per kernel) remembers the devices with ordinal < 64 that are
// already set; any other device is set before every launch.
template <class F>
inline cudaError_t smem_optin(std::atomic<uint64_t>& mask, F kern, int bytes)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const uint64_t bit = (dev >= 0 && dev < kDevAttrSlots) ? (uint64_t(1) << dev) : 0;
    if (bit && (mask.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e != cudaSuccess) return e;
    if (bit) mask.fetch_or(bit, std::memory_order_acq_rel);
    return cudaSuccess;
}

}  // namespace claw2
