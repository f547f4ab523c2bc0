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

// Persistent-grid size (SM count x resident CTAs) of `kern` on the current
// device, after its shared-memory opt-in; `cache` (one per kernel) holds it
// per device ordinal < 64.  Returns 0 on a CUDA error.
template <class F>
inline int persistent_grid(std::atomic<uint64_t>& mask, std::atomic<int> (&cache)[kDevAttrSlots], F kern, int threads,
                           int bytes)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    const bool slot = dev >= 0 && dev < kDevAttrSlots;
    if (slot) {
        const int g = cache[dev].load(std::memory_order_acquire);
        if (g > 0) return g;
    }
    if (smem_optin(mask, kern, bytes) != cudaSuccess) return 0;
    int nsm = 0, occ = 0;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, bytes) != cudaSuccess || occ < 1)
        return 0;
    const int g = nsm * occ;
    if (slot) cache[dev].store(g, std::memory_order_release);
    return g;
}

}  // namespace claw2
