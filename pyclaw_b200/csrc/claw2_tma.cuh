// claw2_tma.cuh -- tensor-memory-accelerator (TMA) staging of a tile's input
// halo into shared memory, for sm_100a.
//
// One thread of the CTA arms an mbarrier with the byte count of the copies
// and issues cp.async.bulk.tensor loads of boxes of the state planes; the TMA
// unit writes the boxes into shared memory (zeros outside the tensor) and
// completes the transaction on the mbarrier, on which every thread then
// waits.  The copies read this GPU's own memory and carry no cluster
// multicast.
//
// Shared-memory layout of one box: the tensor map uses the 128-byte swizzle,
// so a box row is 16 doubles (128 bytes) and the 16-byte chunk k of row r is
// stored at chunk k ^ (r & 7).  A warp reading one row (16 lanes per box)
// touches each bank once per 128 bytes; a warp reading down a column spreads
// over 8 chunks, so the 32 rows cost 4 shared-memory wavefronts instead of 2.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#include <cuda.h>   // CUtensorMap

namespace claw2 {

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    // make the initialised barrier visible to the TMA unit (async proxy)
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for phase `parity` of the barrier, giving up after about `limit`
// SM clock cycles; returns false if it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit)
{
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

// Tiled 3D load of the box at (x, y, z) of `map` into shared memory at dst
// (1024-byte aligned for the 128-byte swizzle), completing on `bar`.  x times
// the element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
        ::"r"(smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_addr(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

}  // namespace claw2
#endif

namespace claw2 {

// Index (in doubles) of element (row r, column c) of a 128-byte-swizzled box
// whose rows are 16 doubles: chunk (c >> 1) of row r is stored at chunk
// (c >> 1) ^ (r & 7).
#if defined(__CUDACC__)
__host__ __device__
#endif
inline int swz128(int r, int c)
{
    return r * 16 + ((((c >> 1) ^ (r & 7)) << 1) | (c & 1));
}

}  // namespace claw2
