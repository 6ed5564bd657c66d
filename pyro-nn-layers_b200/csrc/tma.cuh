// tma.cuh -- Tensor Memory Accelerator (cp.async.bulk.tensor) and mbarrier
// helpers for sm_100a, written as inline PTX.
//
// Only plain (non-multicast) tiled loads from this GPU's own memory are used.
// Every wait is bounded: a wait that does not complete within the spin limit
// records an error code in a device flag and returns false, so a kernel can
// never hang on a lost transaction.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pyronn {

// device error codes written to the workspace header
enum DeviceError : unsigned {
    DEVICE_OK = 0,
    DEVICE_ERROR_MBARRIER_TIMEOUT = 1,
};

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// makes the mbarrier initialisation visible to the async (TMA) proxy
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cta.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity; gives up after max_spins
// attempts (each try_wait itself blocks for a bounded time), recording
// DEVICE_ERROR_MBARRIER_TIMEOUT in *err.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, unsigned *err,
                                                  unsigned max_spins = (1u << 22))
{
    for (unsigned i = 0; i < max_spins; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicCAS(err, (unsigned)DEVICE_OK, (unsigned)DEVICE_ERROR_MBARRIER_TIMEOUT);
    return false;
}

// 3D tiled TMA load (box given by the tensor map) into shared memory,
// completing on the mbarrier.  x must be a multiple of 16 bytes / element size.
__device__ __forceinline__ void tma_load_3d(void *smem_dst, const CUtensorMap *map, int x, int y, int z,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(smem_dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
        : "memory");
}

}  // namespace pyronn
