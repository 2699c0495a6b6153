// Tensor-memory-access (TMA) loads into shared memory and the mbarriers that count their bytes, for sm_100a.
//
// A tile arrives by cp.async.bulk.tensor from a CUtensorMap over a front's panel (built on the host, kept in global
// memory, 64-byte aligned) into 1024-byte aligned shared memory, and signals an mbarrier with its byte count. Every
// wait here is bounded: after MBARRIER_SPIN_LIMIT polls it gives up and returns false, and the caller sets an error
// flag the host turns into a status, so a tensor-core kernel never waits forever on a copy.
//
// These loads never use cluster multicast: every tensor map covers this GPU's own memory only.
#pragma once

#include <cstdint>

namespace oosgpu::device
{

constexpr unsigned MBARRIER_SPIN_LIMIT = 1u << 26;

__device__ __forceinline__ unsigned sharedAddress(const void* p)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbarrierInit(std::uint64_t* bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(sharedAddress(bar)), "r"(count) : "memory");
}

// Makes the barriers' initialisation visible to the async proxy (the TMA unit) before the first copy uses them.
__device__ __forceinline__ void fenceBarrierInit()
{
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// One arrival that also announces `bytes` of copies the barrier must see complete.
__device__ __forceinline__ void mbarrierExpectBytes(std::uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(sharedAddress(bar)), "r"(bytes)
                 : "memory");
}

// Polls the barrier's phase `parity` at most MBARRIER_SPIN_LIMIT times; false when it did not complete.
__device__ __forceinline__ bool mbarrierWait(std::uint64_t* bar, unsigned parity)
{
    const unsigned address = sharedAddress(bar);
    for (unsigned poll = 0; poll < MBARRIER_SPIN_LIMIT; ++poll)
    {
        unsigned done = 0;
        asm volatile("{\n"
                     ".reg .pred p;\n"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     "selp.u32 %0, 1, 0, p;\n"
                     "}\n"
                     : "=r"(done)
                     : "r"(address), "r"(parity)
                     : "memory");
        if (done != 0)
            return true;
    }
    return false;
}

// Orders this thread's later use of a tensor map written to global memory before the kernel started.
__device__ __forceinline__ void acquireTensorMap(const void* map)
{
    asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;\n" ::"l"(map) : "memory");
}

// A 2-D tile of the tensor map at (x, y) (x the contiguous coordinate, in elements) into shared memory, counted on
// `bar`. x * element size must be a multiple of 16 bytes.
__device__ __forceinline__ void tmaLoad2d(void* shared, const void* map, int x, int y, std::uint64_t* bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(sharedAddress(shared)),
                 "l"(map), "r"(x), "r"(y), "r"(sharedAddress(bar))
                 : "memory");
}

// The same with the destination given as a shared-memory address.
__device__ __forceinline__ void tmaLoad2dShared(unsigned shared, const void* map, int x, int y, std::uint64_t* bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(shared),
                 "l"(map), "r"(x), "r"(y), "r"(sharedAddress(bar))
                 : "memory");
}

// Orders this thread's (and, after a barrier, the block's) ordinary shared-memory accesses before later TMA writes
// to the same memory.
__device__ __forceinline__ void fenceProxyAsync()
{
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

} // namespace oosgpu::device
