// tma.cuh -- inline-PTX wrappers for the sm_90+/sm_100a asynchronous copy
// engine: mbarriers and 1-D bulk copies global -> shared (cp.async.bulk).
//
// Every wait has an iteration limit; a wait that runs out returns false so
// the caller can record an error and leave instead of hanging the GPU.
#pragma once

#include <cstdint>

namespace vfb::tma
{

__device__ __forceinline__ uint32_t smemAddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbarInit(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smemAddr(bar)), "r"(count) : "memory");
}

// makes the initialised barriers visible to the async proxy
__device__ __forceinline__ void fenceBarrierInit()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// orders earlier generic-proxy accesses of shared memory before later
// async-proxy (bulk copy) accesses of the same buffer
__device__ __forceinline__ void fenceProxyAsync() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbarArriveExpectTx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smemAddr(bar)), "r"(bytes)
                 : "memory");
}

// bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned) from
// global to shared, completing `bytes` transactions on `bar`
__device__ __forceinline__ void bulkLoad(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smemAddr(dst)),
        "l"(src), "r"(bytes), "r"(smemAddr(bar))
        : "memory");
}

// 32-bit global load kept in program order with the other asm statements
// (the producer issues it one tile ahead of its use)
__device__ __forceinline__ uint32_t ldgOrdered(const uint32_t* p)
{
    uint32_t v;
    asm volatile("ld.global.nc.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// per-thread asynchronous copy of 4 or 8 bytes global -> shared (cp.async,
// completed by cp.async.wait_group of the same thread)
template <int BYTES>
__device__ __forceinline__ void cpAsync(void* dst, const void* src)
{
    static_assert(BYTES == 4 || BYTES == 8, "cp.async.ca copies 4, 8 or 16 bytes");
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smemAddr(dst)), "l"(src), "n"(BYTES) : "memory");
}
__device__ __forceinline__ void cpAsyncCommit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
// waits until at most N of this thread's committed groups are still in flight
template <int N>
__device__ __forceinline__ void cpAsyncWait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// plain arrival (no transaction count)
__device__ __forceinline__ void mbarArrive(uint64_t* bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smemAddr(bar)) : "memory");
}

__device__ __forceinline__ bool mbarTryWait(uint64_t* bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smemAddr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// bounded wait for the phase with the given parity; false if the limit ran out
__device__ __forceinline__ bool mbarWait(uint64_t* bar, uint32_t parity, uint32_t maxIterations)
{
    for (uint32_t i = 0; i < maxIterations; ++i)
        if (mbarTryWait(bar, parity))
            return true;
    return false;
}

} // namespace vfb::tma
