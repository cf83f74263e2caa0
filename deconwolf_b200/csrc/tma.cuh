// tma.cuh -- bulk asynchronous copies (TMA, sm_90+) and mbarriers.
//
// Only the plain, non-multicast forms are used: cp.async.bulk from this
// GPU's global memory into the issuing CTA's shared memory, completing on an
// mbarrier in that CTA.  Every wait is bounded: after kWaitLimit polls the
// waiting thread reports a timeout, and the caller takes a uniform exit
// (see wait_all) so that no barrier is left half-arrived.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace dwcu {

constexpr unsigned kWaitLimit = 1u << 26;  // polls of try_wait (each may suspend briefly)

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t) __cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same memory
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 1-D bulk copy global -> shared; bytes and both addresses multiples of 16
__device__ __forceinline__ void tma_load_1d(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on a barrier phase by every thread of the block, followed by
// a block-wide vote: returns true on all threads, or false on all threads
// when any of them gave up (the caller then skips the rest of its work).
__device__ __forceinline__ bool wait_all(uint64_t *bar, uint32_t parity, int *err_flag, int code,
                                         unsigned limit = kWaitLimit)
{
    unsigned n = 0;
    bool ok = false;
    while (n < limit) {
        if (mbar_try_wait(bar, parity)) {
            ok = true;
            break;
        }
        ++n;
    }
    if (!ok && err_flag) atomicOr(err_flag, code);
    return __syncthreads_and(ok ? 1 : 0) != 0;
}

// 16-byte asynchronous copy global -> shared through the load/store path
// (cp.async, L1 bypassed); completion is awaited with cp_async_wait_all.
__device__ __forceinline__ void cp_async16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Bounded wait by one thread for a copy still in flight before an early exit
// (a CTA must not exit while a bulk copy is writing its shared memory).
__device__ __forceinline__ void drain(uint64_t *bar, uint32_t parity)
{
    for (unsigned n = 0; n < kWaitLimit; ++n)
        if (mbar_try_wait(bar, parity)) return;
}

}  // namespace dwcu
