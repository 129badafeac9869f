// Bulk asynchronous copies global -> shared (the TMA engine, 1-D form) with
// mbarrier completion, and the bounded warp-wide wait on them.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace tg {

// Each CTA copies only into its own shared memory.  Waits are bounded:
// kWaitLimit polls of mbarrier.try_wait (each poll may suspend the thread for
// a short hardware-defined time) before giving up.
constexpr unsigned kWaitLimit = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait of the whole warp; true when every lane saw the phase complete.
__device__ __forceinline__ bool mbar_wait_warp(unsigned long long *bar, uint32_t parity, unsigned limit = kWaitLimit)
{
    bool done = false;
#pragma unroll 1
    for (unsigned i = 0; i < limit && !done; ++i) done = mbar_try_wait(bar, parity);
    return __all_sync(0xffffffffu, done);
}


}  // namespace tg
