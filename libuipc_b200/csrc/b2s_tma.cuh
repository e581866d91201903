// Bulk asynchronous copies (TMA, cp.async.bulk) into shared memory with
// mbarrier completion, for the streaming kernels. Every wait is bounded: a
// wait that runs out sets an error bit and returns false instead of spinning
// forever.
#pragma once
#include <stdint.h>

namespace b2s
{
// bounded mbarrier wait: ~2^22 try_wait rounds (each suspends in hardware for
// a short interval), far beyond any legitimate copy latency
constexpr uint32_t MBAR_WAIT_ROUNDS = 1u << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// make the initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's prior generic-proxy shared-memory accesses before
// subsequent async-proxy writes into the same buffer
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// 1-D bulk copy global -> shared; dst, src 16-byte aligned, bytes % 16 == 0
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
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

// returns false (and sets `err_bit` in *err) when the wait runs out
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, int err_bit)
{
    for(uint32_t i = 0; i < MBAR_WAIT_ROUNDS; ++i)
        if(mbar_try_wait(bar, parity))
            return true;
    if(err)
        atomicOr(err, err_bit);
    return false;
}
}  // namespace b2s
