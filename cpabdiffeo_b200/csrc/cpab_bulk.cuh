// cpab_bulk.cuh -- bulk asynchronous global->shared copies (cp.async.bulk,
// the untiled TMA path) completing on a shared-memory mbarrier, for the
// streaming kernels.  Every copy reads this GPU's own global memory into the
// issuing CTA's own shared memory; no copy is shared between CTAs.
//
// Requirements of cp.async.bulk: source and destination 16-byte aligned,
// size a multiple of 16 bytes.  Callers check these before choosing the
// bulk path.
#pragma once

#include <stdint.h>

namespace cpab {

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async proxy (before first use).
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces `bytes` of transaction (the copies below).
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// dst (shared) <- src (global), `bytes` bytes, completing on bar.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait for phase `parity` of bar to complete, giving up after `limit_ns`
// nanoseconds of global time (each try_wait may itself suspend the thread
// for a short, hardware-chosen time).  Returns false on give-up; the caller
// records the failure instead of hanging.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint64_t limit_ns = 2000000000ull)
{
    const uint32_t a = smem_addr(bar);
    const uint64_t t0 = global_ns();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

}  // namespace cpab
