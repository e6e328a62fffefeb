/*
 * Bulk-copy pipeline primitives (PTX, sm_90+ / sm_100a) shared by the fused
 * step kernels: 1-D bulk copies global -> shared memory that complete on an
 * mbarrier, and bounded waits on it.
 */
#ifndef GC_BULK_PIPE_CUH
#define GC_BULK_PIPE_CUH

#include <stdint.h>

namespace gcpipe {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
/* 1-D bulk copy global -> this CTA's shared memory, completing on `bar`;
 * dst, src and bytes must be multiples of 16 */
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
/* bounded wait: gives up after `limit` polls (each poll may suspend briefly) */
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit) {
    for (int it = 0; it < limit; it++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

} // namespace gcpipe

#endif
