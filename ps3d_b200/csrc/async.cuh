// async.cuh — bulk global->shared copies on the TMA engine (no multicast,
// no tensor map) completing on an mbarrier, with bounded waits.
#pragma once
#include "common.cuh"

namespace ps3d {

constexpr long kMbarWaitLimit = 1L << 21;   // polls of ~1 us at most: a wait ends within seconds

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
// arrive once and add `bytes` to the transaction count of the current phase
__device__ __forceinline__ void mbar_expect(unsigned long long* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// one poll of the phase with the given parity; a thread may be suspended up
// to the 1 us hint inside the instruction
__device__ __forceinline__ bool mbar_try(unsigned long long* bar, unsigned parity) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity), "r"(1000u)
        : "memory");
    return done != 0;
}
// bounded wait: false if the phase did not complete within the limit
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity) {
    for (long it = 0; it < kMbarWaitLimit; ++it)
        if (mbar_try(bar, parity)) return true;
    return false;
}
// orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (bulk copy) accesses
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// bytes (a multiple of 16) from 16-byte aligned global src to shared dst
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace ps3d
