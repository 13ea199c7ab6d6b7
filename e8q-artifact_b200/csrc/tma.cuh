// Bulk-copy (TMA, cp.async.bulk) and mbarrier helpers for sm_100a, with
// bounded waits: a wait that runs out of iterations reports failure instead
// of spinning forever, and the caller records it in a device error word.
#pragma once

#include <stdint.h>

namespace e8qc {

// Error word codes written by kernels (the host maps them to E8QC_ETIMEOUT).
constexpr uint32_t kErrWaitTimeout = 1u;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make mbarrier initialisation visible to the async (bulk-copy) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

// One bulk global -> shared copy completing on `bar` (16-byte aligned
// addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// try_wait with a suspend-time hint: the thread sleeps until the phase
// completes or ~1 ms passes, instead of spinning on issue slots.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t phase) {
    uint32_t ok = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase), "r"(1000000u)
        : "memory");
    return ok != 0;
}

// Wait for `phase` of `bar` with an iteration cap (each try_wait suspends for
// at most ~1 ms). Returns false on timeout (about 2 s).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint32_t max_iter = 2048u) {
    for (uint32_t i = 0; i < max_iter; ++i)
        if (mbar_try_wait(bar, phase)) return true;
    return false;
}

}  // namespace e8qc
