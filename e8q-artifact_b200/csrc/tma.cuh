// Bulk-copy (TMA, cp.async.bulk) and mbarrier helpers for sm_100a, with
// bounded waits: a wait that runs out of time reports failure instead of
// spinning forever, and the caller records it in a device error word.
#pragma once

#include <cuda.h>
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

// One 2D tensor-map (TMA) tile load into shared memory completing on `bar`:
// box origin (x, y) in elements of the map (x * element size must be a
// multiple of 16 bytes). `map` is the address of a __grid_constant__ kernel
// parameter.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_addr(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// One bulk shared -> global copy (16-byte aligned addresses, size a multiple
// of 16), tracked by this thread's bulk groups.
__device__ __forceinline__ void bulk_s2g(void* gdst, const void* ssrc, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(gdst), "r"(smem_addr(ssrc)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// At most N of this thread's bulk groups still reading shared memory.
template <int N>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// At most N of this thread's bulk groups not yet complete.
template <int N>
__device__ __forceinline__ void bulk_wait() {
    asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}
// Generic-proxy shared-memory writes -> visible to the bulk-copy (async) proxy.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Invalidate an mbarrier whose phases are all complete, so its shared
// memory can be reused for plain data.
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while the previous kernel in the stream is still
// running; grid_dependency_wait() blocks until that kernel has completed and
// its memory is visible (a no-op for an ordinary launch), and
// launch_dependents() lets the next such kernel start early.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Plain arrival (count 1) on `bar`.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Non-blocking test of the phase with parity `phase` (true once it completed).
__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t phase) {
    uint32_t ok = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Potentially blocking test of the phase with parity `phase`: the thread is
// suspended until the phase completes or a hardware time limit passes (true
// once it completed).
__device__ __forceinline__ bool mbar_try(uint64_t* bar, uint32_t phase) {
    uint32_t ok = 0;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(phase)
        : "memory");
    return ok != 0;
}

// Wait for `phase` of `bar` (suspending tests, which wake as soon as the
// phase completes), giving up after about max_ms of device time, or as soon
// as *abort (when given) is set by another role of the CTA; a timeout sets
// *abort. Returns false when it gave up.
__device__ __forceinline__ bool mbar_wait_poll(uint64_t* bar, uint32_t phase, volatile int* abort, uint32_t max_ms) {
    if (mbar_try(bar, phase)) return true;
    const uint64_t t0 = global_ns();
    const uint64_t limit = static_cast<uint64_t>(max_ms) * 1000000ull;
    for (uint32_t i = 0; i < (1u << 30); ++i) {
        if (mbar_try(bar, phase)) return true;
        if ((i & 15u) == 15u) {
            if (abort && *abort) return false;
            if (global_ns() - t0 > limit) break;
        }
    }
    if (abort) *abort = 1;
    return false;
}

// Wait for `phase` of `bar`, giving up after about max_ms milliseconds.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t phase, uint32_t max_ms = 2000u) {
    return mbar_wait_poll(bar, phase, nullptr, max_ms);
}

// Like mbar_wait_bounded, but also gives up as soon as *abort is set (another
// role of the CTA timed out), and sets *abort itself on timeout.
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t phase, volatile int* abort,
                                                   uint32_t max_ms = 2000u) {
    return mbar_wait_poll(bar, phase, abort, max_ms);
}

}  // namespace e8qc
