// icb_bulk.cuh — bulk global -> shared copies completed on an mbarrier
// (PTX cp.async.bulk, the untiled form of the Tensor Memory Accelerator),
// and a bounded wait on them.
//
// Rules the callers keep: both addresses and the size are multiples of 16
// bytes; the barrier of a stage is armed (expect_tx) by the issuing thread
// before its copies; a stage that threads have read with ordinary loads is
// refilled only after a CTA barrier and fence_proxy_async() by the issuer.
#pragma once
#include <cstdint>

namespace icb {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Makes the initialised barriers visible to the async proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses of shared memory
// before its later async-proxy ones (a refill of a stage that was read).
__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// One arrival that also expects `bytes` of transactions in this phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// One plain arrival (release semantics at CTA scope).
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0u;
}

// As mbar_try_wait, letting the thread sleep up to hint_ns for the phase
// (it wakes when the phase completes): a waiting warp takes no issue slots.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint64_t* bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0u;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
    return t;
}

// Waits for the phase of the given parity to complete: false after about a
// second (or 2^26 polls) without completion.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 255u) == 0u && globaltimer_ns() - t0 > 1000000000ull) return false;
    }
    return false;
}

// As mbar_wait_bounded, and also gives up as soon as *abort is nonzero
// (another warp of the CTA gave up first).
__device__ __forceinline__ bool mbar_wait_or_abort(uint64_t* bar, uint32_t parity, const volatile int* abort) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t it = 0; it < (1u << 26); ++it) {
        if (mbar_try_wait_sleep(bar, parity, 20000u)) return true;
        if (*abort) return false;
        if (globaltimer_ns() - t0 > 1000000000ull) return false;
    }
    return false;
}

// Named CTA barrier `id` over `nthreads` threads (a multiple of 32) that
// also ORs a predicate across them: every participant gets the same result.
template <int ID, int NTHREADS>
__device__ __forceinline__ bool bar_sync_or(bool pred) {
    uint32_t r;
    asm volatile(
        "{\n .reg .pred q, p;\n setp.ne.u32 q, %1, 0;\n bar.red.or.pred p, %2, %3, q;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(r)
        : "r"(pred ? 1u : 0u), "n"(ID), "n"(NTHREADS)
        : "memory");
    return r != 0u;
}

}  // namespace icb
