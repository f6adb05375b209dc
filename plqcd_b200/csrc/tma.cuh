// tma.cuh -- inline-PTX wrappers for tensor-memory-access loads and the
// shared-memory mbarriers that complete them (sm_90+ instructions, used here
// on sm_100a). Loads are plain tile loads into this CTA's shared memory;
// nothing here multicasts.
//
// Every wait is bounded: a wait gives up after a time limit read from
// %globaltimer and reports failure, so a kernel can record an error and
// return instead of spinning forever.
#pragma once

#include <cstdint>

namespace plqcd {
namespace dev {

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// makes barrier initialisation visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one arrival that also announces `bytes` of transactions for this phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// Proxy fence for shared memory. A buffer's consumers read it with plain
// (generic-proxy) loads and release it on an mbarrier; the producer then
// refills it with tile loads, which write through the async proxy. The
// producer issues this fence after it has acquired the released buffer and
// before the refill: the fence then lies on the causality path from the
// consumers' reads to the refill's writes, so no write can land before a
// read of the old contents. Without it, on B200, a refill now and then
// overwrote a stage that was still being read (whole tiles of wrong results,
// mostly with longer epilogues).
__device__ __forceinline__ void fence_async_proxy_shared() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

// true once the phase of parity `parity` has completed
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

// try_wait that may suspend the thread for up to hint_ns until the phase
// completes (instead of returning at once)
__device__ __forceinline__ bool mbar_try_wait_hint(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}

// Bounded wait. Returns false when `limit_ns` passed first, or when another
// thread of the CTA raised `*abort` meanwhile. hint_ns > 0: each retry may
// suspend the thread up to hint_ns until the phase completes (fewer polls
// issued while waiting).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, uint64_t limit_ns,
                                          const volatile int *abort, uint32_t hint_ns = 0) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    for (;;) {
#pragma unroll 1
        for (int i = 0; i < 32; i++)
            if (hint_ns ? mbar_try_wait_hint(bar, parity, hint_ns) : mbar_try_wait(bar, parity)) return true;
        if (abort && *abort) return false;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// 4-D / 5-D tile loads global -> shared; completion is signalled on `bar`
// as transaction bytes. `map` is the generic address of a CUtensorMap held
// in kernel-parameter (grid-constant) memory. Coordinate 0 is the innermost.
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const void *map, uint32_t bar, int c0, int c1, int c2,
                                            int c3) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(uint32_t dst, const void *map, uint32_t bar, int c0, int c1, int c2,
                                            int c3, int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_prefetch_map(const void *map) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(map) : "memory");
}

}  // namespace dev
}  // namespace plqcd
