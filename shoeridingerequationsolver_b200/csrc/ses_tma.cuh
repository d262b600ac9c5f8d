// Asynchronous tile movement for the pipelined passes: mbarriers, TMA tensor
// loads (cp.async.bulk.tensor) and 1D bulk copies (cp.async.bulk), hand-written
// PTX for sm_100a.  No multicast is used anywhere.
//
// Every wait is bounded: mbar_wait gives up after ~2 s of clock64 time and
// reports failure; callers then abort the CTA collectively, record an error
// word the host reads, and drain their own copies with another bounded wait.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace sesk {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// make initialised barriers visible to the async (TMA) proxy
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// order this thread's generic-proxy shared-memory accesses before later
// async-proxy (TMA) writes to the same addresses
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

constexpr long long kWaitLimitCycles = 4000000000LL;  // ~2 s at the B200's SM clock

// Wait until phase `parity` of the barrier completes, at most `limit` SM clock
// cycles (<= 0: ~2 s).
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, long long limit = 0) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long lim = limit > 0 ? limit : kWaitLimitCycles;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > lim) return false;
    }
    return true;
}

// 1D bulk copy global -> shared; src, dst 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar)
        : "memory");
}

// Tiled TMA loads (no multicast).  Innermost coordinate c0 counts 8-byte
// words and is always a multiple of 2 (16-byte aligned start).
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int c0, int c1,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];" ::"r"(dst),
        "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
        : "memory");
}

}  // namespace sesk
