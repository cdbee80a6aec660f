// Tensor-memory-access (TMA) loads and shared-memory barriers (sm_90+ PTX).
//
// Tiles of global arrays are copied into shared memory by one
// cp.async.bulk.tensor instruction each, issued by one thread; completion is
// tracked by an mbarrier whose transaction count the copies decrement.  Only
// plain (non-multicast) loads from this GPU's own memory are used.  Every wait
// is bounded: after g_bld_wait_limit clock cycles (BLD_WAIT_CYCLES unless the
// host set another limit with bld_set_wait_limit) the waiting thread gives up
// and the kernel reports BLD_FLAG_TIMEOUT through its per-member flag.
#pragma once

#include <cuda.h>
#include <cstdint>

#define BLD_WAIT_CYCLES (1LL << 31)   // about one second at the B200's clocks
#define BLD_FLAG_NONFINITE 1
#define BLD_FLAG_TIMEOUT 2

// limit of the kernels' waits for their own TMA copies, in clock cycles; 0 makes
// every such wait give up at once (a diagnostic setting: the kernels then take
// their timeout exit with no copy missing)
__device__ long long g_bld_wait_limit = BLD_WAIT_CYCLES;

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes generic-proxy shared-memory accesses (barrier initialisation, reads of a
// buffer about to be refilled) ordered before later async-proxy (TMA) accesses
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n"
        " .reg .pred p;\n"
        " mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// waits for the phase `parity` of `bar` to complete; false after `limit` cycles
// (at once for limit <= 0)
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, long long limit = BLD_WAIT_CYCLES) {
    if (limit <= 0) return false;
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}

// 4-d tiled TMA load of the box at coordinates (c0, c1, c2, c3) into `dst`
// (128-byte aligned shared memory); completes `bar`'s transaction count
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

// 2-d and 3-d tiled TMA loads, as tma_load_4d
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int c0, int c1, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, "
        "%4}], [%5];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
    asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// 1-d bulk copy of `bytes` (a multiple of 16, both addresses 16-byte aligned)
// from global memory into shared memory; completes `bar`'s transaction count
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(__cvta_generic_to_global(src)), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}
