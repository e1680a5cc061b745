// tma.cuh -- tensor-memory-accelerator (cp.async.bulk.tensor) tile loads with
// mbarrier completion, for sm_100a.
//
// Rules kept by every caller: the box's innermost coordinate times the element
// size is a multiple of 16 bytes (checked on the host before any launch), the
// shared destination is 128-byte aligned, the tensor maps live in kernel
// parameter space (__grid_constant__), and every wait on an mbarrier is
// bounded: after TMA_SPIN_LIMIT polls the kernel records an error code and
// gives up instead of spinning for ever.
#pragma once

#include <cuda.h>
#include <stdint.h>

namespace ns3d {

constexpr unsigned TMA_SPIN_LIMIT = 1u << 24;  // polls of mbarrier.try_wait (seconds at most)
constexpr int NS3D_DEVERR_TMA_TIMEOUT = 1;      // value written to the device error word

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the barrier initialisation visible to the async (TMA) proxy
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// true once the phase with the given parity has completed
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    uint32_t done;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// bounded wait; false (and the error word set) when the limit ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, int *err,
                                                  unsigned limit = TMA_SPIN_LIMIT) {
    for (unsigned it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicExch(err, NS3D_DEVERR_TMA_TIMEOUT);
    return false;
}

// After a timed-out wait: the copies already issued may still land in this
// block's shared memory, so the block waits for them (bounded by a longer
// limit) before it retires, and issues nothing more.
constexpr unsigned TMA_DRAIN_LIMIT = 1u << 26;
__device__ __forceinline__ bool mbar_drain(uint64_t *bar, unsigned parity) {
    for (unsigned it = 0; it < TMA_DRAIN_LIMIT; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// order this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) writes to the same memory
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// 3-D tiled load of one box into shared memory, completing on bar
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
            smem_u32(dst)),
        "l"((uint64_t)(uintptr_t)map), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace ns3d
