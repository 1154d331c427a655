// Tensor-memory-accelerator (TMA) staging helpers of the fused sweep, sm_100a:
// an mbarrier in shared memory, the tiled bulk tensor load
// (cp.async.bulk.tensor into the issuing CTA's own shared memory only, from a
// tensor map over this GPU's own memory) and a bounded wait on the barrier's
// phase.
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace emg {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// one arrival (the issuing thread's expect_tx) completes a phase once the
// transaction bytes have landed
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
// make the initialised barrier visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
// order this CTA's generic-proxy shared-memory accesses before later async-proxy writes
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// 4-D tiled load of one box at coordinates (c0 innermost .. c3) into shared
// memory at dst (128-byte aligned); completes tx bytes on the barrier
__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap* tm, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n"
        ".reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n"
        "}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the barrier phase with the given parity to complete, giving up
// after `limit` polls (each poll may suspend the thread for a short,
// hardware-chosen time). Returns false when it gave up.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, int limit) {
    for (int i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

constexpr int TMA_WAIT_LIMIT = 1 << 20;
constexpr int STATUS_TIMEOUT = 8;  // EMG_ERR_TIMEOUT

}  // namespace emg
