// tma.cuh -- bulk-copy (TMA) and mbarrier helpers for sm_100a.
//
// Only non-multicast, CTA-local forms are used: cp.async.bulk from this
// GPU's global memory into the issuing CTA's shared memory, completing on an
// mbarrier of the same CTA.  Every wait is bounded: after the limit the
// waiter records an error code in a global flag and gives up, so a fault in
// the pipeline surfaces as a status on the host instead of a hung GPU.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dgpu {

// error codes written to the kernel error flag
constexpr int KERR_WAIT_TIMEOUT = 1;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
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

// Wait for phase `parity` of bar; give up after ~2^22 polls (with backoff,
// on the order of a second), recording KERR_WAIT_TIMEOUT in *err.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* err) {
    for (uint32_t it = 0; it < (1u << 22); ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(128);
    }
    atomicExch(err, KERR_WAIT_TIMEOUT);
    return false;
}

// 1-D bulk copy global -> shared (16-byte aligned, size a multiple of 16),
// completing as tx bytes on bar.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Make this thread's generic-proxy global writes visible to later bulk copies.
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

}  // namespace dgpu
