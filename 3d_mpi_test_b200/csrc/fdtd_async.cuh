// sm_100a asynchronous-copy primitives used by the staged fused pass:
// 1D bulk copies global -> shared (cp.async.bulk, the TMA unit's untiled
// form) completing on a shared-memory mbarrier with a transaction count.
// Only this GPU's own global memory is ever a source; no multicast form is
// used anywhere.
#pragma once

#include <cstdint>

namespace fdtd {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make barrier initialisation visible to the async proxy (the bulk-copy unit)
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// order this thread's earlier shared-memory accesses (and those made
// visible to it by a barrier) before its later async-proxy writes
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// dst, src 16-byte aligned; bytes a multiple of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// hint: bring [p, p + bytes) of this GPU's global memory into L2 (p 16-byte
// aligned, bytes a multiple of 16); no completion to wait for
__device__ __forceinline__ void bulk_prefetch_l2(const void* p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase with the given parity: gives up after `spin`
// polls (each poll may suspend the thread for a while; 0 polls gives up at
// once), so a copy that never lands cannot hang the kernel; the caller
// records the failure.
constexpr long long kMbarSpin = 1LL << 22;

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long spin = kMbarSpin) {
    for (long long it = 0; it < spin; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace fdtd
