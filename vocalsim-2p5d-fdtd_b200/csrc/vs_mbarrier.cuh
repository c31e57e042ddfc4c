// vs_mbarrier.cuh -- mbarrier, bulk-copy and cluster-store helpers for
// sm_100a (inline PTX), shared by the step kernels and the cluster kernel.
// Every wait is bounded: a caller that runs out of polls reports
// VS_ERR_TIMEOUT instead of spinning on.
#pragma once

#include <cstdint>

#include "vs_device.h"

namespace vsb {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
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

// global -> shared bulk copy (no multicast); dst, src 16-byte aligned, bytes % 16 == 0
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Bounded wait on phase 0 of an mbarrier: gives up after `limit` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, 0)) return true;
    return false;
}

constexpr uint32_t kWaitPolls = 1u << 22;

// Poll limit of the waits whose expiry ends the launch with VS_ERR_TIMEOUT.
__device__ __forceinline__ uint32_t first_wait_limit(const RunState* rs) {
    const uint32_t w = rs->wait_polls;
    return w ? w : kWaitPolls;
}

// Bounded wait on the phase with the given parity.
__device__ __forceinline__ bool mbar_wait_parity_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// ---- stores into another CTA of the cluster --------------------------------
// Address of the same shared-memory location in cluster CTA `rank`.
__device__ __forceinline__ uint32_t cluster_addr(const void* local, int rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(smem_u32(local)), "r"(rank));
    return r;
}

// Asynchronous stores into a cluster CTA's shared memory whose bytes count
// against that CTA's mbarrier `bar` (both cluster addresses): the receiver
// learns of their arrival from the mbarrier phase, the sender issues no fence.
__device__ __forceinline__ void st_async_v2(uint32_t addr, float a, float b, uint32_t bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.b32 [%0], {%1, %2}, [%3];" ::"r"(addr),
                 "r"(__float_as_uint(a)), "r"(__float_as_uint(b)), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void st_async_b32(uint32_t addr, float a, uint32_t bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b32 [%0], %1, [%2];" ::"r"(addr),
                 "r"(__float_as_uint(a)), "r"(bar)
                 : "memory");
}

}  // namespace vsb
