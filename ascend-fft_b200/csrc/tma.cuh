// Bulk-copy (TMA), mbarrier and thread-block-cluster helpers for sm_100a, inline PTX.
//
// Copies: the untiled bulk copy of one contiguous span (both addresses 16-byte aligned, size a
// multiple of 16 bytes) and the 2-D tiled tensor copy (tensor map built on the host; the
// innermost coordinate times the element size is a multiple of 16 bytes, the shared-memory
// destination 128-byte aligned).  Both complete transactions on an mbarrier (below its
// 2^20 - 1 byte limit).  No multicast form is used anywhere.  Every wait is bounded: a wait
// that has not completed after kWaitNs of %globaltimer (or kWaitIters polls) reports failure
// so the kernel can record an error and leave instead of hanging.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace bfly {
namespace dev {

constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s
constexpr uint32_t kWaitIters = 1u << 26;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Order this thread's earlier generic-proxy shared-memory accesses before later async-proxy
// (TMA) accesses to the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Contiguous global -> shared bulk copy completing `bytes` transactions on `bar`.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for phase `parity` of `bar`; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    const uint64_t t0 = global_timer_ns();
    for (uint32_t i = 0; i < kWaitIters; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255u) == 255u && global_timer_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

// try_wait with cluster-scope acquire: the phase was completed by st.async writes of other
// CTAs of the cluster, whose data must be visible to this thread afterwards.
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ bool mbar_wait_cluster_bounded(uint64_t* bar, uint32_t parity) {
    const uint64_t t0 = global_timer_ns();
    for (uint32_t i = 0; i < kWaitIters; ++i) {
        if (mbar_try_wait_cluster(bar, parity)) return true;
        if ((i & 255u) == 255u && global_timer_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

// 2-D tiled tensor copy global -> this CTA's shared memory (no multicast): box origin
// (x, y) in elements of the tensor map, completion counted on `bar`.
__device__ __forceinline__ void tensor_load_2d(void* dst, const void* tmap, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];" ::"r"(smem_addr(dst)),
        "l"(tmap), "r"(x), "r"(y), "r"(smem_addr(bar))
        : "memory");
}

// ------------------------------------------------------------------ thread-block clusters
__device__ __forceinline__ uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Split cluster barrier: arrive (release: this thread's earlier memory accesses are ordered
// before the barrier) ... wait (acquire).  Every thread of the cluster alternates them.
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire;" ::: "memory"); }

// Address of the same shared-memory location in CTA `rank` of this cluster.
__device__ __forceinline__ uint32_t cluster_map(uint32_t saddr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
    return r;
}

// Asynchronous 8-byte store into another CTA's shared memory that completes 8 transaction
// bytes on that CTA's mbarrier (both addresses from cluster_map).  The sender does not wait.
__device__ __forceinline__ void st_async_f2(uint32_t raddr, float2 v, uint32_t rbar) {
    // No "memory" clobber: ordering against this CTA's other accesses comes from the cluster
    // barrier and mbarrier waits around the sends, which carry one.
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];" ::"r"(raddr),
                 "f"(v.x), "f"(v.y), "r"(rbar));
}

}  // namespace dev
}  // namespace bfly
