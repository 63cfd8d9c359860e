// Small sm_100a device helpers written as inline PTX: thread-block-cluster
// barriers and distributed shared memory, mbarriers, and the bulk (TMA)
// global->shared copy. No multicast form is used anywhere.
#pragma once

#include <cstdint>

namespace pfb {
namespace dev {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint32_t cluster_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

// Cluster-wide barrier with release/acquire semantics at cluster scope (it
// also orders this CTA's global-memory writes for the other CTAs).
__device__ __forceinline__ void cluster_sync() {
    asm volatile(
        "barrier.cluster.arrive.release.aligned;\n\t"
        "barrier.cluster.wait.acquire.aligned;" ::
            : "memory");
}

// Split cluster barrier without memory ordering: enough to publish mbarrier
// initialisation (after fence.mbarrier_init) before peers signal them.
__device__ __forceinline__ void cluster_arrive_relaxed() {
    asm volatile("barrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
    asm volatile("barrier.cluster.wait.aligned;" ::: "memory");
}

// Asynchronous stores into a peer CTA's shared memory that complete on the
// peer's mbarrier (addresses from map_to_rank).
__device__ __forceinline__ void st_async_v2f64(uint32_t addr, double a, double b, uint32_t bar) {
    asm volatile(
        "st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(
            addr),
        "d"(a), "d"(b), "r"(bar)
        : "memory");
}
__device__ __forceinline__ void st_async_v4b32(uint32_t addr, int a, int b, int c, int d,
                                               uint32_t bar) {
    asm volatile(
        "st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.b32 [%0], {%1, %2, %3, %4}, "
        "[%5];" ::"r"(addr),
        "r"(a), "r"(b), "r"(c), "r"(d), "r"(bar)
        : "memory");
}

// Address of the same shared-memory variable in CTA `rank` of the cluster.
__device__ __forceinline__ uint32_t map_to_rank(uint32_t saddr, uint32_t rank) {
    uint32_t r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
                 : "=r"(r)
                 : "r"(saddr), "r"(rank));
    return r;
}

__device__ __forceinline__ double ld_cluster_f64(uint32_t addr) {
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
    return v;
}

__device__ __forceinline__ double2 ld_cluster_v2f64(uint32_t addr) {
    double2 v;
    asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];"
                 : "=d"(v.x), "=d"(v.y)
                 : "r"(addr)
                 : "memory");
    return v;
}

__device__ __forceinline__ int4 ld_cluster_v4s32(uint32_t addr) {
    int4 v;
    asm volatile("ld.shared::cluster.v4.s32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr)
                 : "memory");
    return v;
}

// Sum over lanes 0..n-1 of v in ascending lane order, result in every lane
// (a fixed order, so the result does not depend on timing).
__device__ __forceinline__ double ordered_lane_sum(double v, int n) {
    double s = 0.0;
    for (int l = 0; l < n; ++l) s += __shfl_sync(0xFFFFFFFFu, v, l);
    return s;
}

__device__ __forceinline__ int ld_cluster_s32(uint32_t addr) {
    int v;
    asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}

// ---- mbarrier ---------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
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

// Bounded wait: returns false after `limit` unsuccessful polls (each poll
// suspends the thread for a hardware-defined interval).
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity,
                                                  uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Bulk asynchronous copy of `bytes` (multiple of 16) from global to this CTA's
// shared memory, completing on `bar`. Both addresses 16-byte aligned.
__device__ __forceinline__ void bulk_g2s(void* dst_smem, const void* src_gmem, uint32_t bytes,
                                         uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// ---- L2 eviction-priority policies -------------------------------------------
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Bulk copy as bulk_g2s, with an L2 eviction-priority policy for the source.
__device__ __forceinline__ void bulk_g2s_hint(void* dst_smem, const void* src_gmem,
                                              uint32_t bytes, uint64_t* bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint "
        "[%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

// 16-byte global store with an L2 eviction-priority policy.
__device__ __forceinline__ void st_global_v4_hint(float4* p, float4 v, uint64_t policy) {
    asm volatile("st.global.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p),
                 "f"(v.x), "f"(v.y), "f"(v.z), "f"(v.w), "l"(policy)
                 : "memory");
}

// atomicAdd of v to *p issued as one predicated instruction when v != 0
// (adding zero is skipped, as a branch around atomicAdd would); returns the
// previous value, or 0 when nothing was added. Only S scatter targets are
// passed here, which the calling pass does not otherwise read.
__device__ __forceinline__ uint32_t atom_add_nonzero(uint32_t* p, uint32_t v) {
    uint32_t old;
    asm volatile(
        "{\n\t.reg .pred nz;\n\t"
        "setp.ne.u32 nz, %2, 0;\n\t"
        "mov.u32 %0, 0;\n\t"
        "@nz atom.global.add.u32 %0, [%1], %2;\n\t}"
        : "=r"(old)
        : "l"(p), "r"(v));
    return old;
}

// ---- warp reductions (fixed butterfly-down order) ------------------------
__device__ __forceinline__ double warp_sum_down(double v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, d);
    return v;
}
__device__ __forceinline__ int warp_min_down(int v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = min(v, __shfl_down_sync(0xFFFFFFFFu, v, d));
    return v;
}
__device__ __forceinline__ int warp_max_down(int v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = max(v, __shfl_down_sync(0xFFFFFFFFu, v, d));
    return v;
}

}  // namespace dev
}  // namespace pfb
