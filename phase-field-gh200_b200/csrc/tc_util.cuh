// Fifth-generation tensor-core (tcgen05) helpers for sm_100a, as inline PTX:
// shared-memory matrix descriptors, the kind::f16 instruction descriptor,
// single-CTA MMA issue and commit, tensor-memory (TMEM) allocation and
// loads, and the 16-byte cp.async staging copy used to build operand tiles.
//
// Operand tiles use the canonical no-swizzle ("interleaved") layouts, whose
// unit is a core matrix of 8 rows x 16 bytes stored contiguously (128 B):
//   K-major : rows along M (or N) at 16 B inside a core matrix; the next 8
//             rows at SBO bytes; the next 16-byte K chunk at LBO bytes.
//   MN-major: 8 consecutive M (or N) elements in 16 B; the 8 K rows of a
//             core matrix at 16 B; the next 8 M elements at SBO bytes; the
//             next 8 K rows at LBO bytes.
#pragma once

#include <cstdint>

#include "device_util.cuh"

namespace pfb {
namespace tc {

// Polls of an mbarrier before a wait gives up (each poll suspends the thread
// for a hardware-bounded interval).
constexpr uint32_t kMmaWaitPolls = 1u << 24;

// Matrix descriptor for a no-swizzle operand tile at shared address `saddr`
// (16-byte aligned): start address, leading and stride byte offsets, the
// descriptor version 1 of sm_100 at bits 46-47, base offset 0, layout 0.
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16 with bfloat16 A and B and a binary32
// accumulator: D format at bits 4-5 (1 = f32), A and B formats at bits 7-9
// and 10-12 (1 = bf16), A and B major at bits 15 and 16 (1 = MN-major),
// N / 8 at bits 17-22, M / 16 at bits 24-28.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) |
           ((b_mn ? 1u : 0u) << 16) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K = 16 slice; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc,
                                         uint32_t idesc, uint32_t accumulate) {
    const uint32_t z = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(z)
        : "memory");
}

// Arrive on `bar` once every MMA issued so far by this thread has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     dev::smem_addr(bar))
                 : "memory");
}

// Warp-collective TMEM allocation of `ncols` columns (a power of two >= 32);
// the base address is written to *slot in shared memory.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     dev::smem_addr(slot)),
                 "r"(ncols)
                 : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Make this thread's generic-proxy shared-memory writes visible to the
// tensor cores' (async proxy) operand reads.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// 16 columns (32x32b shape): lane l of warp w (w = warp index mod 4) gets
// TMEM lane 32 w + l, columns taddr.col .. +15.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// 16-byte asynchronous global->shared copy; src_bytes = 0 fills the 16 bytes
// with zeros (the source address is not read).
__device__ __forceinline__ void cp_async16(uint32_t saddr, const void* gsrc, uint32_t src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr), "l"(gsrc),
                 "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;" ::: "memory");
}

}  // namespace tc
}  // namespace pfb
