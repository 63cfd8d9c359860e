// Shared-memory ring of whole brick planes for the 3D kernels.
//
// A brick plane (B x B values of the pool's storage type T, x fastest) is
// contiguous in HBM, so one bulk asynchronous copy (cp.async.bulk, no
// multicast) stages it; a plane that stands for the zero halo is written with
// zeros by the CTA instead. Slot
// j of the ring serves requests k = j, j + R, j + 2R, ...; request k waits
// on the slot's mbarrier with parity (k / R) & 1.
//
// Usage contract (all threads of the CTA): issue() requests in increasing k,
// never more than R ahead of the oldest request still being read, and with a
// __syncthreads() between the last read of a slot and its reissue, and
// between a zero fill and its first read.
#pragma once

#include <cstdint>

#include "device_util.cuh"

namespace pfb {
namespace p3 {

// Bounded polls of a staged-plane wait (each poll suspends the thread for a
// hardware-defined interval).
constexpr uint32_t kPlaneWaitPolls = 1u << 24;

template <int R, typename T = float>
struct PlaneRing {
    T* base;          // R * plane_words values, 16-byte aligned
    uint64_t* bars;   // R mbarriers
    int plane_words;  // B * B

    __device__ __forceinline__ T* slot(int k) const {
        return base + (size_t)(k % R) * (size_t)plane_words;
    }

    // Thread 0 initialises the barriers; the caller synchronises the CTA.
    __device__ __forceinline__ void init() const {
        if (threadIdx.x == 0)
            for (int j = 0; j < R; ++j) dev::mbar_init(&bars[j], 1);
    }

    // Request k: local plane `src` of `field` (src < 0: a zero plane).
    __device__ __forceinline__ void issue(int k, const T* field, int src) const {
        T* dst = slot(k);
        uint64_t* bar = &bars[k % R];
        if (src >= 0) {
            if (threadIdx.x == 0) {
                const uint32_t bytes = (uint32_t)plane_words * (uint32_t)sizeof(T);
                // earlier generic-proxy writes to this slot precede the copy
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                dev::mbar_arrive_expect_tx(bar, bytes);
                dev::bulk_g2s(dst, field + (size_t)src * (size_t)plane_words, bytes, bar);
            }
        } else {
            float4* d4 = reinterpret_cast<float4*>(dst);
            const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
            const int n4 = plane_words * (int)sizeof(T) / 16;
            for (int i = threadIdx.x; i < n4; i += blockDim.x) d4[i] = z;
            if (threadIdx.x == 0) dev::mbar_arrive_expect_tx(bar, 0u);
        }
    }

    // Wait for request k; false after the poll limit.
    __device__ __forceinline__ bool wait(int k) const {
        return dev::mbar_wait_bounded(&bars[k % R], (uint32_t)((k / R) & 1), kPlaneWaitPolls);
    }
};

}  // namespace p3
}  // namespace pfb
