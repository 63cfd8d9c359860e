// Storage types of the phi pools of the 2D step: binary32 (the reference's
// layout) or 16-bit (binary16 / bfloat16) with binary32 arithmetic.
//
// A 16-bit pool rounds every stored value stochastically: the value is
// rounded up with probability equal to its distance from the lower
// neighbour in ulps, using 13 (binary16) or 16 (bfloat16) pseudo-random bits
// added below the kept mantissa before truncation. Round-to-nearest would
// drop the per-step Euler increments (about 1e-6 to 1e-5, below one ulp at
// phi ~ 0.5: 2.4e-4 for binary16, 2e-3 for bfloat16) and freeze interface
// motion; stochastic rounding keeps them in expectation. binary16 values in
// its subnormal range (|phi| < 2^-14) are rounded to nearest. The bits come
// from an integer hash of (seed, step, cell, pixel), so runs are
// reproducible. Every quantity derived from the stored field (moments, the
// Q5.27 scatter, the support box) is computed from the rounded value.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

namespace pfb {

enum PhiStorage { kStoreF32 = 0, kStoreF16 = 1, kStoreBF16 = 2 };

// 32-bit integer finaliser (a published xor-shift-multiply mix).
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7FEB352Du;
    x ^= x >> 15;
    x *= 0x846CA68Bu;
    x ^= x >> 16;
    return x;
}

template <typename T>
struct Store;

template <>
struct Store<float> {
    static constexpr bool kHalf = false;
    __device__ static __forceinline__ float round(float v, uint32_t) { return v; }
    __device__ static __forceinline__ float encode(float v) { return v; }
};

template <>
struct Store<__half> {
    static constexpr bool kHalf = true;
    // stochastically rounded value, as binary16 bits
    __device__ static __forceinline__ uint16_t bits(float v, uint32_t r) {
        if (fabsf(v) >= 6.103515625e-05f && fabsf(v) < 65504.0f) {
            const float t = __uint_as_float(__float_as_uint(v) + (r & 0x1FFFu));
            return __half_as_ushort(__float2half_rz(t));
        }
        return __half_as_ushort(__float2half_rn(v));
    }
    __device__ static __forceinline__ float value(uint16_t b) {
        return __half2float(__ushort_as_half(b));
    }
};

template <>
struct Store<__nv_bfloat16> {
    static constexpr bool kHalf = true;
    __device__ static __forceinline__ uint16_t bits(float v, uint32_t r) {
        if (isfinite(v)) {
            const float t = __uint_as_float(__float_as_uint(v) + (r & 0xFFFFu));
            if (isfinite(t)) return __bfloat16_as_ushort(__float2bfloat16_rz(t));
        }
        return __bfloat16_as_ushort(__float2bfloat16_rn(v));
    }
    __device__ static __forceinline__ float value(uint16_t b) {
        return __bfloat162float(__ushort_as_bfloat16(b));
    }
};

}  // namespace pfb
