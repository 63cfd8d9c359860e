// Phi pool access of the 3D kernels for the storage types of storage2d.cuh:
// binary32 (the reference's layout) or binary16 / bfloat16 with binary32
// arithmetic. Loads widen to binary32; a 16-bit store rounds stochastically
// with bits drawn from a hash of (seed, step, cell, voxel), and every
// quantity derived from a stored value (the Q5.27 scatter, the support and
// clamp tests, the next step's moments) uses the rounded value.
#pragma once

#include <cstdint>

#include "storage2d.cuh"

namespace pfb {
namespace p3 {

template <typename T>
__device__ __forceinline__ float phi_ld1(const T* p) {
    if constexpr (!Store<T>::kHalf)
        return *p;
    else
        return Store<T>::value(*reinterpret_cast<const uint16_t*>(p));
}

// four consecutive values from a 4-value aligned address
template <typename T>
__device__ __forceinline__ void phi_ld4(const T* p, float* v) {
    if constexpr (!Store<T>::kHalf) {
        const float4 m = *reinterpret_cast<const float4*>(p);
        v[0] = m.x;
        v[1] = m.y;
        v[2] = m.z;
        v[3] = m.w;
    } else {
        const uint2 u = *reinterpret_cast<const uint2*>(p);
        v[0] = Store<T>::value((uint16_t)(u.x & 0xFFFFu));
        v[1] = Store<T>::value((uint16_t)(u.x >> 16));
        v[2] = Store<T>::value((uint16_t)(u.y & 0xFFFFu));
        v[3] = Store<T>::value((uint16_t)(u.y >> 16));
    }
}

// Stochastic-rounding stream of one cell and step.
__device__ __forceinline__ uint32_t sr_stream(uint64_t step, int64_t gid, uint64_t seed) {
    return mix32((uint32_t)step * 0x85EBCA6Bu ^ (uint32_t)gid * 0xC2B2AE35u ^ (uint32_t)seed);
}

// Value (and bits) a store of v at brick voxel `pix` holds.
template <typename T>
__device__ __forceinline__ float phi_round(float v, uint32_t sr, uint32_t pix, uint16_t* bits) {
    if constexpr (!Store<T>::kHalf) {
        return v;
    } else {
        *bits = Store<T>::bits(v, mix32(sr ^ (pix * 0x9E3779B9u)));
        return Store<T>::value(*bits);
    }
}

// Streaming store of four values (rounded already; bits of a 16-bit pool).
template <typename T>
__device__ __forceinline__ void phi_st4(T* o, const float* v, const uint16_t* b) {
    if constexpr (!Store<T>::kHalf) {
        __stcs(reinterpret_cast<float4*>(o), make_float4(v[0], v[1], v[2], v[3]));
    } else {
        __stcs(reinterpret_cast<uint2*>(o), make_uint2((uint32_t)b[0] | ((uint32_t)b[1] << 16),
                                                       (uint32_t)b[2] | ((uint32_t)b[3] << 16)));
    }
}

}  // namespace p3
}  // namespace pfb
