// Shared numerics and index maps of the 3D update: brick geometry, the
// 27-point stencil order, the 3D Q5.27 encoding, boundary z maps, sticky
// flags and the Philox counter domains of the 3D draws. Host and device use
// the same definitions.
//
// Contract sources in the reference (behaviour restated here, not copied):
//   stencil weights and order  include/pf3d/params.cuh:66-79,
//                              src/pf3d/device_common.cuh:218-245
//   q_of (NaN maps to 0)       include/pf3d/params.cuh:88-100
//   z maps (slab, channel)     src/pf3d/device_common.cuh:125-154,
//                              include/pf3d/bounded_z_map.hpp:14-64
//   Philox domains             include/pf3d/rng.cuh:35-150
//   recentring, support check  src/pf3d/kernels.cu:397-497
#pragma once

#include <cstdint>
#include <cmath>

#include "../../include/pfb200_3d.h"
#include "pfb_common.cuh"

namespace pfb {
namespace p3 {

constexpr int kBrickAlign = 8;
// Adaptive bricks: a grown cube adds kBrickGrowth planes, rounded up to a
// multiple of kBrickTier; a crop keeps kBrickShrinkSpare spare planes beyond
// the support on every face; compaction runs every kBrickCompactEvery
// accepted steps. Promoted cubes are at most kMaxPromotedEdge voxels wide.
constexpr int kBrickGrowth = 32;
constexpr int kBrickTier = 16;
constexpr int kBrickShrinkSpare = 16;
constexpr long long kBrickCompactEvery = 1024;
constexpr int kMaxPromotedEdge = 1024;
constexpr float kSupportEps3 = 1.0e-5f;
constexpr double kSafetyMargin = 8.0;
constexpr int kMaxShift3 = 4;
constexpr float kQClamp3 = 4.0f;

// 27-point Laplacian weights by the number of non-zero offsets.
constexpr int kWFace = 14, kWEdge = 3, kWCorner = 1, kWCentre = -128;

PFB_HD constexpr bool periodic_xyz(uint32_t b) { return b == PFB3D_BOUNDARY_PERIODIC_XYZ; }
PFB_HD constexpr bool substrate_slab(uint32_t b) { return b == PFB3D_BOUNDARY_SUBSTRATE_SLAB; }
PFB_HD constexpr bool hard_wall_channel(uint32_t b) {
    return b == PFB3D_BOUNDARY_HARD_WALL_CHANNEL;
}
PFB_HD constexpr bool bounded_z(uint32_t b) { return substrate_slab(b) || hard_wall_channel(b); }

// min(phi^2, 4) * 2^27 to nearest even as u32; a NaN square is not clamped
// and converts to 0 on the device.
PFB_HD PFB_INLINE uint32_t q_of3(float phi) {
#if defined(__CUDA_ARCH__)
    float v = __fmul_rn(phi, phi);
    if (v > kQClamp3) v = kQClamp3;
    return __float2uint_rn(__fmul_rn(v, kQScale));
#else
    volatile float sq = phi * phi;
    float v = sq;
    if (v > kQClamp3) v = kQClamp3;
    return (uint32_t)std::lrint(v * kQScale);
#endif
}

PFB_HD PFB_INLINE int wrap_origin(int64_t origin, int n) {
    if (origin >= 0 && origin < n) return (int)origin;
    if (origin < 0 && origin >= -(int64_t)n) return (int)(origin + n);
    int64_t v = origin % (int64_t)n;
    if (v < 0) v += n;
    return (int)v;
}

PFB_HD PFB_INLINE int wrap_offset(int wrapped_origin, int offset, int n) {
    int v = wrapped_origin + offset;
    if (v >= n) v -= n;
    return v;
}

PFB_HD PFB_INLINE size_t s_index(const pfb_layout3d& L, int x, int y, int z) {
    return ((size_t)z * (size_t)L.ny + (size_t)y) * (size_t)L.pitch_x + (size_t)x;
}

// World z plane of local plane `local_z` of a brick at origin_z, or false
// when it lies outside a bounded domain (periodic domains wrap).
PFB_HD PFB_INLINE bool aggregate_z(const pfb_layout3d& L, int64_t origin_z, int local_z,
                                   int* world_z) {
    if (periodic_xyz(L.boundary_flags)) {
        *world_z = wrap_offset(wrap_origin(origin_z, L.nz), local_z, L.nz);
        return true;
    }
    const int64_t w = origin_z + (int64_t)local_z;
    if (w < 0 || w >= (int64_t)L.nz) return false;
    *world_z = (int)w;
    return true;
}

// Local plane whose values stand for requested local plane `z` of a brick
// (the stencil's z neighbours): inside the brick and the domain itself;
// bounded domains reflect the ghost below world z = 0 onto plane 0 and, for
// the channel, the ghost above nz - 1 onto nz - 1; everything else is zero
// (returns false). Periodic domains use the brick's own zero halo.
PFB_HD PFB_INLINE bool fetch_plane(const pfb_layout3d& L, int64_t origin_z, int z, int B,
                                   int* source) {
    if (periodic_xyz(L.boundary_flags)) {
        if ((unsigned)z >= (unsigned)B) return false;
        *source = z;
        return true;
    }
    int64_t w = origin_z + (int64_t)z;
    if (hard_wall_channel(L.boundary_flags) && w == (int64_t)L.nz) w = L.nz - 1;
    if (w >= (int64_t)L.nz) return false;
    if (w < -1) return false;
    if (w == -1) w = 0;
    const int64_t local = w - origin_z;
    if (local < 0 || local >= (int64_t)B) return false;
    *source = (int)local;
    return true;
}

// Recentring shift limited to +-limit and to keep every supported voxel
// inside the brick after x' = x - s.
PFB_HD PFB_INLINE int clamp_shift(int proposed, int limit, int lo, int hi, int B) {
    proposed = proposed < -limit ? -limit : (proposed > limit ? limit : proposed);
    if (hi >= lo) {
        proposed = proposed < lo ? proposed : lo;
        proposed = proposed > hi - (B - 1) ? proposed : hi - (B - 1);
    }
    return proposed;
}

// ---- Philox draws of the 3D cells ------------------------------------------
constexpr uint32_t kDomainPOLI = 0x504F4C49u;  // initial polarity
constexpr uint32_t kDomainVALO = 0x56414C4Fu;  // initial active speed
constexpr uint32_t kDomainTUME = 0x54554D45u;  // tumble event
constexpr uint32_t kDomainTUMV = 0x54554D56u;  // tumble direction

struct Dir3 {
    double x, y, z;
};

PFB_HD PFB_INLINE Dir3 isotropic_dir(double axial_u, double azimuth_u) {
    const double z = 2.0 * axial_u - 1.0;
    const double r2 = 1.0 - z * z;
    const double r = sqrt(r2 > 0.0 ? r2 : 0.0);
    const double a = 2.0 * kPi * azimuth_u;
    return Dir3{r * cos(a), r * sin(a), z};
}

PFB_HD PFB_INLINE Dir3 planar_dir(double azimuth_u) {
    const double a = 2.0 * kPi * azimuth_u;
    return Dir3{cos(a), sin(a), 0.0};
}

PFB_HD PFB_INLINE Words4 draw3(uint64_t c01, uint32_t c2, uint32_t c3, uint64_t key) {
    return philox10((uint32_t)c01, (uint32_t)(c01 >> 32), c2, c3, (uint32_t)key,
                    (uint32_t)(key >> 32));
}

PFB_HD PFB_INLINE Dir3 initial_polarity3(int64_t gid, uint64_t stream, bool planar) {
    const Words4 r = draw3((uint64_t)gid, kDomainPOLI, 0u, stream);
    if (planar) return planar_dir(u53(r.w[2], r.w[3]));
    return isotropic_dir(u53(r.w[0], r.w[1]), u53(r.w[2], r.w[3]));
}

PFB_HD PFB_INLINE double initial_speed3(int64_t gid, uint64_t seed, double median,
                                        double sigma) {
    if (!(sigma > 0.0)) return median;
    const Words4 r = draw3((uint64_t)gid, kDomainVALO, 0u, seed);
    double u1 = u53(r.w[0], r.w[1]);
    if (u1 < 1.0e-300) u1 = 1.0e-300;
    const double u2 = u53(r.w[2], r.w[3]);
    const double normal = sqrt(-2.0 * log(u1)) * cos(2.0 * kPi * u2);
    return median * exp(sigma * normal);
}

// Tumble of accepted step `step` (already reduced by the aging steps): an
// event when u53 of the TUME words 0-1 is below p; the new direction takes
// its axial draw from TUME words 2-3 and its azimuth from TUMV words 0-1
// (planar: TUMV words 0-1 alone).
PFB_HD PFB_INLINE bool tumble3(uint64_t step, int64_t gid, uint64_t stream, double p,
                               bool planar, Dir3* dir) {
    const uint64_t g = (uint64_t)gid;
    const Words4 ev = draw3(step, (uint32_t)g, (uint32_t)(g >> 32) ^ kDomainTUME, stream);
    if (!(u53(ev.w[0], ev.w[1]) < p)) return false;
    const Words4 vec = draw3(step, (uint32_t)g, (uint32_t)(g >> 32) ^ kDomainTUMV, stream);
    *dir = planar ? planar_dir(u53(vec.w[0], vec.w[1]))
                  : isotropic_dir(u53(ev.w[2], ev.w[3]), u53(vec.w[0], vec.w[1]));
    return true;
}

}  // namespace p3
}  // namespace pfb
