// Shared numerics of the 2D update: model coefficients, the Philox counter
// generator, the Q5.27 aggregate encoding, the shape-class table and the
// per-pixel right-hand side. Host and device use the same definitions.
//
// Contract sources in the reference (behaviour restated here, not copied):
//   coefficients      common/model_coefficients.cuh:23-53
//   Philox4x32-10     common/philox.cuh:32-67
//   Q5.27             include/params.cuh:94-111
//   shape classes     include/params.cuh:121-242
//   RHS               include/kernels.cuh:121-138
#pragma once

#include <cstdint>
#include <cmath>

#include "../../include/pfb200.h"

#if defined(__CUDACC__)
#define PFB_HD __host__ __device__
#define PFB_INLINE __forceinline__
#else
#define PFB_HD
#define PFB_INLINE inline
#endif

namespace pfb {

constexpr double kPi = 3.14159265358979323846;
// Allen-Cahn mobility the coefficient helpers already include (M0 = 1/2).
constexpr double kMobilityM0 = 0.5;

// ---- model coefficients (Palmieri et al. 2015, Eq. S15, M = 1/2 folded) --
// dphi/dt = g*lap - (30/l^2) g phi(1-phi)(1-2phi) + (2 mu/A0)(A0-V) phi
//           - (60 k/l^2) phi S_other - v.grad(phi)
// v = v_A p + (60 k / (xi l^2)) * int phi grad(phi) S_other
template <typename T> PFB_HD constexpr T coeff_bulk(T lambda) {
    return T(30) / (lambda * lambda);
}
template <typename T> PFB_HD constexpr T coeff_interaction(T kappa, T lambda) {
    return T(60) * kappa / (lambda * lambda);
}
template <typename T> PFB_HD constexpr T coeff_motility(T kappa, T xi, T lambda) {
    return coeff_interaction(kappa, lambda) / xi;
}
template <typename T> PFB_HD constexpr T coeff_volume(T mu, T target) {
    return T(2) * mu / target;
}
// Interface steepness k = sqrt(7.5)/lambda of phi = (1 - tanh(k d))/2.
template <typename T> PFB_HD PFB_INLINE T iface_k(T lambda) {
    return T(2.7386127875258306) / lambda;
}
// Seeded radius shifted by 1/(2k) so that integral(phi^2) = pi R^2.
template <typename T> PFB_HD PFB_INLINE T seed_radius(T radius, T lambda) {
    return radius + T(0.5) / iface_k(lambda);
}

// ---- Philox4x32-10 (Salmon et al., SC'11) ------------------------------
struct Words4 {
    uint32_t w[4];
};

PFB_HD PFB_INLINE uint32_t mul_hi_u32(uint32_t a, uint32_t b) {
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * (uint64_t)b) >> 32);
#endif
}

// Ten rounds; the key is bumped by the Weyl constants before every round
// after the first.
PFB_HD PFB_INLINE Words4 philox10(uint32_t x0, uint32_t x1, uint32_t x2,
                                  uint32_t x3, uint32_t key0, uint32_t key1) {
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        if (r != 0) {
            key0 += 0x9E3779B9u;
            key1 += 0xBB67AE85u;
        }
        const uint32_t m0 = 0xD2511F53u, m1 = 0xCD9E8D57u;
        const uint32_t a_hi = mul_hi_u32(m0, x0), a_lo = m0 * x0;
        const uint32_t b_hi = mul_hi_u32(m1, x2), b_lo = m1 * x2;
        const uint32_t y0 = b_hi ^ x1 ^ key0;
        const uint32_t y2 = a_hi ^ x3 ^ key1;
        x0 = y0;
        x1 = b_lo;
        x2 = y2;
        x3 = a_lo;
    }
    Words4 out;
    out.w[0] = x0;
    out.w[1] = x1;
    out.w[2] = x2;
    out.w[3] = x3;
    return out;
}

// [0,1) from the top 53 bits of the 64-bit word (hi:lo).
PFB_HD PFB_INLINE double u53(uint32_t hi, uint32_t lo) {
    const uint64_t bits = (((uint64_t)hi << 32) | (uint64_t)lo) >> 11;
    return (double)bits * 0x1.0p-53;
}

// Counter domains of the 2D initial-condition draws.
constexpr uint32_t kDomainJitter = 1u;
constexpr uint32_t kDomainPolarity = 2u;
constexpr uint32_t kDomainSpeed = 3u;
// Fourth counter word of the per-step tumble draw.
constexpr uint32_t kTumbleTag = 0xA5A5A5A5u;

// ---- Q5.27 aggregate ------------------------------------------------------
constexpr float kQScale = 134217728.0f;        // 2^27
constexpr float kQInv = 7.45058059692382812e-09f;  // 2^-27
constexpr double kQInvD = 7.45058059692382812e-09;
constexpr float kPhiSqCap = 4.0f;

// round-to-nearest-even of min(phi*phi, 4) * 2^27 as u32; the square is one
// rounded multiply (no contraction with the scale).
PFB_HD PFB_INLINE uint32_t q_encode(float phi) {
#if defined(__CUDA_ARCH__)
    const float sq = fminf(__fmul_rn(phi, phi), kPhiSqCap);
    return __float2uint_rn(__fmul_rn(sq, kQScale));
#else
    volatile float sq = phi * phi;  // volatile: no host contraction
    const float s = sq < kPhiSqCap ? (float)sq : kPhiSqCap;  // NaN -> 4, as fminf
    return (uint32_t)std::lrint(s * kQScale);
#endif
}

// Support threshold of the bounding box.
constexpr float kSupportEps = 1e-5f;

// ---- fixed tile and shape classes ---------------------------------------
constexpr int kTilePitch = PFB_TILE_PITCH;
constexpr int kTileArea = PFB_TILE_AREA;
constexpr int kNumClasses = PFB_NUM_CLASSES;
constexpr int kClassFallback = 5;
constexpr int kClassLargest = 4;

struct Window {
    int wx, wy, tx0, ty0;
};

// Window size and origin inside the 288^2 tile of each class: round, wide,
// tall, larger square, large (phi staged, S global in the reference), and the
// 286^2 fallback that leaves a one-pixel zero ring.
PFB_HD constexpr Window window_of(int c) {
    return c == 1   ? Window{176, 144, 32, 64}
           : c == 2 ? Window{144, 176, 64, 32}
           : c == 3 ? Window{160, 160, 32, 32}
           : c == 4 ? Window{224, 224, 32, 32}
           : c == 5 ? Window{286, 286, 1, 1}
                    : Window{144, 144, 64, 64};
}

// Hysteresis of the class choice: promote when extent + 8 exceeds the window;
// demote into a smaller class only with 20 px slack, after 200 checks.
constexpr int kPromoteSlack = 8;
constexpr int kDemoteSlack = 20;
constexpr int kDemoteDwell = 200;
constexpr int kMaxShift = 4;

// Smallest lattice side this build accepts: the class-0 window must fit.
// Sides up to 286 (which the reference refuses: its largest window is 286)
// use only the classes whose window fits the side (a window never overlaps
// itself on the periodic lattice); above 286 every class is available and
// the choice is the reference's.
constexpr int kMinSide = 144;
PFB_HD PFB_INLINE bool class_fits(int c, int L) {
    const Window w = window_of(c);
    return w.wx <= L && w.wy <= L;
}

// Smallest-area class fitting the side L whose window holds (ex + slack,
// ey + slack); -1 if none.
PFB_HD PFB_INLINE int smallest_class_holding(int ex, int ey, int slack, int L) {
    int best = -1, best_area = 0;
    for (int c = 0; c < kNumClasses; ++c) {
        const Window w = window_of(c);
        if (ex + slack <= w.wx && ey + slack <= w.wy && w.wx <= L && w.wy <= L) {
            const int area = w.wx * w.wy;
            if (best < 0 || area < best_area) {
                best = c;
                best_area = area;
            }
        }
    }
    return best;
}

// ---- the per-pixel right-hand side ----------------------------------------
// The operation order is kept identical to the reference expression so that
// the same compiler contracts it the same way; mrel == 1 is the default path
// without a multiply by one (advection always stays outside the mobility).
PFB_HD PFB_INLINE float rhs_pixel(float lap, float phi, float s_other, float gx,
                                  float gy, float gam, float dwC, float volC,
                                  float repC, float vx, float vy, float mrel) {
    if (mrel == 1.0f) {
        return gam * lap - dwC * (phi * (1.0f - phi) * (1.0f - 2.0f * phi)) +
               volC * phi - repC * phi * s_other - (vx * gx + vy * gy);
    }
    return mrel * (gam * lap - dwC * (phi * (1.0f - phi) * (1.0f - 2.0f * phi)) +
                   volC * phi - repC * phi * s_other) -
           (vx * gx + vy * gy);
}

#if defined(__CUDACC__)
// rhs_pixel without the branch on mrel: for mrel == 1 the product mrel * X
// is X exactly, so both forms of rhs_pixel give the same value.
__device__ __forceinline__ float rhs_pixel_m(float lap, float phi, float s_other, float gx,
                                             float gy, float gam, float dwC, float volC,
                                             float repC, float vx, float vy, float mrel) {
    return mrel * (gam * lap - dwC * (phi * (1.0f - phi) * (1.0f - 2.0f * phi)) +
                   volC * phi - repC * phi * s_other) -
           (vx * gx + vy * gy);
}
#endif

// Nine-point isotropic Laplacian (4 edges + diagonals - 20 centre) / 6, h=1.
PFB_HD PFB_INLINE float lap9(float nW, float nC, float nE, float cW, float cC,
                             float cE, float sW, float sC, float sE) {
    return (4.0f * (nC + sC + cE + cW) + 1.0f * (nE + nW + sE + sW) +
            (-20.0f) * cC) *
           (float)(1.0 / 6.0);
}

}  // namespace pfb
