// Host helpers of the 3D path: seed-radius calibration, brick sizing and the
// per-cell Philox draws (reference include/pf3d/reference.hpp:601-745,
// include/pf3d/params.cuh:112-166, include/pf3d/rng.cuh:35-150).
#include <cmath>
#include <cstdint>
#include <limits>
#include <utility>
#include <vector>

#include "pfb3d_common.cuh"
#include "pfb_internal.h"

namespace {

// Discrete sum of phi^2 of a tanh sphere of radius `seed` centred in a brick
// of edge B (centre (B-1)/2 on every axis), in binary64.
double seeded_volume(int B, double seed, double lambda) {
    const double centre = 0.5 * (double)(B - 1);
    const double k = std::sqrt(7.5) / lambda;
    double v = 0.0;
    for (int z = 0; z < B; ++z) {
        const double dz = (double)z - centre;
        for (int y = 0; y < B; ++y) {
            const double dy = (double)y - centre;
            for (int x = 0; x < B; ++x) {
                const double dx = (double)x - centre;
                const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                const double phi = 0.5 * (1.0 - std::tanh(k * (r - seed)));
                v += phi * phi;
            }
        }
    }
    return v;
}

}  // namespace

extern "C" {

int pfb3d_calibrate_seed_radius(double radius, double lambda, int B, double* seed_radius,
                                double* measured_volume) {
    if (!(radius > 0.0) || !(lambda > 0.0) || B < 3 || !seed_radius)
        return pfb::set_error(PFB_E_ARG, "invalid seed-radius calibration request");
    const double target = 4.0 * pfb::kPi * radius * radius * radius / 3.0;
    double lo = 0.0, hi = (double)B;
    if (seeded_volume(B, lo, lambda) > target || seeded_volume(B, hi, lambda) < target)
        return pfb::set_error(PFB_E_ARG, "target volume is not bracketed by the brick");
    // bisection to a relative error of 1e-10, at most 80 halvings
    double mid = 0.0, v = 0.0;
    bool converged = false;
    for (int it = 1; it <= 80; ++it) {
        mid = 0.5 * (lo + hi);
        v = seeded_volume(B, mid, lambda);
        if (std::fabs(v - target) / target <= 1.0e-10) {
            converged = true;
            break;
        }
        if (v < target)
            lo = mid;
        else
            hi = mid;
    }
    if (!converged) return pfb::set_error(PFB_E_STATE, "seed-radius calibration did not converge");
    *seed_radius = mid;
    if (measured_volume) *measured_volume = v;
    return PFB_OK;
}

int pfb3d_automatic_brick_edge(double radius, double lambda) {
    if (!(radius > 0.0) || !(lambda > 0.0)) return -1;
    const double k = 2.7386127875258306 / lambda;
    const double eff = radius + 0.5 / k;
    const double tail = std::log(1.0 / (double)pfb::p3::kSupportEps3 - 1.0) / (2.0 * k);
    const double need = 2.0 * (eff + tail) + pfb::p3::kSafetyMargin;
    if (!std::isfinite(need) || need > (double)std::numeric_limits<int>::max() - 8) return -1;
    const int c = (int)std::ceil(need);
    return (c + pfb::p3::kBrickAlign - 1) / pfb::p3::kBrickAlign * pfb::p3::kBrickAlign;
}

void pfb3d_initial_polarity(int64_t gid, uint64_t stream, int planar, double* out3) {
    const pfb::p3::Dir3 d = pfb::p3::initial_polarity3(gid, stream, planar != 0);
    out3[0] = d.x;
    out3[1] = d.y;
    out3[2] = d.z;
}

double pfb3d_initial_active_speed(int64_t gid, uint64_t seed, double median, double sigma) {
    return pfb::p3::initial_speed3(gid, seed, median, sigma);
}

int pfb3d_soft_membership(int n, double fraction, uint64_t seed, uint8_t* out) {
    if (n < 1 || !out || !std::isfinite(fraction) || fraction < 0.0 || fraction > 1.0)
        return pfb::set_error(PFB_E_ARG, "invalid soft-cell selection parameters");
    constexpr uint32_t kDomainSoft = 0x33544653u;  // "SFT3"
    const int count = (int)std::llround(fraction * (double)n);
    std::vector<int> ids((size_t)n);
    for (int i = 0; i < n; ++i) ids[(size_t)i] = i;
    for (int i = 0; i < count; ++i) {
        // uniform in [0, n - i): reject words below 2^64 mod bound
        const uint64_t bound = (uint64_t)(n - i);
        const uint64_t threshold = (0ull - bound) % bound;
        uint64_t pick = 0;
        for (uint32_t attempt = 0;; ++attempt) {
            const pfb::Words4 r = pfb::p3::draw3((uint64_t)i, kDomainSoft, attempt, seed);
            const uint64_t word = ((uint64_t)r.w[0] << 32) | r.w[1];
            if (word >= threshold) {
                pick = word % bound;
                break;
            }
            if (attempt == 0xFFFFFFFFu) return pfb::set_error(PFB_E_STATE, "soft-cell draw did not converge");
        }
        std::swap(ids[(size_t)i], ids[(size_t)i + (size_t)pick]);
    }
    for (int i = 0; i < n; ++i) out[i] = 0;
    for (int i = 0; i < count; ++i) out[ids[(size_t)i]] = 1;
    return PFB_OK;
}

int pfb3d_tumble(uint64_t step, int64_t gid, uint64_t stream, double p, int planar, double* out3) {
    pfb::p3::Dir3 d{0.0, 0.0, 0.0};
    const bool ev = pfb::p3::tumble3(step, gid, stream, p, planar != 0, &d);
    if (ev && out3) {
        out3[0] = d.x;
        out3[1] = d.y;
        out3[2] = d.z;
    }
    return ev ? 1 : 0;
}

}  // extern "C"
