// Host-side helpers of the C ABI: error text, Philox and the Q5.27 encoder
// for binding layers, the reference's two centre initialisers, initial
// polarity and speed draws, and the step-argument coefficients.
//
// Placement follows the reference's sequential periodic initialiser
// (include/palmieri_initializer.hpp:66-103) and grid-and-jitter layout
// (src/sim.cu:107-129); this file is compiled without floating-point
// contraction so the accepted binary32 centres are reproducible.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "pfb_common.cuh"
#include "pfb_internal.h"

namespace pfb {

namespace {
thread_local char g_err[512] = {0};
}

int set_error(int code, const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

void clear_error() { g_err[0] = '\0'; }

const char* last_error() { return g_err; }

}  // namespace pfb

using namespace pfb;

extern "C" {

const char* pfb_version(void) { return "pfb200 0.1.0 (sm_100a)"; }

const char* pfb_last_error(void) { return pfb::last_error(); }

size_t pfb_sizeof(int which) {
    switch (which) {
        case 0: return sizeof(pfb_cell2d);
        case 1: return sizeof(pfb_step_args2d);
        case 2: return sizeof(pfb_params2d);
        case 3: return sizeof(pfb_traj_cell2d);
        default: return 0;
    }
}

void pfb_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                       uint32_t k1, uint32_t* out) {
    const Words4 r = philox10(c0, c1, c2, c3, k0, k1);
    if (out) std::memcpy(out, r.w, sizeof(r.w));
}

double pfb_philox_uniform53(uint32_t a, uint32_t b) { return u53(a, b); }

uint32_t pfb_q_of(float phi) { return q_encode(phi); }

static double nearest_image(double d, double side) { return d - side * std::floor(d / side + 0.5); }

int pfb_palmieri_centres(int n, double side, double min_sep, unsigned long long seed, float* x,
                         float* y) {
    if (!x || !y || n < 1 || !(side > 0.0) || !(min_sep > 0.0))
        return set_error(PFB_E_ARG, "palmieri_centres: invalid arguments");
    std::mt19937_64 rng(seed);
    x[0] = (float)(0.5 * side);
    y[0] = (float)(0.5 * side);
    int have = 1;
    unsigned long long draws = 0;
    const double r2 = min_sep * min_sep;
    while (have < n) {
        if (++draws > 1000000000ull)
            return set_error(PFB_E_ARG, "palmieri_centres: placement did not terminate");
        const double cx = side * ((double)(rng() >> 11) * 0x1.0p-53);
        const double cy = side * ((double)(rng() >> 11) * 0x1.0p-53);
        bool ok = true;
        for (int j = 0; j < have; ++j) {
            const double dx = nearest_image(cx - (double)x[j], side);
            const double dy = nearest_image(cy - (double)y[j], side);
            if (dx * dx + dy * dy < r2) {
                ok = false;
                break;
            }
        }
        if (!ok) continue;
        x[have] = (float)cx;
        y[have] = (float)cy;
        ++have;
    }
    return PFB_OK;
}

int pfb_grid_jitter_centres(int n, int side, unsigned long long seed, float* x, float* y) {
    if (!x || !y || n < 1 || side < 1) return set_error(PFB_E_ARG, "grid_jitter: invalid arguments");
    const int nx = (int)std::ceil(std::sqrt((double)n));
    const double sp = (double)side / (double)nx;
    for (int i = 0; i < n; ++i) {
        const int gxi = i % nx, gyi = i / nx;
        const Words4 r = philox10((uint32_t)i, kDomainJitter, 0u, 0u,
                                  (uint32_t)(seed & 0xFFFFFFFFull), (uint32_t)(seed >> 32));
        const double jx = (u53(r.w[0], r.w[1]) - 0.5) * 0.10 * sp;
        const double jy = (u53(r.w[2], r.w[3]) - 0.5) * 0.10 * sp;
        double px = ((double)gxi + 0.5 + ((gyi & 1) ? 0.5 : 0.0)) * sp + jx;
        double py = ((double)gyi + 0.5) * sp + jy;
        px -= std::floor(px / (double)side) * (double)side;
        py -= std::floor(py / (double)side) * (double)side;
        x[i] = (float)px;
        y[i] = (float)py;
    }
    return PFB_OK;
}

float pfb_ic_theta(int32_t gid, unsigned long long stream) {
    const Words4 r = philox10((uint32_t)gid, kDomainPolarity, 0u, 0u,
                              (uint32_t)(stream & 0xFFFFFFFFull), (uint32_t)(stream >> 32));
    return (float)(2.0 * kPi * u53(r.w[0], r.w[1]));
}

double pfb_ic_v_A(int32_t gid, unsigned long long seed, double v_A, double sigma) {
    if (!(sigma > 0.0)) return v_A;
    const Words4 r = philox10((uint32_t)gid, kDomainSpeed, 0u, 0u,
                              (uint32_t)(seed & 0xFFFFFFFFull), (uint32_t)(seed >> 32));
    double u1 = u53(r.w[0], r.w[1]);
    if (u1 < 1e-300) u1 = 1e-300;
    const double u2 = u53(r.w[2], r.w[3]);
    const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
    return v_A * std::exp(sigma * z);
}

int pfb_domain_side_for(int n, double radius, double rho) {
    const double a = (double)n * (kPi * radius * radius) / rho;
    const double side = std::ceil(std::sqrt(a));
    return (std::isfinite(side) && side >= 1.0 && side <= 2147483647.0) ? (int)side : -1;
}

int pfb_fill_coefficients2d(const pfb_params2d* p, pfb_step_args2d* a) {
    if (!p || !a) return set_error(PFB_E_ARG, "fill_coefficients2d: null");
    const double A0 = kPi * p->target_radius * p->target_radius;
    a->physical_dt = p->dt;
    a->dt = (float)p->dt;
    a->A0 = A0;
    a->vol_scale = coeff_volume(p->mu, A0);
    a->bulk_scale = (float)coeff_bulk(p->lambda);
    a->rep_coeff = (float)coeff_interaction(p->kappa, p->lambda);
    a->mot_coeff = (float)coeff_motility(p->kappa, p->xi, p->lambda);
    a->seed = p->seed;
    a->polarity_seed = p->polarity_seed ? p->polarity_seed : p->seed;
    a->p_tumble = -std::expm1(-p->dt / p->tau);
    a->full_moment_every = p->full_moment_every;
    return PFB_OK;
}

}  // extern "C"
