// ORACLE -- test infrastructure only. C entry points over the reference's
// dense FP64 one-step evaluation and seed-radius calibration
// (include/pf3d/reference.hpp, header-only; compiled in place by
// oracle/Makefile into oracle/_ref/libref3d_cpu.so), and the reference's
// fresh-start placements, centre-table readers and centre-table hash
// (include/palmieri_initializer.hpp, include/relaxed_centres.hpp,
// include/pf3d/palmieri_initializer.hpp, include/pf3d/initializer.hpp). The
// tests pin the 3D oracle, the placement restatement and the command lines'
// table readers against it.
#include <cstdint>
#include <cstring>
#include <exception>

#include "palmieri_initializer.hpp"
#include "relaxed_centres.hpp"
#include "pf3d/palmieri_initializer.hpp"
#include "pf3d/reference.hpp"
#include "pf3d/rng.cuh"

namespace ref = pf3d::reference;

extern "C" {

// Periodic cube of `side`, `cells` cells: phi (cells * side^3, x fastest),
// gamma/speed per cell, polarity 3 per cell. Outputs: phi_next, volume,
// integral (3 per cell), velocity (3 per cell). Returns 0, or -1 when the
// reference rejects the input.
int ref3d_cpu_one_step(int side, int cells, const double* phi, const double* gamma,
                       const double* speed, const double* polarity, double dt, double lambda,
                       double target_radius, double kappa, double mu, double xi,
                       double* phi_next, double* volume, double* integral, double* velocity) {
    try {
        ref::DenseState st;
        st.side = side;
        st.cells.resize((size_t)cells);
        for (int c = 0; c < cells; ++c) {
            st.cells[(size_t)c].gamma = gamma[c];
            st.cells[(size_t)c].active_speed = speed[c];
            st.cells[(size_t)c].polarity = ref::Vector3{polarity[3 * c], polarity[3 * c + 1],
                                                        polarity[3 * c + 2]};
        }
        st.phi.assign(phi, phi + (size_t)cells * side * side * side);
        ref::ModelParameters m;
        m.dt = dt;
        m.lambda = lambda;
        m.target_radius = target_radius;
        m.kappa = kappa;
        m.mu = mu;
        m.xi = xi;
        const ref::OneStepResult r = ref::one_euler_step(st, m);
        std::memcpy(phi_next, r.phi_next.data(), r.phi_next.size() * sizeof(double));
        for (int c = 0; c < cells; ++c) {
            volume[c] = r.volume[(size_t)c];
            integral[3 * c] = r.interaction_integral[(size_t)c].x;
            integral[3 * c + 1] = r.interaction_integral[(size_t)c].y;
            integral[3 * c + 2] = r.interaction_integral[(size_t)c].z;
            velocity[3 * c] = r.velocity[(size_t)c].x;
            velocity[3 * c + 1] = r.velocity[(size_t)c].y;
            velocity[3 * c + 2] = r.velocity[(size_t)c].z;
        }
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref3d_cpu_calibrate(double radius, double lambda, int edge, double* seed, double* measured) {
    try {
        const ref::SeedRadiusCalibration c = ref::calibrate_seed_radius(radius, lambda, edge);
        *seed = c.seed_radius;
        *measured = c.measured_volume;
        return c.converged ? 0 : 1;
    } catch (const std::exception&) {
        return -1;
    }
}

// The reference's 3D Philox draws (include/pf3d/rng.cuh:41-150).
void ref3d_cpu_initial_polarity(int64_t gid, uint64_t stream, int planar, double* out) {
    const pf3d::Vec3 v = planar ? pf3d::initial_planar_polarity(gid, stream)
                                : pf3d::initial_polarity(gid, stream);
    out[0] = v.x;
    out[1] = v.y;
    out[2] = v.z;
}

double ref3d_cpu_initial_speed(int64_t gid, uint64_t seed, double median, double sigma) {
    return pf3d::initial_active_speed(gid, seed, median, sigma);
}

int ref3d_cpu_tumble(uint64_t step, int64_t gid, uint64_t stream, double p, int planar,
                     double* out) {
    const pf3d::Vec3 cur{0.0, 0.0, 0.0};
    const pf3d::TumbleSample t = planar ? pf3d::tumble_sample_planar(step, gid, stream, p, cur)
                                        : pf3d::tumble_sample(step, gid, stream, p, cur);
    out[0] = t.polarity.x;
    out[1] = t.polarity.y;
    out[2] = t.polarity.z;
    return t.tumbled ? 1 : 0;
}

// Sequential placements: x, y (and z) receive n binary32 centres; 0, or -1
// when the reference throws.
static void put(const std::vector<float>& v, float* out) { std::memcpy(out, v.data(), v.size() * 4); }

int ref3d_cpu_palmieri2d(int n, double side, double radius, uint64_t seed, float* x, float* y) {
    try {
        std::vector<float> a, b;
        pf::palmieri_sequential_centres(n, side, radius, seed, &a, &b, nullptr);
        put(a, x);
        put(b, y);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref3d_cpu_palmieri3d(int n, double side, double radius, uint64_t seed, float* x, float* y,
                         float* z) {
    try {
        std::vector<float> a, b, c;
        pf3d::palmieri3d_sequential_centres(n, side, radius, seed, &a, &b, &c, nullptr);
        put(a, x);
        put(b, y);
        put(c, z);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

int ref3d_cpu_channel3d(int n, double side, int height, double radius, uint64_t seed, float* x,
                        float* y, float* z) {
    try {
        std::vector<float> a, b, c;
        pf3d::channel3d_sequential_centres(n, side, height, radius, seed, &a, &b, &c, nullptr);
        put(a, x);
        put(b, y);
        put(c, z);
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

uint64_t ref3d_cpu_table_hash(int n, const float* x, const float* y, const float* z) {
    const std::vector<float> a(x, x + n), b(y, y + n), c(z, z + n);
    return pf3d::centre_table_fnv1a64(pf3d::ordered_global_ids((std::size_t)n), a, b, c);
}

// The reference's soft identities (include/pf3d/initializer.hpp:81-95).
int ref_soft_membership(int n, double fraction, uint64_t seed, uint8_t* out) {
    try {
        const std::vector<std::uint8_t> m = pf3d::soft_id_membership(n, fraction, seed);
        std::memcpy(out, m.data(), m.size());
        return 0;
    } catch (const std::exception&) {
        return -1;
    }
}

// The reference's --initial-centres readers: 0 and the table's hash (and
// its centres) when accepted, -1 when refused.
int ref_read_table2(const char* path, int n, double side, double radius, float* x, float* y,
                    uint64_t* hash) {
    std::vector<float> a, b;
    pf::PalmieriCentresCsvDiagnostics d{};
    std::string err;
    if (!pf::palmieri_read_centres_csv(path, n, side, radius, &a, &b, &d, &err)) return -1;
    put(a, x);
    put(b, y);
    *hash = d.table_fnv1a64;
    return 0;
}

int ref_read_relaxed2(const char* path, int n, double side, int need_source_side, float* x, float* y) {
    std::vector<std::int64_t> ids;
    std::vector<float> a, b;
    pf::RelaxedCentresCsvDiagnostics d{};
    std::string err;
    if (!pf::relaxed_read_centres_csv(path, n, side, &ids, &a, &b, &d, &err, need_source_side != 0))
        return -1;
    put(a, x);
    put(b, y);
    return 0;
}

int ref_read_table3(const char* path, int n, double side, double radius, float* x, float* y,
                    float* z, uint64_t* hash) {
    std::vector<float> a, b, c;
    pf3d::PalmieriCentres3DCsvDiagnostics d{};
    std::string err;
    if (!pf3d::palmieri3d_read_centres_csv(path, n, side, radius, &a, &b, &c, &d, &err)) return -1;
    put(a, x);
    put(b, y);
    put(c, z);
    *hash = d.table_fnv1a64;
    return 0;
}

int ref_read_channel3(const char* path, int n, double side, int height, double radius, float* x,
                      float* y, float* z, uint64_t* hash) {
    std::vector<float> a, b, c;
    pf3d::PalmieriCentres3DCsvDiagnostics d{};
    std::string err;
    if (!pf3d::channel3d_read_centres_csv(path, n, side, height, radius, &a, &b, &c, &d, &err))
        return -1;
    put(a, x);
    put(b, y);
    put(c, z);
    *hash = d.table_fnv1a64;
    return 0;
}

}  // extern "C"
