// ORACLE -- test infrastructure only. A CPU restatement of the reference's 3D
// cell step (measurement, motion, moment-free update, recentring, Q5.27
// aggregate), used by tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg as the checker and the CPU timing. The product never
// links, loads or calls this file.
//
// Two arithmetic modes of the same algorithm:
//   * f32: binary32 fields and field arithmetic, binary64 reductions, every
//     operation separately rounded (compiled without contraction);
//   * f64: fields, coefficients, velocities and the aggregate quantisation in
//     binary64 (the FP64 transcription).
// The update walks source voxels into a zeroed destination, as the
// reference's tiled update does; for fully periodic cells that gives the
// same field and flags as its rolling-plane kernel.
//
// Algorithm sources in the reference, followed step by step:
//   measurement + commit   src/pf3d/kernels.cu:397-497, :1271-1409
//   motion + tumble        src/pf3d/kernels.cu:1739-1788, include/pf3d/rng.cuh:35-150
//   update                 src/pf3d/kernels.cu:498-793,
//                          src/pf3d/kernels_periodic_slab_walk.cu:54-318
//   z maps, flags, q_of    src/pf3d/device_common.cuh:100-213, include/pf3d/params.cuh:88-100
//   stencil                src/pf3d/device_common.cuh:218-245
//   sequencing kernels     src/pf3d/kernels.cu:2128-2321
//   sphere seeding         src/pf3d/kernels.cu:1071-1122
// Pinned by the reference's dense FP64 one-step (include/pf3d/reference.hpp)
// compiled in place into oracle/_ref and by its property tests
// (tests/3d/model_one_step_cpu_test.cpp), in tests/test_oracle3d_cpu.py.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/pfb200_3d.h"

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr float kEps = 1.0e-5f;

uint32_t mulhi(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

// common/philox.cuh:32-59 (Philox4x32, ten rounds)
void philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
            uint32_t out[4]) {
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint32_t h0 = mulhi(0xD2511F53u, c0), l0 = 0xD2511F53u * c0;
        const uint32_t h1 = mulhi(0xCD9E8D57u, c2), l1 = 0xCD9E8D57u * c2;
        const uint32_t n0 = h1 ^ c1 ^ k0, n2 = h0 ^ c3 ^ k1;
        c0 = n0;
        c1 = l1;
        c2 = n2;
        c3 = l0;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

double u53(uint32_t a, uint32_t b) {
    return (double)((((uint64_t)a << 32) | b) >> 11) * (1.0 / 9007199254740992.0);
}

bool periodic(uint32_t b) { return b == PFB3D_BOUNDARY_PERIODIC_XYZ; }
bool slab(uint32_t b) { return b == PFB3D_BOUNDARY_SUBSTRATE_SLAB; }
bool channel(uint32_t b) { return b == PFB3D_BOUNDARY_HARD_WALL_CHANNEL; }

// Q5.27 of a binary32 value: rn(min(phi^2, 4) 2^27); NaN squares give 0.
uint32_t q32(float phi) {
    volatile float s = phi * phi;
    float v = s;
    if (v > 4.0f) v = 4.0f;
    if (std::isnan(v)) return 0u;
    return (uint32_t)std::lrint(v * 134217728.0f);
}
// binary64 quantisation of the FP64 transcription (reference.hpp:141-152)
uint32_t q64(double phi) {
    double s = phi * phi;
    if (s > 4.0) s = 4.0;
    if (std::isnan(s)) return 0u;
    return (uint32_t)std::nearbyint(s * 134217728.0);
}
uint32_t qof(float v) { return q32(v); }
uint32_t qof(double v) { return q64(v); }

int wrap_origin(int64_t o, int n) {
    int64_t v = o % n;
    if (v < 0) v += n;
    return (int)v;
}
int wrap_add(int o, int d, int n) {
    int v = o + d;
    if (v >= n) v -= n;
    return v;
}

bool agg_z(const pfb_layout3d& L, int64_t oz, int z, int* wz) {
    if (periodic(L.boundary_flags)) {
        *wz = wrap_add(wrap_origin(oz, L.nz), z, L.nz);
        return true;
    }
    const int64_t w = oz + z;
    if (w < 0 || w >= L.nz) return false;
    *wz = (int)w;
    return true;
}

// z-neighbour source plane (device_common.cuh:125-154)
bool fetch_z(const pfb_layout3d& L, int64_t oz, int z, int B, int* src) {
    if (periodic(L.boundary_flags)) {
        if (z < 0 || z >= B) return false;
        *src = z;
        return true;
    }
    int64_t w = oz + z;
    if (channel(L.boundary_flags) && w == L.nz) w = L.nz - 1;
    if (w >= L.nz || w < -1) return false;
    if (w == -1) w = 0;
    const int64_t l = w - oz;
    if (l < 0 || l >= B) return false;
    *src = (int)l;
    return true;
}

size_t sidx(const pfb_layout3d& L, int x, int y, int z) {
    return ((size_t)z * L.ny + y) * (size_t)L.pitch_x + x;
}

bool fatal_any(const uint32_t* g) {
    if (!g) return false;
    for (int f = 0; f < PFB3D_FLAG_COUNT; ++f)
        if (((PFB3D_FATAL_MASK >> f) & 1u) && g[f]) return true;
    return false;
}

void raise(pfb_cell3d& c, uint32_t* g, int flag) {
#pragma omp atomic
    c.flags |= 1u << flag;
    if (g) {
#pragma omp atomic
        g[flag] += 1u;
    }
}

int clamp_shift(int p, int limit, int lo, int hi, int B) {
    p = p < -limit ? -limit : (p > limit ? limit : p);
    if (hi >= lo) {
        p = p < lo ? p : lo;
        p = p > hi - (B - 1) ? p : hi - (B - 1);
    }
    return p;
}

int round_half_even(double v) { return (int)std::nearbyint(v); }

template <typename R>
struct Field {
    const R* f;
    int B;
    const pfb_layout3d* L;
    int64_t oz;
    R at(int x, int y, int z) const {
        if (x < 0 || x >= B || y < 0 || y >= B) return R(0);
        int s;
        if (!fetch_z(*L, oz, z, B, &s)) return R(0);
        return f[((size_t)s * B + y) * B + x];
    }
};

// stencil27_at order: centre weight first, then z, y, x.
template <typename R>
void stencil(const Field<R>& F, int x, int y, int z, R* lap, R* gx, R* gy, R* gz) {
    R acc = R(-128) * F.at(x, y, z);
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int d = (dx != 0) + (dy != 0) + (dz != 0);
                if (d == 0) continue;
                const R w = d == 1 ? R(14) : d == 2 ? R(3) : R(1);
                const R prod = w * F.at(x + dx, y + dy, z + dz);
                acc = acc + prod;
            }
    *lap = acc * (R)(1.0 / 30.0);
    *gx = R(0.5) * (F.at(x + 1, y, z) - F.at(x - 1, y, z));
    *gy = R(0.5) * (F.at(x, y + 1, z) - F.at(x, y - 1, z));
    *gz = R(0.5) * (F.at(x, y, z + 1) - F.at(x, y, z - 1));
}

struct MArgs {
    const pfb_layout3d* L;
    int N, B;
    const float* wall;
    uint64_t step, polarity_stream, aging;
    double p_tumble;
    float mot;
    int max_shift, margin, apply_tumble, surface;
};

// measure_one_cell + commit_measurement for every cell
template <typename R>
void measure(const R* phi, const uint32_t* S, pfb_cell3d* cells, uint32_t* g, const MArgs& A) {
    const pfb_layout3d& L = *A.L;
    const int B = A.B;
#pragma omp parallel for schedule(dynamic)
    for (int n = 0; n < A.N; ++n) {
        pfb_cell3d& c = cells[n];
        if (c.storage_edge != 0u) continue;
        const Field<R> F{phi + (size_t)n * B * B * B, B, &L, c.origin_z};
        const int ox = wrap_origin(c.origin_x, L.nx), oy = wrap_origin(c.origin_y, L.ny);
        double V = 0, Cx = 0, Cy = 0, Cz = 0, Sf = 0, Ix = 0, Iy = 0, Iz = 0;
        int lo[3] = {B, B, B}, hi[3] = {-1, -1, -1};
        uint32_t pmax = 0;
        for (int z = 0; z < B; ++z) {
            int wz;
            if (!agg_z(L, c.origin_z, z, &wz)) continue;
            for (int y = 0; y < B; ++y)
                for (int x = 0; x < B; ++x) {
                    const R v = F.f[((size_t)z * B + y) * B + x];
                    if (!std::isfinite((double)v)) {
                        raise(c, g, PFB3D_FLAG_NONFINITE);
                        continue;
                    }
                    const R gx = R(0.5) * (F.at(x + 1, y, z) - F.at(x - 1, y, z));
                    const R gy = R(0.5) * (F.at(x, y + 1, z) - F.at(x, y - 1, z));
                    const R gz = R(0.5) * (F.at(x, y, z + 1) - F.at(x, y, z - 1));
                    R other = R(0);
                    if (v != R(0)) {
                        const uint32_t agg =
                            S[sidx(L, wrap_add(ox, x, L.nx), wrap_add(oy, y, L.ny), wz)];
                        const uint32_t own = qof(v);
                        if (agg >= own)
                            other = (R)(agg - own) * (R)7.450580596923828125e-9;
                        else
                            raise(c, g, PFB3D_FLAG_S_NEGATIVE);
                    }
                    if (channel(L.boundary_flags) && A.wall) other = other + (R)A.wall[wz];
                    const double sq = (double)v * (double)v;
                    V += sq;
                    Cx += sq * x;
                    Cy += sq * y;
                    Cz += sq * z;
                    if (A.surface)
                        Sf += std::sqrt((double)gx * gx + (double)gy * gy + (double)gz * gz);
                    const R ax = v * gx, ay = v * gy, az = v * gz;
                    Ix += (double)(ax * other);
                    Iy += (double)(ay * other);
                    Iz += (double)(az * other);
                    float fv = (float)std::fabs((double)v);
                    uint32_t bits;
                    std::memcpy(&bits, &fv, 4);
                    if (bits > pmax) pmax = bits;
                    if (std::fabs((double)v) > (double)kEps) {
                        if (slab(L.boundary_flags) && wz == L.nz - 1)
                            raise(c, g, PFB3D_FLAG_SLAB_TOP_CONTACT);
                        lo[0] = std::min(lo[0], x), hi[0] = std::max(hi[0], x);
                        lo[1] = std::min(lo[1], y), hi[1] = std::max(hi[1], y);
                        lo[2] = std::min(lo[2], z), hi[2] = std::max(hi[2], z);
                    }
                }
        }
        c.V = V;
        c.Cx = Cx;
        c.Cy = Cy;
        c.Cz = Cz;
        if (A.surface) c.surface = Sf;
        c.Ix = Ix;
        c.Iy = Iy;
        c.Iz = Iz;
        c.bb_lo_x = lo[0], c.bb_hi_x = hi[0];
        c.bb_lo_y = lo[1], c.bb_hi_y = hi[1];
        c.bb_lo_z = lo[2], c.bb_hi_z = hi[2];
        std::memcpy(&c.phi_max, &pmax, 4);
        int s[3] = {0, 0, 0};
        if (V > 0.0 && std::isfinite(V)) {
            const double mid = 0.5 * (double)(B - 1);
            const double cs[3] = {Cx, Cy, Cz};
            for (int a = 0; a < 3; ++a)
                s[a] = clamp_shift(round_half_even(cs[a] / V - mid), A.max_shift, lo[a], hi[a], B);
        } else {
            raise(c, g, PFB3D_FLAG_V_NONPOSITIVE);
        }
        c.pending_shift_x = s[0];
        c.pending_shift_y = s[1];
        c.pending_shift_z = s[2];
        if (hi[0] >= lo[0]) {
            const int m = A.margin, ml = m / 2, mu = m - ml;
            bool bad = false;
            for (int a = 0; a < 3; ++a) {
                const int ext = hi[a] - lo[a] + 1;
                if (ext + m > B || lo[a] - s[a] < ml || hi[a] - s[a] >= B - mu) bad = true;
            }
            if (bad) raise(c, g, PFB3D_FLAG_SUPPORT_EXHAUSTED);
        }
    }
}

void iso_dir(double au, double zu, double* d) {
    const double z = 2.0 * au - 1.0;
    const double r2 = 1.0 - z * z;
    const double r = std::sqrt(r2 > 0.0 ? r2 : 0.0);
    const double a = 2.0 * kPi * zu;
    d[0] = r * std::cos(a);
    d[1] = r * std::sin(a);
    d[2] = z;
}

// Motion of every cell; vel receives the velocities the update uses: the
// binary32 values of the record, or (f64) the same formula in binary64 with
// motility coefficient mot64.
void motion(pfb_cell3d* cells, uint32_t* g, const MArgs& A, bool f64, double mot64,
            std::vector<double>& vel) {
    vel.assign((size_t)3 * A.N, 0.0);
    for (int n = 0; n < A.N; ++n) {
        vel[3 * n] = cells[n].velocity_x;
        vel[3 * n + 1] = cells[n].velocity_y;
        vel[3 * n + 2] = cells[n].velocity_z;
    }
    const bool sl = slab(A.L->boundary_flags);
    const bool gfatal = fatal_any(g);
    for (int n = 0; n < A.N; ++n) {
        pfb_cell3d& c = cells[n];
        if ((c.flags & PFB3D_FATAL_MASK) || gfatal) continue;
        const bool active = A.step >= A.aging;
        double p[3] = {c.polarity_x, c.polarity_y, c.polarity_z};
        bool tumbled = false;
        if (A.apply_tumble && active) {
            const uint64_t st = A.step - A.aging, gid = (uint64_t)c.global_id;
            uint32_t ev[4], vec[4];
            philox((uint32_t)st, (uint32_t)(st >> 32), (uint32_t)gid,
                   (uint32_t)(gid >> 32) ^ 0x54554D45u, (uint32_t)A.polarity_stream,
                   (uint32_t)(A.polarity_stream >> 32), ev);
            if (u53(ev[0], ev[1]) < A.p_tumble) {
                philox((uint32_t)st, (uint32_t)(st >> 32), (uint32_t)gid,
                       (uint32_t)(gid >> 32) ^ 0x54554D56u, (uint32_t)A.polarity_stream,
                       (uint32_t)(A.polarity_stream >> 32), vec);
                if (sl) {
                    const double a = 2.0 * kPi * u53(vec[0], vec[1]);
                    p[0] = std::cos(a);
                    p[1] = std::sin(a);
                    p[2] = 0.0;
                } else {
                    iso_dir(u53(ev[2], ev[3]), u53(vec[0], vec[1]), p);
                }
                tumbled = true;
            }
        }
        const float px = (float)p[0], py = (float)p[1], pz = sl ? 0.0f : (float)p[2];
        const float sp = active ? c.v_A : 0.0f;
        volatile float t0 = sp * px, t1 = A.mot * (float)c.Ix;
        const float vx = t0 + t1;
        t0 = sp * py;
        t1 = A.mot * (float)c.Iy;
        const float vy = t0 + t1;
        t0 = sp * pz;
        t1 = A.mot * (float)c.Iz;
        const float vz = sl ? 0.0f : (float)(t0 + t1);
        if (!std::isfinite(px) || !std::isfinite(py) || !std::isfinite(pz) || !std::isfinite(vx) ||
            !std::isfinite(vy) || !std::isfinite(vz)) {
            raise(c, g, PFB3D_FLAG_NONFINITE);
            continue;
        }
        c.polarity_x = px;
        c.polarity_y = py;
        c.polarity_z = pz;
        c.velocity_x = vx;
        c.velocity_y = vy;
        c.velocity_z = vz;
        if (f64) {
            const double s = active ? (double)c.v_A : 0.0;
            vel[3 * n] = s * p[0] + mot64 * c.Ix;
            vel[3 * n + 1] = s * p[1] + mot64 * c.Iy;
            vel[3 * n + 2] = sl ? 0.0 : s * p[2] + mot64 * c.Iz;
        } else {
            vel[3 * n] = vx;
            vel[3 * n + 1] = vy;
            vel[3 * n + 2] = vz;
        }
        if (tumbled) ++c.tumble_ctr;
    }
}

struct UArgs {
    const pfb_layout3d* L;
    int N, B;
    const float* wall;
    double dt, V0, volume_scale, bulk_scale, inter;
};

template <typename R>
void scatter_one(uint32_t* S, size_t i, R v, pfb_cell3d& c, uint32_t* g) {
    const R sq = v * v;
    if (sq > R(4)) raise(c, g, PFB3D_FLAG_Q_CLAMP);
    const uint32_t q = qof(v);
    if (!q) return;
    uint32_t old;
#pragma omp atomic capture
    {
        old = S[i];
        S[i] += q;
    }
    if (old > 0xFFFFFFFFu - q) raise(c, g, PFB3D_FLAG_S_OVERFLOW);
}

// moment-free update with recentring (tiled-path order), abort copy on a
// fatal flag
template <typename R>
void update(const R* in, R* out, const uint32_t* Sin, uint32_t* Sout, pfb_cell3d* cells,
            uint32_t* g, const UArgs& A, const std::vector<double>& vel) {
    const pfb_layout3d& L = *A.L;
    const int B = A.B;
    const size_t words = (size_t)B * B * B;
    std::vector<char> abort_cell(A.N, 0);
    for (int n = 0; n < A.N; ++n) {
        const pfb_cell3d& c = cells[n];
        abort_cell[n] = ((c.flags & PFB3D_FATAL_MASK) || fatal_any(g)) ? 1 : 0;
    }
#pragma omp parallel for schedule(dynamic)
    for (int n = 0; n < A.N; ++n) {
        pfb_cell3d& c = cells[n];
        if (c.storage_edge != 0u) continue;
        const R* src = in + (size_t)n * words;
        R* dst = out + (size_t)n * words;
        const int ox = wrap_origin(c.origin_x, L.nx), oy = wrap_origin(c.origin_y, L.ny);
        if (abort_cell[n]) {
            for (size_t q = 0; q < words; ++q) {
                dst[q] = src[q];
                if (Sout && std::isfinite((double)src[q])) {
                    const int x = (int)(q % B), y = (int)((q / B) % B), z = (int)(q / ((size_t)B * B));
                    int wz;
                    if (!agg_z(L, c.origin_z, z, &wz)) continue;
                    scatter_one(Sout, sidx(L, wrap_add(ox, x, L.nx), wrap_add(oy, y, L.ny), wz),
                                src[q], c, g);
                }
            }
            c.pending_shift_x = c.pending_shift_y = c.pending_shift_z = 0;
            continue;
        }
        std::fill(dst, dst + words, R(0));
        const int sx = c.pending_shift_x, sy = c.pending_shift_y, sz = c.pending_shift_z;
        const R gamma = (R)c.gamma;
        const R vx = (R)vel[3 * n], vy = (R)vel[3 * n + 1], vz = (R)vel[3 * n + 2];
        const R bulk = (R)A.bulk_scale * gamma;
        const R volume = (R)(A.volume_scale * (A.V0 - c.V));
        const R inter = (R)A.inter, dt = (R)A.dt;
        const Field<R> F{src, B, &L, c.origin_z};
        for (int z = 0; z < B; ++z) {
            int wz;
            if (!agg_z(L, c.origin_z, z, &wz)) continue;
            const R wallv = (channel(L.boundary_flags) && A.wall) ? (R)A.wall[wz] : R(0);
            for (int y = 0; y < B; ++y)
                for (int x = 0; x < B; ++x) {
                    const R v = src[((size_t)z * B + y) * B + x];
                    if (!std::isfinite((double)v)) {
                        raise(c, g, PFB3D_FLAG_NONFINITE);
                        continue;
                    }
                    R lap, gx, gy, gz;
                    stencil(F, x, y, z, &lap, &gx, &gy, &gz);
                    if (v == R(0) && lap == R(0) && gx == R(0) && gy == R(0) && gz == R(0)) continue;
                    const int wx = wrap_add(ox, x, L.nx), wy = wrap_add(oy, y, L.ny);
                    const uint32_t agg = Sin[sidx(L, wx, wy, wz)];
                    const uint32_t own = qof(v);
                    R other;
                    if (agg >= own) {
                        other = (R)(agg - own) * (R)7.450580596923828125e-9;
                    } else {
                        other = R(0);
                        raise(c, g, PFB3D_FLAG_S_NEGATIVE);
                    }
                    other = other + wallv;
                    // gamma lap - bulk c (1-c)(1-2c) + vol c - inter c other - v.grad
                    const R t1 = gamma * lap;
                    const R t2 = ((bulk * v) * (R(1) - v)) * (R(1) - R(2) * v);
                    const R t3 = volume * v;
                    const R t4 = (inter * v) * other;
                    const R adv = (vx * gx + vy * gy) + vz * gz;
                    const R rhs = (((t1 - t2) + t3) - t4) - adv;
                    const R next = v + dt * rhs;
                    if (!std::isfinite((double)next)) {
                        raise(c, g, PFB3D_FLAG_NONFINITE);
                        continue;
                    }
                    if (slab(L.boundary_flags) && wz == L.nz - 1 &&
                        std::fabs((double)next) > (double)kEps) {
                        raise(c, g, PFB3D_FLAG_SLAB_TOP_CONTACT);
                        continue;
                    }
                    const int dx = x - sx, dy = y - sy, dz = z - sz;
                    if (dx < 0 || dx >= B || dy < 0 || dy >= B || dz < 0 || dz >= B) {
                        if (std::fabs((double)next) > (double)kEps)
                            raise(c, g, PFB3D_FLAG_DESTINATION_CLIP);
                        continue;
                    }
                    dst[((size_t)dz * B + dy) * B + dx] = next;
                    if (Sout) scatter_one(Sout, sidx(L, wx, wy, wz), next, c, g);
                }
        }
    }
}

template <typename R>
void scatter_all(const R* phi, pfb_cell3d* cells, uint32_t* S, uint32_t* g, const pfb_layout3d& L,
                 int N, int B) {
#pragma omp parallel for schedule(dynamic)
    for (int n = 0; n < N; ++n) {
        pfb_cell3d& c = cells[n];
        if (c.storage_edge != 0u) continue;
        const R* f = phi + (size_t)n * B * B * B;
        const int ox = wrap_origin(c.origin_x, L.nx), oy = wrap_origin(c.origin_y, L.ny);
        for (int z = 0; z < B; ++z) {
            int wz;
            if (!agg_z(L, c.origin_z, z, &wz)) continue;
            for (int y = 0; y < B; ++y)
                for (int x = 0; x < B; ++x) {
                    const R v = f[((size_t)z * B + y) * B + x];
                    if (!std::isfinite((double)v)) {
                        raise(c, g, PFB3D_FLAG_NONFINITE);
                        continue;
                    }
                    scatter_one(S, sidx(L, wrap_add(ox, x, L.nx), wrap_add(oy, y, L.ny), wz), v, c, g);
                }
        }
    }
}

void finalize(pfb_cell3d* cells, int N) {
    for (int n = 0; n < N; ++n) {
        pfb_cell3d& c = cells[n];
        if (c.flags & PFB3D_FATAL_MASK) {
            c.pending_shift_x = c.pending_shift_y = c.pending_shift_z = 0;
            continue;
        }
        const int sx = c.pending_shift_x, sy = c.pending_shift_y, sz = c.pending_shift_z;
        c.origin_x += sx;
        c.origin_y += sy;
        c.origin_z += sz;
        if (sx || sy || sz) ++c.shift_ctr;
        c.pending_shift_x = c.pending_shift_y = c.pending_shift_z = 0;
    }
}

void set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

}  // namespace

extern "C" {

// One step of the reference's Sim3D sequence on host buffers (phi_in,
// phi_out of N B^3 values; S_in read, S_out cleared and scattered; cells and
// the 10 global flag counters updated; *step advanced unless a fatal flag
// is set). f64 != 0: phi is double. wall: nz values or null. threads <= 0
// keeps the OpenMP default.
int oracle3d_step(int f64, const void* phi_in, void* phi_out, const uint32_t* S_in,
                  uint32_t* S_out, pfb_cell3d* cells, uint32_t* gflags, uint64_t* step,
                  const pfb_layout3d* L, int N, int B, const float* wall, double dt,
                  double lambda, double kappa, double mu, double xi, double tau,
                  double target_radius, uint64_t polarity_stream, uint64_t aging_steps,
                  int surface, int threads) {
    set_threads(threads);
    std::vector<pfb_cell3d> accepted(cells, cells + N);
    MArgs m{L, N, B, wall, *step, polarity_stream, aging_steps, -std::expm1(-dt / tau),
            (float)(60.0 * kappa / (lambda * lambda) / xi), 4, 8, 1, surface};
    if (f64) {
        measure((const double*)phi_in, S_in, cells, gflags, m);
    } else {
        measure((const float*)phi_in, S_in, cells, gflags, m);
    }
    std::vector<double> vel;
    const double mot64 = 60.0 * kappa / (xi * lambda * lambda);
    motion(cells, gflags, m, f64 != 0, mot64, vel);
    const size_t sw = (size_t)L->pitch_x * L->ny * L->nz;
    std::memset(S_out, 0, sw * sizeof(uint32_t));
    const double sphere = 4.0 * kPi * target_radius * target_radius * target_radius / 3.0;
    const double V0 = slab(L->boundary_flags) ? 0.5 * sphere : sphere;
    UArgs u{L, N, B, wall, (double)(float)dt, V0, 2.0 * mu / V0,
            (double)(float)(30.0 / (lambda * lambda)), (double)(float)(60.0 * kappa / (lambda * lambda))};
    if (f64) {
        u.dt = dt;
        u.bulk_scale = 30.0 / (lambda * lambda);
        u.inter = 60.0 * kappa / (lambda * lambda);
        update((const double*)phi_in, (double*)phi_out, S_in, S_out, cells, gflags, u, vel);
    } else {
        update((const float*)phi_in, (float*)phi_out, S_in, S_out, cells, gflags, u, vel);
    }
    const size_t words = (size_t)N * B * B * B;
    if (fatal_any(gflags)) {
        // repair: keep phi_in, rebuild S_out, restore the accepted records
        std::memset(S_out, 0, sw * sizeof(uint32_t));
        if (f64) {
            std::memcpy(phi_out, phi_in, words * sizeof(double));
            scatter_all((const double*)phi_in, cells, S_out, gflags, *L, N, B);
        } else {
            std::memcpy(phi_out, phi_in, words * sizeof(float));
            scatter_all((const float*)phi_in, cells, S_out, gflags, *L, N, B);
        }
        for (int n = 0; n < N; ++n)
            cells[n].pending_shift_x = cells[n].pending_shift_y = cells[n].pending_shift_z = 0;
        finalize(cells, N);
        for (int n = 0; n < N; ++n) cells[n] = accepted[n];
        return 1;
    }
    finalize(cells, N);
    ++*step;
    return 0;
}

// Measurement + motion only (no tumble when apply_tumble = 0), as after a
// fresh start.
void oracle3d_measure(int f64, const void* phi, const uint32_t* S, pfb_cell3d* cells,
                      uint32_t* gflags, uint64_t step, const pfb_layout3d* L, int N, int B,
                      const float* wall, double dt, double lambda, double kappa, double xi,
                      double tau, uint64_t polarity_stream, uint64_t aging_steps,
                      int apply_tumble, int surface, int motion_too) {
    MArgs m{L, N, B, wall, step, polarity_stream, aging_steps, -std::expm1(-dt / tau),
            (float)(60.0 * kappa / (lambda * lambda) / xi), 4, 8, apply_tumble, surface};
    if (f64)
        measure((const double*)phi, S, cells, gflags, m);
    else
        measure((const float*)phi, S, cells, gflags, m);
    std::vector<double> vel;
    if (motion_too) motion(cells, gflags, m, f64 != 0, 60.0 * kappa / (xi * lambda * lambda), vel);
}

void oracle3d_scatter(int f64, const void* phi, pfb_cell3d* cells, uint32_t* S, uint32_t* gflags,
                      const pfb_layout3d* L, int N, int B) {
    if (f64)
        scatter_all((const double*)phi, cells, S, gflags, *L, N, B);
    else
        scatter_all((const float*)phi, cells, S, gflags, *L, N, B);
}

uint32_t oracle3d_q32(float v) { return q32(v); }

}  // extern "C"
