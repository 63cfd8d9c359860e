// ORACLE -- test infrastructure only. A CPU restatement of the reference's 2D
// active multi-phase-field step, used by tests/, __graft_entry__.smoke() and
// the CPU-baseline leg of bench.py as the checker and the CPU timing. The
// product never links, loads or calls this file.
//
// Two arithmetic modes of the same algorithm:
//   * f32: binary32 field arithmetic with binary64 reductions, the arithmetic
//     of the GPU kernels (compiled without contraction: every operation is
//     separately rounded), OpenMP-parallel over cells;
//   * f64: every field, coefficient and velocity in binary64 (the "FP64
//     transcription" used to report per-observable error).
// Decisions that the reference makes in integers (Philox draws, class choice,
// shifts, the Q5.27 aggregate) are the same in both modes.
//
// Algorithm sources in the reference, followed step by step:
//   tumble + class + shift     src/kernels.cu:93-191, :624-711
//   interaction integral       src/kernels.cu:254-342, :714-780
//   Euler update               src/kernels.cu:354-443, :789-842 (+ include/kernels.cuh:121-138)
//   store / scatter / moments  src/kernels.cu:447-590, :844-935
//   slot clear, step counter   src/kernels.cu:955-973
//   initialisation             src/kernels.cu:1050-1190
//   Philox / coefficients      common/philox.cuh:32-67, common/model_coefficients.cuh:23-53
// Pinned by the reference's golden vectors (tests/common_primitives_cpu_test.cpp:48-61,
// tests/mobility_model_cpu_test.cpp:61-88) in tests/test_oracle_golden.py.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <algorithm>
#include <cstring>
#include <random>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/pfb200.h"

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr int kPitch = 288;
constexpr int kArea = 288 * 288;

struct Win {
    int wx, wy, tx0, ty0;
};

// Shape-class table, include/params.cuh:138-147.
Win win(int c) {
    static const Win t[6] = {{144, 144, 64, 64}, {176, 144, 32, 64}, {144, 176, 64, 32},
                             {160, 160, 32, 32}, {224, 224, 32, 32}, {286, 286, 1, 1}};
    return t[(c >= 0 && c < 6) ? c : 0];
}

// include/params.cuh:222-235; on sides up to 286 (below the reference's
// minimum) only the classes whose window fits the side L take part
int class_containing(int ex, int ey, int slack, int L) {
    int best = -1, area = 0;
    for (int c = 0; c < 6; ++c) {
        const Win w = win(c);
        if (w.wx > L || w.wy > L) continue;
        if (ex + slack <= w.wx && ey + slack <= w.wy && (best < 0 || w.wx * w.wy < area)) {
            best = c;
            area = w.wx * w.wy;
        }
    }
    return best;
}

uint32_t mulhi(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

// common/philox.cuh:32-59
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

// common/philox.cuh:62-67
double u53(uint32_t a, uint32_t b) {
    return (double)((((uint64_t)a << 32) | b) >> 11) * (1.0 / 9007199254740992.0);
}

// include/params.cuh:103-111: rn(min(phi^2, 4) * 2^27)
uint32_t q_f(float phi) {
    float s = phi * phi;
    s = std::fmin(s, 4.0f);
    return (uint32_t)std::lrint(s * 134217728.0f);
}
// Binary64 analogue for the f64 transcription.
uint32_t q_d(double phi) {
    double s = phi * phi;
    s = std::fmin(s, 4.0);
    return (uint32_t)std::llrint(s * 134217728.0);
}

template <typename R> uint32_t q_of(R v);
template <> uint32_t q_of<float>(float v) { return q_f(v); }
template <> uint32_t q_of<double>(double v) { return q_d(v); }

template <typename R> R r_sin(R v);
template <typename R> R r_cos(R v);
template <> float r_sin<float>(float v) { return std::sin(v); }
template <> float r_cos<float>(float v) { return std::cos(v); }
template <> double r_sin<double>(double v) { return std::sin(v); }
template <> double r_cos<double>(double v) { return std::cos(v); }

// include/kernels.cuh:121-138 (same operation order).
template <typename R>
R rhs(R lap, R phi, R So, R gx, R gy, R gam, R dwC, R volC, R repC, R vx, R vy, R mrel) {
    const R one = 1, two = 2;
    if (mrel == one)
        return gam * lap - dwC * (phi * (one - phi) * (one - two * phi)) + volC * phi -
               repC * phi * So - (vx * gx + vy * gy);
    return mrel * (gam * lap - dwC * (phi * (one - phi) * (one - two * phi)) + volC * phi -
                   repC * phi * So) -
           (vx * gx + vy * gy);
}

int wrap(int v, int L) {
    v %= L;
    return v < 0 ? v + L : v;
}

void add_u32(uint32_t* p, uint32_t v, uint32_t* old) {
    *old = __atomic_fetch_add(p, v, __ATOMIC_RELAXED);
}
void flag_or(uint32_t* f, int i) { __atomic_fetch_or(f + i, 1u, __ATOMIC_RELAXED); }
void flag_add(uint32_t* f, int i, uint32_t v) { __atomic_fetch_add(f + i, v, __ATOMIC_RELAXED); }

// Working record of one cell in the arithmetic type R.
template <typename R> struct Cell {
    int gx0, gy0, cls, cls_written[2], gid;
    R gamma, v_A, theta, M_pf, vx, vy, phi_max;
    double V, Cx, Cy, perim, Ix, Iy;
    int bb[4];
    uint32_t promote, shifts, tumbles, reserved[2];
};

template <typename R> struct Args {
    const R* phi_in;
    R* phi_out;
    const uint32_t* S_rd;
    uint32_t* S_sc;
    Cell<R>* cell;
    uint32_t* flags;
    unsigned long long step;
    int N, L, P, parity_out;
    R dt;
    double A0, vol_scale;
    R bulk, rep;
    R mot;
    unsigned long long polarity_seed;
    double p_tumble;
    int full_moment_every;
};

// One cell of one step (reference process_cell / process_cell_fallback).
template <typename R> void step_cell(const Args<R>& A, int n, std::vector<R>& tmp) {
    Cell<R>& c = A.cell[n];
    const int CLS = c.cls;
    const Win W = win(CLS);
    const bool staged = CLS <= 3;
    const bool fallback = CLS == 5;
    const unsigned long long step = A.step;

    uint32_t r[4];
    philox((uint32_t)step, (uint32_t)(step >> 32), (uint32_t)c.gid, 0xA5A5A5A5u,
           (uint32_t)A.polarity_seed, (uint32_t)(A.polarity_seed >> 32), r);
    R theta = c.theta;
    int tumbled = 0;
    if (u53(r[0], r[1]) < A.p_tumble) {
        theta = (R)(2.0 * kPi * u53(r[2], r[3]));
        tumbled = 1;
    }
    const R ps = r_sin<R>(theta), pc = r_cos<R>(theta);
    const R gam = c.gamma;
    const R dwC = A.bulk * gam;
    const R volC = (R)(A.vol_scale * (A.A0 - c.V));
    const R mrel = c.M_pf * (R)2;

    const int ex = c.bb[1] - c.bb[0] + 1, ey = c.bb[3] - c.bb[2] + 1;
    int dcls = CLS, no_margin = 0;
    unsigned pctr = c.promote;
    if (ex > 0) {
        if (ex + 8 > W.wx || ey + 8 > W.wy) {
            const int grow = class_containing(ex, ey, 8, A.L);
            if (grow >= 0)
                dcls = grow;
            else if (fallback && ex <= W.wx && ey <= W.wy)
                no_margin = 1;
            else
                flag_add(A.flags, PFB_FLAG_CLASS_EXHAUSTED, 1u);
            pctr = 0;
        } else {
            const int small = class_containing(ex, ey, 20, A.L);
            if (small >= 0 && small != CLS && win(small).wx * win(small).wy < W.wx * W.wy) {
                if (++pctr >= 200u) {
                    dcls = small;
                    pctr = 0;
                }
            } else {
                pctr = 0;
            }
        }
    }
    const Win D = win(dcls);
    int sx = 0, sy = 0;
    if (c.V > 0.0) {
        sx = (int)std::nearbyint(c.Cx / c.V - 0.5 * (double)(D.wx - 1));
        sy = (int)std::nearbyint(c.Cy / c.V - 0.5 * (double)(D.wy - 1));
        const int mx = dcls == CLS ? 4 : W.wx, my = dcls == CLS ? 4 : W.wy;
        sx = sx < -mx ? -mx : (sx > mx ? mx : sx);
        sy = sy < -my ? -my : (sy > my ? my : sy);
    } else {
        flag_or(A.flags, PFB_FLAG_V_NONPOS);
    }
    const int fm = A.full_moment_every > 0 && ((step + 1ull) % (unsigned long long)A.full_moment_every) == 0ull;

    const R* tin = A.phi_in + (size_t)n * kArea;
    auto phi = [&](int x, int y) -> R {
        if (x < 0 || y < 0 || x >= W.wx || y >= W.wy) return (R)0;
        return tin[(size_t)(W.ty0 + y) * kPitch + W.tx0 + x];
    };
    const int L = A.L, P = A.P;
    auto qS_at = [&](int x, int y) -> uint32_t {
        int gy = c.gy0 + y;
        if (gy >= L) gy -= L;
        int gx = c.gx0 + x;
        if (gx >= L) gx -= L;
        return A.S_rd[(size_t)gy * P + gx];
    };
    auto s_other = [&](uint32_t qS, R v) -> R {
        const uint32_t qc = q_of<R>(v);
        if (qS >= qc) return (R)(qS - qc) * (R)7.45058059692382812e-09;
        flag_add(A.flags, PFB_FLAG_S_NEGATIVE, 1u);
        return (R)0;
    };

    // Interaction integral, row-major, one accumulator per component.
    double sIx = 0.0, sIy = 0.0;
    for (int y = 0; y < W.wy; ++y)
        for (int x = 0; x < W.wx; ++x) {
            const R v = phi(x, y);
            const R So = s_other(qS_at(x, y), v);
            const R gx = (R)0.5 * (phi(x + 1, y) - phi(x - 1, y));
            const R gy = (R)0.5 * (phi(x, y + 1) - phi(x, y - 1));
            sIx += (double)(v * gx * So);
            sIy += (double)(v * gy * So);
        }
    const double vxd = (double)c.v_A * (double)pc + (double)A.mot * sIx;
    const double vyd = (double)c.v_A * (double)ps + (double)A.mot * sIy;
    const R vx = (R)vxd, vy = (R)vyd;
    c.vx = vx;
    c.vy = vy;
    c.Ix = sIx;
    c.Iy = sIy;

    // Euler update of the source window.
    tmp.assign((size_t)W.wx * W.wy, (R)0);
    for (int y = 0; y < W.wy; ++y)
        for (int x = 0; x < W.wx; ++x) {
            const R cC = phi(x, y);
            const R nC = phi(x, y + 1), sC = phi(x, y - 1), cE = phi(x + 1, y), cW = phi(x - 1, y);
            const R nE = phi(x + 1, y + 1), nW = phi(x - 1, y + 1), sE = phi(x + 1, y - 1),
                    sW = phi(x - 1, y - 1);
            const R lap = ((R)4 * (nC + sC + cE + cW) + (nE + nW + sE + sW) + (R)(-20) * cC) *
                          (R)(1.0 / 6.0);
            const R gx = (R)0.5 * (cE - cW), gy = (R)0.5 * (nC - sC);
            const R So = s_other(qS_at(x, y), cC);
            const R rr = rhs<R>(lap, cC, So, gx, gy, gam, dwC, volC, A.rep, vx, vy, mrel);
            tmp[(size_t)y * W.wx + x] = cC + A.dt * rr;
        }

    // Store, scatter, moments.
    R* tout = A.phi_out + (size_t)n * kArea;
    if (dcls != c.cls_written[A.parity_out])
        for (int i = 0; i < kArea; ++i) tout[i] = (R)0;
    auto src = [&](int i, int j) -> R {
        if (i < 0 || j < 0 || i >= W.wx || j >= W.wy) return (R)0;
        return tmp[(size_t)j * W.wx + i];
    };
    if (!staged) {
        for (int b = 0; b < D.wy; ++b)
            for (int a = 0; a < D.wx; ++a)
                tout[(size_t)(D.ty0 + b) * kPitch + D.tx0 + a] = src(a + sx, b + sy);
    }
    auto dst = [&](int a, int b) -> R {
        if (a < 0 || b < 0 || a >= D.wx || b >= D.wy) return (R)0;
        return tout[(size_t)(D.ty0 + b) * kPitch + D.tx0 + a];
    };
    const int gx0n = wrap(c.gx0 + sx, L), gy0n = wrap(c.gy0 + sy, L);
    double aV = 0.0, aCx = 0.0, aCy = 0.0, aPer = 0.0;
    int blox = D.wx, bhix = -1, bloy = D.wy, bhiy = -1;
    R pmax = (R)0;
    for (int b = 0; b < D.wy; ++b) {
        int gy = gy0n + b;
        if (gy >= L) gy -= L;
        for (int a = 0; a < D.wx; ++a) {
            const int i = a + sx, j = b + sy;
            R pn;
            if (staged) {
                pn = src(i, j);
                tout[(size_t)(D.ty0 + b) * kPitch + D.tx0 + a] = pn;
            } else {
                pn = dst(a, b);
            }
            if (!std::isfinite((double)pn)) flag_or(A.flags, PFB_FLAG_NONFINITE);
            if (pn * pn > (R)4) flag_or(A.flags, PFB_FLAG_Q_CLAMP);
            const R apn = std::fabs(pn);
            if (apn > pmax) pmax = apn;
            const uint32_t q = q_of<R>(pn);
            if (q) {
                int gx = gx0n + a;
                if (gx >= L) gx -= L;
                uint32_t old;
                add_u32(A.S_sc + (size_t)gy * P + gx, q, &old);
                if (old > 0xFFFFFFFFu - q) flag_or(A.flags, PFB_FLAG_S_OVERFLOW);
            }
            const double d = (double)pn * (double)pn;
            aV += d;
            aCx += d * (double)a;
            aCy += d * (double)b;
            if (pn > (R)1e-5f) {
                if (a < blox) blox = a;
                if (a > bhix) bhix = a;
                if (b < bloy) bloy = b;
                if (b > bhiy) bhiy = b;
            }
            if (fm) {
                R e, w, nn, ss;
                if (staged) {
                    const bool jin = j >= 0 && j < W.wy, iin = i >= 0 && i < W.wx;
                    e = jin ? src(i + 1, j) : (R)0;
                    w = jin ? src(i - 1, j) : (R)0;
                    nn = iin ? src(i, j + 1) : (R)0;
                    ss = iin ? src(i, j - 1) : (R)0;
                } else {
                    e = dst(a + 1, b);
                    w = dst(a - 1, b);
                    nn = dst(a, b + 1);
                    ss = dst(a, b - 1);
                }
                const R pgx = (R)0.5 * (e - w), pgy = (R)0.5 * (nn - ss);
                aPer += (double)std::sqrt(pgx * pgx + pgy * pgy);
            }
        }
    }
    c.gx0 = gx0n;
    c.gy0 = gy0n;
    c.cls = dcls;
    c.cls_written[A.parity_out] = dcls;
    c.theta = theta;
    c.V = aV;
    c.Cx = aCx;
    c.Cy = aCy;
    if (fm) c.perim = aPer;
    c.bb[0] = blox;
    c.bb[1] = bhix;
    c.bb[2] = bloy;
    c.bb[3] = bhiy;
    c.promote = pctr;
    c.shifts += (sx | sy) ? 1u : 0u;
    c.tumbles += (uint32_t)tumbled;
    c.phi_max = pmax;
    if (fallback) {
        const bool edge = bhix >= 0 && (blox == 0 || bhix == D.wx - 1 || bloy == 0 || bhiy == D.wy - 1);
        c.reserved[0] = 1u;
        if (no_margin || (dcls == 5 && edge)) ++c.reserved[1];
    }
}

template <typename R> void step_all(const Args<R>& A, int threads) {
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
    {
        std::vector<R> tmp;
#pragma omp for schedule(dynamic, 1)
        for (int n = 0; n < A.N; ++n) step_cell<R>(A, n, tmp);
    }
#else
    (void)threads;
    std::vector<R> tmp;
    for (int n = 0; n < A.N; ++n) step_cell<R>(A, n, tmp);
#endif
}

template <typename R> Cell<R> from_abi(const pfb_cell2d& s) {
    Cell<R> c;
    c.gx0 = s.gx0;
    c.gy0 = s.gy0;
    c.cls = s.cls;
    c.cls_written[0] = s.cls_written[0];
    c.cls_written[1] = s.cls_written[1];
    c.gid = s.global_id;
    c.gamma = (R)s.gamma;
    c.v_A = (R)s.v_A;
    c.theta = (R)s.theta;
    c.M_pf = (R)s.M_pf;
    c.vx = (R)s.vx;
    c.vy = (R)s.vy;
    c.phi_max = (R)s.phi_max;
    c.V = s.V;
    c.Cx = s.Cx;
    c.Cy = s.Cy;
    c.perim = s.perim;
    c.Ix = s.Ix;
    c.Iy = s.Iy;
    c.bb[0] = s.bb_lo_x;
    c.bb[1] = s.bb_hi_x;
    c.bb[2] = s.bb_lo_y;
    c.bb[3] = s.bb_hi_y;
    c.promote = s.promote_ctr;
    c.shifts = s.shift_ctr;
    c.tumbles = s.tumble_ctr;
    c.reserved[0] = s.reserved[0];
    c.reserved[1] = s.reserved[1];
    return c;
}

template <typename R> void to_abi(const Cell<R>& c, pfb_cell2d& s) {
    s.gx0 = c.gx0;
    s.gy0 = c.gy0;
    s.cls = (uint8_t)c.cls;
    s.cls_written[0] = (uint8_t)c.cls_written[0];
    s.cls_written[1] = (uint8_t)c.cls_written[1];
    s.global_id = c.gid;
    s.gamma = (float)c.gamma;
    s.v_A = (float)c.v_A;
    s.theta = (float)c.theta;
    s.M_pf = (float)c.M_pf;
    s.vx = (float)c.vx;
    s.vy = (float)c.vy;
    s.phi_max = (float)c.phi_max;
    s.V = c.V;
    s.Cx = c.Cx;
    s.Cy = c.Cy;
    s.perim = c.perim;
    s.Ix = c.Ix;
    s.Iy = c.Iy;
    s.bb_lo_x = c.bb[0];
    s.bb_hi_x = c.bb[1];
    s.bb_lo_y = c.bb[2];
    s.bb_hi_y = c.bb[3];
    s.promote_ctr = c.promote;
    s.shift_ctr = c.shifts;
    s.tumble_ctr = c.tumbles;
    s.reserved[0] = c.reserved[0];
    s.reserved[1] = c.reserved[1];
}

// A whole simulation in the manner of the reference host driver
// (src/sim.cu:578-618 slot scheme): two phi pools, three S slots.
template <typename R> struct Sim {
    pfb_params2d p;
    int N, L, P;
    long long step;
    std::vector<R> phi[2];
    std::vector<uint32_t> S[3];
    std::vector<Cell<R>> cells;
    uint32_t flags[PFB_FLAG_COUNT];
    std::vector<R> scratch;

    Args<R> args() {
        const int pin = (int)(step % 2), pout = 1 - pin, rs = (int)(step % 3);
        pfb_step_args2d co;
        std::memset(&co, 0, sizeof(co));
        const double A0 = kPi * p.target_radius * p.target_radius;
        Args<R> a;
        a.phi_in = phi[pin].data();
        a.phi_out = phi[pout].data();
        a.S_rd = S[rs].data();
        a.S_sc = S[(rs + 1) % 3].data();
        a.cell = cells.data();
        a.flags = flags;
        a.step = (unsigned long long)step;
        a.N = N;
        a.L = L;
        a.P = P;
        a.parity_out = pout;
        a.dt = (R)p.dt;
        a.A0 = A0;
        a.vol_scale = 2.0 * p.mu / A0;
        a.bulk = (R)(30.0 / (p.lambda * p.lambda));
        a.rep = (R)(60.0 * p.kappa / (p.lambda * p.lambda));
        a.mot = (R)((60.0 * p.kappa / (p.lambda * p.lambda)) / p.xi);
        a.polarity_seed = p.polarity_seed ? p.polarity_seed : p.seed;
        a.p_tumble = -std::expm1(-p.dt / p.tau);
        a.full_moment_every = p.full_moment_every;
        return a;
    }

    void rebuild_S() {
        const int rot = (int)(step % 3), pin = (int)(step % 2);
        for (auto& s : S) std::fill(s.begin(), s.end(), 0u);
        for (int n = 0; n < N; ++n) {
            const Cell<R>& c = cells[(size_t)n];
            const Win w = win(c.cls);
            for (int b = 0; b < w.wy; ++b)
                for (int a = 0; a < w.wx; ++a) {
                    const R v = phi[pin][(size_t)n * kArea + (size_t)(w.ty0 + b) * kPitch + w.tx0 + a];
                    const uint32_t q = q_of<R>(v);
                    if (!q) continue;
                    uint32_t& t = S[rot][(size_t)wrap(c.gy0 + b, L) * P + wrap(c.gx0 + a, L)];
                    if (t > 0xFFFFFFFFu - q) flags[PFB_FLAG_S_OVERFLOW] |= 1u;
                    t += q;
                }
        }
    }

    void advance(long long steps, int threads) {
        for (long long k = 0; k < steps; ++k) {
            Args<R> a = args();
            const int rs = (int)(step % 3);
            // The slot two steps ahead is cleared during the step (reference
            // src/kernels.cu:958-965); whole slot here, as P*L is a multiple of 4.
            std::fill(S[(rs + 2) % 3].begin(), S[(rs + 2) % 3].end(), 0u);
            step_all<R>(a, threads);
            ++step;
        }
    }
};

template <typename R> Sim<R>* make_sim(const pfb_params2d* p, const pfb_cell2d* cells,
                                       const float* phi, const double* phi64, long long step) {
    Sim<R>* s = new Sim<R>();
    s->p = *p;
    s->N = p->num_cells;
    s->L = p->L;
    s->P = 32 * ((p->L + 31) / 32);
    s->step = step;
    std::memset(s->flags, 0, sizeof(s->flags));
    const size_t pool = (size_t)s->N * kArea;
    s->phi[0].assign(pool, (R)0);
    s->phi[1].assign(pool, (R)0);
    const int pin = (int)(step % 2);
    for (size_t i = 0; i < pool; ++i) s->phi[pin][i] = phi64 ? (R)phi64[i] : (R)phi[i];
    for (auto& sl : s->S) sl.assign((size_t)s->P * s->L, 0u);
    s->cells.resize((size_t)s->N);
    for (int i = 0; i < s->N; ++i) {
        s->cells[(size_t)i] = from_abi<R>(cells[i]);
        s->cells[(size_t)i].cls_written[0] = cells[i].cls;
        s->cells[(size_t)i].cls_written[1] = cells[i].cls;
    }
    s->rebuild_S();
    return s;
}

}  // namespace

extern "C" {

// ---- primitives for golden-vector tests ----------------------------------
void oracle_philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                          uint32_t k1, uint32_t* out) {
    philox(c0, c1, c2, c3, k0, k1, out);
}
double oracle_u53(uint32_t a, uint32_t b) { return u53(a, b); }
uint32_t oracle_q_of(float phi) { return q_f(phi); }
float oracle_rhs_f32(float lap, float phi, float So, float gx, float gy, float gam, float dwC,
                     float volC, float repC, float vx, float vy, float mrel) {
    return rhs<float>(lap, phi, So, gx, gy, gam, dwC, volC, repC, vx, vy, mrel);
}
// common/model_coefficients.cuh:23-53, binary32 and binary64:
// out = {bulk, interaction, motility, volume, interface_k, init_radius}
void oracle_coefficients_f32(float lambda, float kappa, float xi, float mu, float target, float* out) {
    out[0] = 30.0f / (lambda * lambda);
    out[1] = 60.0f * kappa / (lambda * lambda);
    out[2] = out[1] / xi;
    out[3] = 2.0f * mu / target;
    out[4] = 2.7386127875258306f / lambda;
    out[5] = target + 0.5f / out[4];
}
void oracle_coefficients_f64(double lambda, double kappa, double xi, double mu, double target,
                             double* out) {
    out[0] = 30.0 / (lambda * lambda);
    out[1] = 60.0 * kappa / (lambda * lambda);
    out[2] = out[1] / xi;
    out[3] = 2.0 * mu / target;
    out[4] = 2.7386127875258306 / lambda;
    out[5] = target + 0.5 / out[4];
}

// ---- one step on caller-owned host buffers (the ABI record layout) --------
// `a` holds HOST pointers; the same semantics as pfb_step2d_launch.
int oracle_step2d_f32(const pfb_step_args2d* a, int threads) {
    if (!a || !a->phi_in || !a->phi_out || !a->S_rd || !a->S_sc || !a->cell || !a->cell_cls ||
        !a->step_rd || !a->step_wr || !a->flags)
        return -1;
    std::vector<Cell<float>> cells((size_t)a->N);
    for (int i = 0; i < a->N; ++i) cells[(size_t)i] = from_abi<float>(a->cell[i]);
    if (a->clear_ahead_words && a->S_cl)
        std::memset(a->S_cl, 0, (size_t)(a->clear_ahead_words >> 2) * 16);
    Args<float> A;
    A.phi_in = a->phi_in;
    A.phi_out = a->phi_out;
    A.S_rd = a->S_rd;
    A.S_sc = a->S_sc;
    A.cell = cells.data();
    A.flags = a->flags;
    A.step = *a->step_rd;
    A.N = a->N;
    A.L = a->L;
    A.P = a->P;
    A.parity_out = a->parity_out;
    A.dt = a->dt;
    A.A0 = a->A0;
    A.vol_scale = a->vol_scale;
    A.bulk = a->bulk_scale;
    A.rep = a->rep_coeff;
    A.mot = a->mot_coeff;
    A.polarity_seed = a->polarity_seed;
    A.p_tumble = a->p_tumble;
    A.full_moment_every = a->full_moment_every;
    // Visit cells in the caller's queue order when given (the result does
    // not depend on it: every update reads only step-n state).
    step_all<float>(A, threads);
    for (int i = 0; i < a->N; ++i) {
        to_abi<float>(cells[(size_t)i], a->cell[i]);
        a->cell_cls[i] = (uint8_t)cells[(size_t)i].cls;
    }
    if (a->cursor_clear) *a->cursor_clear = 0ull;
    *a->step_wr = *a->step_rd + 1ull;
    return 0;
}

// ---- whole-run drivers ----------------------------------------------------
void* oracle_sim_create(const pfb_params2d* p, const pfb_cell2d* cells, const float* phi,
                        long long step, int f64) {
    if (!p || !cells || !phi) return nullptr;
    if (f64) return make_sim<double>(p, cells, phi, nullptr, step);
    return make_sim<float>(p, cells, phi, nullptr, step);
}
void oracle_sim_destroy(void* h, int f64) {
    if (f64)
        delete static_cast<Sim<double>*>(h);
    else
        delete static_cast<Sim<float>*>(h);
}
void oracle_sim_advance(void* h, int f64, long long steps, int threads) {
    if (f64)
        static_cast<Sim<double>*>(h)->advance(steps, threads);
    else
        static_cast<Sim<float>*>(h)->advance(steps, threads);
}
long long oracle_sim_step(void* h, int f64) {
    return f64 ? static_cast<Sim<double>*>(h)->step : static_cast<Sim<float>*>(h)->step;
}
// Cells in the ABI record (binary64 values rounded where the record is f32).
void oracle_sim_get_cells(void* h, int f64, pfb_cell2d* out) {
    if (f64) {
        auto* s = static_cast<Sim<double>*>(h);
        for (int i = 0; i < s->N; ++i) to_abi<double>(s->cells[(size_t)i], out[i]);
    } else {
        auto* s = static_cast<Sim<float>*>(h);
        for (int i = 0; i < s->N; ++i) to_abi<float>(s->cells[(size_t)i], out[i]);
    }
}
// Velocities at full precision of the mode: out[2*i], out[2*i+1].
void oracle_sim_get_velocity(void* h, int f64, double* out) {
    if (f64) {
        auto* s = static_cast<Sim<double>*>(h);
        for (int i = 0; i < s->N; ++i) {
            out[2 * i] = s->cells[(size_t)i].vx;
            out[2 * i + 1] = s->cells[(size_t)i].vy;
        }
    } else {
        auto* s = static_cast<Sim<float>*>(h);
        for (int i = 0; i < s->N; ++i) {
            out[2 * i] = s->cells[(size_t)i].vx;
            out[2 * i + 1] = s->cells[(size_t)i].vy;
        }
    }
}
// phi^step pool as binary64 (N*288*288).
void oracle_sim_get_phi(void* h, int f64, double* out) {
    if (f64) {
        auto* s = static_cast<Sim<double>*>(h);
        const auto& v = s->phi[s->step % 2];
        std::memcpy(out, v.data(), v.size() * sizeof(double));
    } else {
        auto* s = static_cast<Sim<float>*>(h);
        const auto& v = s->phi[s->step % 2];
        for (size_t i = 0; i < v.size(); ++i) out[i] = v[i];
    }
}
void oracle_sim_get_S(void* h, int f64, uint32_t* out) {
    if (f64) {
        auto* s = static_cast<Sim<double>*>(h);
        std::memcpy(out, s->S[s->step % 3].data(), s->S[0].size() * 4);
    } else {
        auto* s = static_cast<Sim<float>*>(h);
        std::memcpy(out, s->S[s->step % 3].data(), s->S[0].size() * 4);
    }
}
void oracle_sim_get_flags(void* h, int f64, uint32_t* out) {
    if (f64)
        std::memcpy(out, static_cast<Sim<double>*>(h)->flags, sizeof(uint32_t) * PFB_FLAG_COUNT);
    else
        std::memcpy(out, static_cast<Sim<float>*>(h)->flags, sizeof(uint32_t) * PFB_FLAG_COUNT);
}

// ---- initial state (reference src/kernels.cu:1050-1165, binary32) ---------
// Fills cells[n].gx0/gy0/cls/cls_written and moments, and phi (N*288*288,
// zeroed first) with the tanh disks of the class-0 window.
void oracle_init_state2d(const pfb_params2d* p, const float* cx, const float* cy,
                         pfb_cell2d* cells, float* phi) {
    const int N = p->num_cells, L = p->L;
    const double k = 2.7386127875258306 / p->lambda;
    const float kf = (float)k;
    const float reff = (float)(p->target_radius + 0.5 / k);
    std::memset(phi, 0, sizeof(float) * (size_t)N * kArea);
    for (int n = 0; n < N; ++n) {
        const Win w = win(cells[n].cls);
        const int gx0 = wrap((int)std::lrint(cx[n] - 0.5f * (float)(w.wx - 1)), L);
        const int gy0 = wrap((int)std::lrint(cy[n] - 0.5f * (float)(w.wy - 1)), L);
        double aV = 0, aCx = 0, aCy = 0;
        int blox = w.wx, bhix = -1, bloy = w.wy, bhiy = -1;
        float pmax = 0.0f;
        for (int b = 0; b < w.wy; ++b)
            for (int a = 0; a < w.wx; ++a) {
                float dx = (float)(gx0 + a) - cx[n], dy = (float)(gy0 + b) - cy[n];
                if (dx > 0.5f * L) dx -= (float)L;
                if (dx < -0.5f * L) dx += (float)L;
                if (dy > 0.5f * L) dy -= (float)L;
                if (dy < -0.5f * L) dy += (float)L;
                const float r = std::sqrt(dx * dx + dy * dy);
                const float v = 0.5f * (1.0f - std::tanh(kf * (r - reff)));
                phi[(size_t)n * kArea + (size_t)(w.ty0 + b) * kPitch + w.tx0 + a] = v;
                const double d = (double)v * v;
                aV += d;
                aCx += d * a;
                aCy += d * b;
                if (std::fabs(v) > pmax) pmax = std::fabs(v);
                if (v > 1e-5f) {
                    if (a < blox) blox = a;
                    if (a > bhix) bhix = a;
                    if (b < bloy) bloy = b;
                    if (b > bhiy) bhiy = b;
                }
            }
        pfb_cell2d& c = cells[n];
        c.gx0 = gx0;
        c.gy0 = gy0;
        c.cls_written[0] = c.cls;
        c.cls_written[1] = c.cls;
        c.V = aV;
        c.Cx = aCx;
        c.Cy = aCy;
        c.bb_lo_x = blox;
        c.bb_hi_x = bhix;
        c.bb_lo_y = bloy;
        c.bb_hi_y = bhiy;
        c.phi_max = pmax;
        c.promote_ctr = 0;
        c.Ix = 0;
        c.Iy = 0;
    }
}

// Q5.27 aggregate of a phi pool (reference src/kernels.cu:1167-1190).
void oracle_scatter_all2d(const float* phi, const pfb_cell2d* cells, int N, int L, int P,
                          uint32_t* S, uint32_t* flags) {
    for (int n = 0; n < N; ++n) {
        const Win w = win(cells[n].cls);
        for (int b = 0; b < w.wy; ++b)
            for (int a = 0; a < w.wx; ++a) {
                const float v = phi[(size_t)n * kArea + (size_t)(w.ty0 + b) * kPitch + w.tx0 + a];
                const uint32_t q = q_f(v);
                if (!q) continue;
                uint32_t& t = S[(size_t)wrap(cells[n].gy0 + b, L) * P + wrap(cells[n].gx0 + a, L)];
                if (t > 0xFFFFFFFFu - q) flags[PFB_FLAG_S_OVERFLOW] |= 1u;
                if (v * v > 4.0f) flags[PFB_FLAG_Q_CLAMP] |= 1u;
                t += q;
            }
    }
}

// ---- fresh-start draws (host code of the reference) -------------------------
// Sequential periodic placement: cell 0 at the box centre, candidates from
// std::mt19937_64 (top 53 bits times 2^-53), accepted centres rounded to
// binary32 before later distance tests, minimum-image separation test
// (include/palmieri_initializer.hpp:48-103). Returns 0, or -1 when the
// placement does not terminate.
int oracle_palmieri_centres(int n, double side, double min_sep, unsigned long long seed,
                            float* x, float* y) {
    if (n < 1 || !(side > 0.0) || !(min_sep > 0.0)) return -1;
    std::mt19937_64 eng(seed);
    auto image = [side](double d) { return d - side * std::floor(d / side + 0.5); };
    x[0] = (float)(0.5 * side);
    y[0] = (float)(0.5 * side);
    int placed = 1;
    for (unsigned long long tries = 0; placed < n; ++tries) {
        if (tries >= 1000000000ull) return -1;
        const double px = side * ((double)(eng() >> 11) * 0x1.0p-53);
        const double py = side * ((double)(eng() >> 11) * 0x1.0p-53);
        int j = 0;
        for (; j < placed; ++j) {
            const double dx = image(px - (double)x[j]), dy = image(py - (double)y[j]);
            if (dx * dx + dy * dy < min_sep * min_sep) break;
        }
        if (j < placed) continue;
        x[placed] = (float)px;
        y[placed] = (float)py;
        ++placed;
    }
    return 0;
}

// Initial polarity angle: Philox4x32-10 on (gid, 2, 0, 0) keyed by the
// polarity stream, theta = (float)(2 pi u53(w0, w1)) (include/kernels.cuh:146-158).
float oracle_ic_theta(int32_t gid, unsigned long long stream) {
    uint32_t w[4];
    philox((uint32_t)gid, 2u, 0u, 0u, (uint32_t)stream, (uint32_t)(stream >> 32), w);
    return (float)(2.0 * kPi * u53(w[0], w[1]));
}

// Initial active speed: lognormal with median v_A from a Box-Muller normal on
// Philox (gid, 3, 0, 0) keyed by the seed (include/kernels.cuh:160-172).
double oracle_ic_v_A(int32_t gid, unsigned long long seed, double v_A, double sigma) {
    if (!(sigma > 0.0)) return v_A;
    uint32_t w[4];
    philox((uint32_t)gid, 3u, 0u, 0u, (uint32_t)seed, (uint32_t)(seed >> 32), w);
    const double u1 = std::max(1e-300, u53(w[0], w[1]));
    const double u2 = u53(w[2], w[3]);
    const double z = std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * kPi * u2);
    return v_A * std::exp(sigma * z);
}

// Cell records of a fresh start: ids, stiffness (the first round(f N) ids
// soft), speed, mobility, target radius and angle (src/sim.cu:136-145, 324-340).
void oracle_fresh_cells2d(const pfb_params2d* p, pfb_cell2d* cells) {
    const int N = p->num_cells;
    const int soft = (int)std::lround(p->cancer_fraction * N);
    const unsigned long long stream = p->polarity_seed ? p->polarity_seed : p->seed;
    std::memset(cells, 0, sizeof(pfb_cell2d) * (size_t)N);
    for (int i = 0; i < N; ++i) {
        pfb_cell2d& c = cells[i];
        c.global_id = i;
        c.gamma = (float)(i < soft ? p->gamma_cancer : p->gamma_normal);
        c.v_A = (float)oracle_ic_v_A(i, p->seed, p->v_A, p->v_A_sigma);
        c.M_pf = (float)p->phase_field_mobility;
        c.R_tgt = (float)p->target_radius;
        c.theta = oracle_ic_theta(i, stream);
    }
}

}  // extern "C"
