// The 2D fused step on sm_100a: one thread-block cluster of K CTAs per cell.
//
// Behaviour follows the reference step (src/kernels.cu:53-592 process_cell,
// :604-937 process_cell_fallback, :948-1024 step_body). The B200 design:
//
//  * A cell's active window is split into K horizontal bands, one per CTA of a
//    cluster (K = 2, 4 or 8), so a small population (64 cells) still fills all
//    148 SMs and a CTA needs ~57 KB of shared memory instead of ~210 KB: three
//    CTAs share an SM and hide each other's latency.
//  * Each CTA stages its band of phi^n (plus a two-row halo) with bulk TMA
//    copies (cp.async.bulk, one per window row, completing on an mbarrier)
//    while thread 0 draws the tumble and chooses the class, and the other warps
//    gather the band of the Q5.27 aggregate S from L2.
//  * The interaction integral and the moments are reduced per CTA (warp
//    butterfly, then ascending warp) and across the cluster through
//    distributed shared memory in ascending rank order, so every CTA derives
//    the same velocity and the result is deterministic run to run.
//  * The Euler update writes phi^{n+1} over the staged S in place; the
//    recentring store, the Q5.27 scatter (integer atomics into L2) and the
//    FP64 moments are fused into one pass over destination rows. Each CTA
//    recomputes a one-row halo of phi^{n+1} so the perimeter and the recentring
//    shift never need a neighbour's band.
//  * Classes 4 and 5 (224^2, 286^2 windows: rare) take a global-memory path
//    with the same cluster split, mirroring the reference's non-staged path.
//
// The grid is N*K CTAs; a cell is owned by one cluster for the whole step.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_util.cuh"
#include "pfb_common.cuh"
#include "pfb_internal.h"

namespace pfb {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kHeaderBytes = 1024;
// Polls of an mbarrier before a CTA gives up (each poll suspends briefly).
constexpr uint32_t kWaitPolls = 1u << 24;

// Error word of the library (device side): bit 0 = a CTA gave up waiting for
// its staged band. Read with pfb_device_status().
__device__ unsigned int g_step2d_status = 0u;

struct __align__(16) StepShared {
    uint64_t bar;
    int abort;
    int gx0, gy0;
    // decided by thread 0 (phase 0)
    int sx, sy, gx0n, gy0n, dcls, zero_tile, fm, pctr, tumbled;
    int dwx, dwy, dtx0, dty0, no_margin;
    float gam, dwC, volC, vA, pcos, psin, theta, mrel;
    float vx, vy;
    // per-warp partials
    double red_d[kWarps][4];
    int red_i[kWarps][5];
    // this CTA's partials, read by rank 0 through distributed shared memory
    double part_I[2];
    double part_M[4];
    int part_B[5];
};
static_assert(sizeof(StepShared) <= kHeaderBytes, "shared header too large");

__host__ __device__ constexpr int band_rows(int wy, int k) { return (wy + k - 1) / k; }

// Rows per work item of the column-rolling passes: balances the 256 threads
// against the (rows + 2) shared loads a column run costs.
__host__ __device__ constexpr int pick_run(int wx, int rows) {
    int best_h = 1;
    long best = -1;
    for (int h = 2; h <= 16; ++h) {
        const int runs = (rows + h - 1) / h;
        const int iters = (wx * runs + kThreads - 1) / kThreads;
        const long cost = (long)iters * (h + 2);
        if (best < 0 || cost < best) {
            best = cost;
            best_h = h;
        }
    }
    return best_h;
}

__host__ __device__ constexpr int staged_bytes(int cls, int k) {
    return kHeaderBytes +
           (band_rows(window_of(cls).wy, k) + 4) * (window_of(cls).wx + 8) * 4 +
           (band_rows(window_of(cls).wy, k) + 2) * window_of(cls).wx * 4;
}

__host__ __device__ constexpr int step_smem_bytes(int k) {
    int m = 0;
    for (int c = 0; c <= 3; ++c) m = staged_bytes(c, k) > m ? staged_bytes(c, k) : m;
    return m;
}

// S_other = (q_S - q(phi)) 2^-27; a negative difference is counted, not
// floored silently (reference src/kernels.cu:19-25).
__device__ __forceinline__ float s_other(uint32_t qS, float phi, uint32_t* flags) {
    const uint32_t qc = q_encode(phi);
    if (qS >= qc) return (float)(qS - qc) * kQInv;
    if (flags) atomicAdd(flags + PFB_FLAG_S_NEGATIVE, 1u);
    return 0.0f;
}

// Tumble, class choice and recentring shift of cell n (reference
// src/kernels.cu:93-191 and :624-711). Run by one thread of every CTA of the
// cluster; all CTAs compute identical values from identical inputs, and only
// the leader raises flags.
template <int CLS>
__device__ __forceinline__ void phase0(const pfb_step_args2d& A, int n, StepShared& sh,
                                       bool leader) {
    constexpr Window W = window_of(CLS);
    const pfb_cell2d& cs = A.cell[n];
    const unsigned long long step = *A.step_rd;

    const Words4 r = philox10((uint32_t)(step & 0xFFFFFFFFull), (uint32_t)(step >> 32),
                              (uint32_t)cs.global_id, kTumbleTag,
                              (uint32_t)(A.polarity_seed & 0xFFFFFFFFull),
                              (uint32_t)(A.polarity_seed >> 32));
    float theta = cs.theta;
    int tumbled = 0;
    if (u53(r.w[0], r.w[1]) < A.p_tumble) {
        theta = (float)(2.0 * kPi * u53(r.w[2], r.w[3]));
        tumbled = 1;
    }
    float ps, pc;
    sincosf(theta, &ps, &pc);

    const float gam = cs.gamma;
    const float dwC = A.bulk_scale * gam;
    const float volC = (float)(A.vol_scale * (A.A0 - cs.V));
    const float mrel = cs.M_pf * (float)(1.0 / kMobilityM0);

    const int ex = cs.bb_hi_x - cs.bb_lo_x + 1;
    const int ey = cs.bb_hi_y - cs.bb_lo_y + 1;
    int dcls = CLS;
    int no_margin = 0;
    unsigned pctr = cs.promote_ctr;
    if (ex > 0) {
        if (ex + kPromoteSlack > W.wx || ey + kPromoteSlack > W.wy) {
            const int grow = smallest_class_holding(ex, ey, kPromoteSlack);
            if (grow >= 0) {
                dcls = grow;
            } else if (CLS == kClassFallback && ex <= W.wx && ey <= W.wy) {
                no_margin = 1;
            } else if (leader) {
                atomicAdd(A.flags + PFB_FLAG_CLASS_EXHAUSTED, 1u);
            }
            pctr = 0u;
        } else {
            const int small = smallest_class_holding(ex, ey, kDemoteSlack);
            if (small >= 0 && small != CLS &&
                window_of(small).wx * window_of(small).wy < W.wx * W.wy) {
                if (++pctr >= (unsigned)kDemoteDwell) {
                    dcls = small;
                    pctr = 0u;
                }
            } else {
                pctr = 0u;
            }
        }
    }
    const Window D = window_of(dcls);

    int sx = 0, sy = 0;
    if (cs.V > 0.0) {
        const double cxr = cs.Cx / cs.V;
        const double cyr = cs.Cy / cs.V;
        sx = __double2int_rn(cxr - 0.5 * (double)(D.wx - 1));
        sy = __double2int_rn(cyr - 0.5 * (double)(D.wy - 1));
        if (dcls == CLS) {
            sx = max(-kMaxShift, min(kMaxShift, sx));
            sy = max(-kMaxShift, min(kMaxShift, sy));
        } else {
            sx = max(-W.wx, min(W.wx, sx));
            sy = max(-W.wy, min(W.wy, sy));
        }
    } else if (leader) {
        atomicOr(A.flags + PFB_FLAG_V_NONPOS, 1u);
    }

    const int L = A.L;
    int gx0n = (cs.gx0 + sx) % L;
    if (gx0n < 0) gx0n += L;
    int gy0n = (cs.gy0 + sy) % L;
    if (gy0n < 0) gy0n += L;

    sh.gx0 = cs.gx0;
    sh.gy0 = cs.gy0;
    sh.sx = sx;
    sh.sy = sy;
    sh.gx0n = gx0n;
    sh.gy0n = gy0n;
    sh.dcls = dcls;
    sh.zero_tile = (dcls != (int)cs.cls_written[A.parity_out]);
    sh.fm = (A.full_moment_every > 0 &&
             ((step + 1ull) % (unsigned long long)A.full_moment_every) == 0ull);
    sh.pctr = (int)pctr;
    sh.tumbled = tumbled;
    sh.dwx = D.wx;
    sh.dwy = D.wy;
    sh.dtx0 = D.tx0;
    sh.dty0 = D.ty0;
    sh.no_margin = no_margin;
    sh.gam = gam;
    sh.dwC = dwC;
    sh.volC = volC;
    sh.vA = cs.v_A;
    sh.pcos = pc;
    sh.psin = ps;
    sh.theta = theta;
    sh.mrel = mrel;
}

// Interaction integral of this CTA -> cluster total -> velocity (all CTAs).
template <int K>
__device__ __forceinline__ void reduce_force(const pfb_step_args2d& A, int n, int rank,
                                             StepShared& sh, double aIx, double aIy) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    aIx = dev::warp_sum_down(aIx);
    aIy = dev::warp_sum_down(aIy);
    if (lane == 0) {
        sh.red_d[warp][0] = aIx;
        sh.red_d[warp][1] = aIy;
    }
    __syncthreads();
    if (tid == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < kWarps; ++w) {
            s0 += sh.red_d[w][0];
            s1 += sh.red_d[w][1];
        }
        sh.part_I[0] = s0;
        sh.part_I[1] = s1;
    }
    dev::cluster_sync();
    if (tid == 0) {
        double sIx = 0.0, sIy = 0.0;
        const uint32_t base = dev::smem_addr(&sh.part_I[0]);
        for (int r = 0; r < K; ++r) {
            const uint32_t a = dev::map_to_rank(base, (uint32_t)r);
            sIx += dev::ld_cluster_f64(a);
            sIy += dev::ld_cluster_f64(a + 8);
        }
        const double vxd = (double)sh.vA * (double)sh.pcos + (double)A.mot_coeff * sIx;
        const double vyd = (double)sh.vA * (double)sh.psin + (double)A.mot_coeff * sIy;
        sh.vx = (float)vxd;
        sh.vy = (float)vyd;
        if (rank == 0) {
            pfb_cell2d& cs = A.cell[n];
            cs.vx = (float)vxd;
            cs.vy = (float)vyd;
            cs.Ix = sIx;
            cs.Iy = sIy;
        }
    }
    __syncthreads();
}

// Moments of this CTA -> cluster total -> commit by rank 0 (reference
// src/kernels.cu:542-590 and :883-935).
template <int K, bool FALLBACK>
__device__ __forceinline__ void reduce_commit(const pfb_step_args2d& A, int n, int rank,
                                              StepShared& sh, double aV, double aCx,
                                              double aCy, double aPer, int blox, int bhix,
                                              int bloy, int bhiy, int pmaxb) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    aV = dev::warp_sum_down(aV);
    aCx = dev::warp_sum_down(aCx);
    aCy = dev::warp_sum_down(aCy);
    aPer = dev::warp_sum_down(aPer);
    blox = dev::warp_min_down(blox);
    bhix = dev::warp_max_down(bhix);
    bloy = dev::warp_min_down(bloy);
    bhiy = dev::warp_max_down(bhiy);
    pmaxb = dev::warp_max_down(pmaxb);
    if (lane == 0) {
        sh.red_d[warp][0] = aV;
        sh.red_d[warp][1] = aCx;
        sh.red_d[warp][2] = aCy;
        sh.red_d[warp][3] = aPer;
        sh.red_i[warp][0] = blox;
        sh.red_i[warp][1] = bhix;
        sh.red_i[warp][2] = bloy;
        sh.red_i[warp][3] = bhiy;
        sh.red_i[warp][4] = pmaxb;
    }
    __syncthreads();
    if (tid == 0) {
        double m[4] = {0.0, 0.0, 0.0, 0.0};
        int b[5] = {sh.dwx, -1, sh.dwy, -1, 0};
        for (int w = 0; w < kWarps; ++w) {
            for (int k = 0; k < 4; ++k) m[k] += sh.red_d[w][k];
            b[0] = min(b[0], sh.red_i[w][0]);
            b[1] = max(b[1], sh.red_i[w][1]);
            b[2] = min(b[2], sh.red_i[w][2]);
            b[3] = max(b[3], sh.red_i[w][3]);
            b[4] = max(b[4], sh.red_i[w][4]);
        }
        for (int k = 0; k < 4; ++k) sh.part_M[k] = m[k];
        for (int k = 0; k < 5; ++k) sh.part_B[k] = b[k];
    }
    dev::cluster_sync();
    if (rank == 0 && tid == 0) {
        double m[4] = {0.0, 0.0, 0.0, 0.0};
        int b[5] = {sh.dwx, -1, sh.dwy, -1, 0};
        const uint32_t bm = dev::smem_addr(&sh.part_M[0]);
        const uint32_t bb = dev::smem_addr(&sh.part_B[0]);
        for (int r = 0; r < K; ++r) {
            const uint32_t am = dev::map_to_rank(bm, (uint32_t)r);
            const uint32_t ab = dev::map_to_rank(bb, (uint32_t)r);
            for (int k = 0; k < 4; ++k) m[k] += dev::ld_cluster_f64(am + 8u * k);
            b[0] = min(b[0], dev::ld_cluster_s32(ab + 0));
            b[1] = max(b[1], dev::ld_cluster_s32(ab + 4));
            b[2] = min(b[2], dev::ld_cluster_s32(ab + 8));
            b[3] = max(b[3], dev::ld_cluster_s32(ab + 12));
            b[4] = max(b[4], dev::ld_cluster_s32(ab + 16));
        }
        pfb_cell2d& cs = A.cell[n];
        const int dcls = sh.dcls;
        cs.gx0 = sh.gx0n;
        cs.gy0 = sh.gy0n;
        cs.cls = (uint8_t)dcls;
        cs.cls_written[A.parity_out] = (uint8_t)dcls;
        cs.theta = sh.theta;
        cs.V = m[0];
        cs.Cx = m[1];
        cs.Cy = m[2];
        if (sh.fm) cs.perim = m[3];
        cs.bb_lo_x = b[0];
        cs.bb_hi_x = b[1];
        cs.bb_lo_y = b[2];
        cs.bb_hi_y = b[3];
        cs.promote_ctr = (uint32_t)sh.pctr;
        cs.shift_ctr += (sh.sx | sh.sy) ? 1u : 0u;
        cs.tumble_ctr += (uint32_t)sh.tumbled;
        cs.phi_max = __uint_as_float((uint32_t)b[4]);
        A.cell_cls[n] = (uint8_t)dcls;
        if (FALLBACK) {
            const bool edge = b[1] >= 0 &&
                              (b[0] == 0 || b[1] == sh.dwx - 1 || b[2] == 0 || b[3] == sh.dwy - 1);
            cs.reserved[0] = 1u;
            if (sh.no_margin || (dcls == kClassFallback && edge)) ++cs.reserved[1];
        }
    }
    // Keep every CTA's shared memory alive until rank 0 has read it.
    dev::cluster_sync();
}

// Flags, phi_max, Q5.27 scatter and moments of one destination pixel.
struct PixelAcc {
    double V = 0.0, Cx = 0.0, Cy = 0.0, Per = 0.0;
    int blox, bhix = -1, bloy, bhiy = -1, pmaxb = 0;
};

__device__ __forceinline__ void dest_pixel(const pfb_step_args2d& A, PixelAcc& acc, float pn,
                                           int a, int b, uint32_t* srow, int gx0n, int L) {
    if (!isfinite(pn)) atomicOr(A.flags + PFB_FLAG_NONFINITE, 1u);
    if (pn * pn > kPhiSqCap) atomicOr(A.flags + PFB_FLAG_Q_CLAMP, 1u);
    acc.pmaxb = max(acc.pmaxb, (int)__float_as_uint(fabsf(pn)));
    const uint32_t q = q_encode(pn);
    if (q) {
        int gx = gx0n + a;
        if (gx >= L) gx -= L;
        const uint32_t old = atomicAdd(srow + gx, q);
        if (old > 0xFFFFFFFFu - q) atomicOr(A.flags + PFB_FLAG_S_OVERFLOW, 1u);
    }
    const double d = (double)pn * (double)pn;
    acc.V += d;
    acc.Cx += d * (double)a;
    acc.Cy += d * (double)b;
    if (pn > kSupportEps) {
        acc.blox = min(acc.blox, a);
        acc.bhix = max(acc.bhix, a);
        acc.bloy = min(acc.bloy, b);
        acc.bhiy = max(acc.bhiy, b);
    }
}

// ---------------------------------------------------------------------------
// Staged path: classes 0-3.
// Shared layout after the header:
//   phi_s [RB+4][WX+8] f32 : window rows y0-2 .. y0+RB+1; column x at 4+x,
//                            columns -1 and WX are the synthesized zero ring
//   ps_s  [RB+2][WX]  u32  : window rows y0-1 .. y0+RB; holds q_S, then
//                            phi^{n+1} written in place
// ---------------------------------------------------------------------------
template <int CLS, int K>
__device__ __forceinline__ void staged_cell(const pfb_step_args2d& A, int n, int rank,
                                            char* smem) {
    constexpr Window W = window_of(CLS);
    constexpr int WX = W.wx, WY = W.wy, TX0 = W.tx0, TY0 = W.ty0;
    constexpr int RB = band_rows(WY, K);
    constexpr int PX = WX + 8;
    constexpr int PHI_ROWS = RB + 4;
    static_assert(WY % K == 0, "staged classes split into equal bands");
    static_assert((WX * 4) % 16 == 0 && (TX0 * 4) % 16 == 0, "bulk copies need 16-B rows");

    StepShared& sh = *reinterpret_cast<StepShared*>(smem);
    float* phi_s = reinterpret_cast<float*>(smem + kHeaderBytes);
    uint32_t* ps_s = reinterpret_cast<uint32_t*>(smem + kHeaderBytes + PHI_ROWS * PX * 4);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int y0 = rank * RB;
    const int y1 = y0 + RB;
    const float* tile_in = A.phi_in + (size_t)n * kTileArea;
    const int L = A.L, P = A.P;

    if (tid == 0) {
        sh.abort = 0;
        sh.gx0 = A.cell[n].gx0;
        sh.gy0 = A.cell[n].gy0;
        dev::mbar_init(&sh.bar, 1);
    }
    __syncthreads();

    const int ra = max(0, y0 - 2), rb = min(WY, y1 + 2);
    if (warp == 0) {
        if (lane == 0) dev::mbar_arrive_expect_tx(&sh.bar, (uint32_t)((rb - ra) * WX * 4));
        __syncwarp();
        for (int y = ra + lane; y < rb; y += 32)
            dev::bulk_g2s(phi_s + (y - y0 + 2) * PX + 4,
                          tile_in + (size_t)(TY0 + y) * kTilePitch + TX0, (uint32_t)(WX * 4),
                          &sh.bar);
        if (lane == 0) phase0<CLS>(A, n, sh, rank == 0);
    } else {
        const int t = tid - 32;
        constexpr int NT = kThreads - 32;
        const int gx0 = sh.gx0, gy0 = sh.gy0;
        const int split = min(WX, L - gx0);
        const int sa = max(0, y0 - 1), sb = min(WY, y1 + 1);
        const int cnt = (sb - sa) * WX;
        for (int idx = t; idx < cnt; idx += NT) {
            const int yy = idx / WX;
            const int x = idx - yy * WX;
            const int y = sa + yy;
            int gy = gy0 + y;
            if (gy >= L) gy -= L;
            const int gx = x < split ? gx0 + x : x - split;
            ps_s[(y - y0 + 1) * WX + x] = __ldg(A.S_rd + (size_t)gy * P + gx);
        }
        // Zero ring columns of in-window rows; whole rows outside the window.
        for (int k = t; k < PHI_ROWS; k += NT) {
            const int y = y0 - 2 + k;
            if (y >= 0 && y < WY) {
                phi_s[k * PX + 3] = 0.0f;
                phi_s[k * PX + 4 + WX] = 0.0f;
            }
        }
        for (int k = 0; k < PHI_ROWS; ++k) {
            const int y = y0 - 2 + k;
            if (y >= 0 && y < WY) continue;
            for (int c = t; c < PX; c += NT) phi_s[k * PX + c] = 0.0f;
        }
    }
    if (!dev::mbar_wait_bounded(&sh.bar, 0, kWaitPolls)) {
        sh.abort = 1;
        atomicOr(&g_step2d_status, 1u);
    }
    __syncthreads();
    const bool abort = sh.abort != 0;

    // ---- pass 1: interaction integral over own rows
    double aIx = 0.0, aIy = 0.0;
    if (!abort) {
        constexpr int H = pick_run(WX, RB);
        constexpr int RUNS = (RB + H - 1) / H;
        for (int item = tid; item < WX * RUNS; item += kThreads) {
            const int c = item / WX;
            const int x = item - c * WX;
            const int ya = y0 + c * H;
            const int yb = min(y1, ya + H);
            const float* p = phi_s + (ya - y0 + 2) * PX + 4 + x;
            const uint32_t* q = ps_s + (ya - y0 + 1) * WX + x;
            float sC = p[-PX];
            float cW = p[-1], cC = p[0], cE = p[1];
            for (int y = ya; y < yb; ++y) {
                const float nC = p[PX];
                const float So = s_other(*q, cC, A.flags);
                const float gx = 0.5f * (cE - cW);
                const float gy = 0.5f * (nC - sC);
                aIx += (double)(cC * gx * So);
                aIy += (double)(cC * gy * So);
                p += PX;
                q += WX;
                sC = cC;
                cC = nC;
                cW = p[-1];
                cE = p[1];
            }
        }
    }
    reduce_force<K>(A, n, rank, sh, aIx, aIy);

    // ---- pass 2: Euler update of own rows plus a one-row halo, in place
    if (!abort) {
        const float gam = sh.gam, dwC = sh.dwC, volC = sh.volC;
        const float vx = sh.vx, vy = sh.vy, mrel = sh.mrel;
        const float repC = A.rep_coeff, dtf = A.dt;
        const int ua = max(0, y0 - 1), ub = min(WY, y1 + 1);
        constexpr int H = pick_run(WX, RB + 2);
        constexpr int RUNS = (RB + 2 + H - 1) / H;
        for (int item = tid; item < WX * RUNS; item += kThreads) {
            const int c = item / WX;
            const int x = item - c * WX;
            const int ya = ua + c * H;
            if (ya >= ub) continue;
            const int yb = min(ub, ya + H);
            const float* p = phi_s + (ya - y0 + 2) * PX + 4 + x;
            uint32_t* q = ps_s + (ya - y0 + 1) * WX + x;
            float sW = p[-PX - 1], sC = p[-PX], sE = p[-PX + 1];
            float cW = p[-1], cC = p[0], cE = p[1];
            for (int y = ya; y < yb; ++y) {
                const float nW = p[PX - 1], nC = p[PX], nE = p[PX + 1];
                const float lap = lap9(nW, nC, nE, cW, cC, cE, sW, sC, sE);
                const float gx = 0.5f * (cE - cW);
                const float gy = 0.5f * (nC - sC);
                const bool own = (y >= y0) && (y < y1);
                const float So = s_other(*q, cC, own ? A.flags : nullptr);
                const float rhs =
                    rhs_pixel(lap, cC, So, gx, gy, gam, dwC, volC, repC, vx, vy, mrel);
                const float pnew = cC + dtf * rhs;
                *q = __float_as_uint(pnew);
                sW = cW;
                sC = cC;
                sE = cE;
                cW = nW;
                cC = nC;
                cE = nE;
                p += PX;
                q += WX;
            }
        }
    }
    __syncthreads();

    // ---- pass 3: recentring store, scatter, moments over owned destination rows
    PixelAcc acc;
    acc.blox = sh.dwx;
    acc.bloy = sh.dwy;
    if (!abort) {
        const int sx = sh.sx, sy = sh.sy;
        const int dwx = sh.dwx, dwy = sh.dwy, dtx0 = sh.dtx0, dty0 = sh.dty0;
        const int gx0n = sh.gx0n, gy0n = sh.gy0n;
        const bool fm = sh.fm != 0;
        float* tile_out = A.phi_out + (size_t)n * kTileArea;
        // Destination row b reads source row j = b + sy; rows above the window
        // belong to rank 0, rows below it to rank K-1.
        const int jlo = (rank == 0) ? -(1 << 20) : y0;
        const int jhi = (rank == K - 1) ? (1 << 20) : y1;
        const int b_lo = max(0, jlo - sy), b_hi = min(dwy, jhi - sy);

        if (sh.zero_tile) {
            for (int b = b_lo + warp; b < b_hi; b += kWarps) {
                float* trow = tile_out + (size_t)(dty0 + b) * kTilePitch;
                for (int c = lane; c < kTilePitch; c += 32)
                    if (c < dtx0 || c >= dtx0 + dwx) trow[c] = 0.0f;
            }
            for (int t = rank + K * warp; t < kTilePitch; t += K * kWarps) {
                if (t >= dty0 && t < dty0 + dwy) continue;
                float* trow = tile_out + (size_t)t * kTilePitch;
                for (int c = lane; c < kTilePitch; c += 32) trow[c] = 0.0f;
            }
        }

        for (int b = b_lo + warp; b < b_hi; b += kWarps) {
            const int j = b + sy;
            const bool jin = (unsigned)j < (unsigned)WY;
            const int jr = j - y0 + 1;  // ps_s row of source row j
            int gy = gy0n + b;
            if (gy >= L) gy -= L;
            float* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
            uint32_t* srow = A.S_sc + (size_t)gy * P;
            for (int a = lane; a < dwx; a += 32) {
                const int i = a + sx;
                const bool iin = (unsigned)i < (unsigned)WX;
                const float pn = (jin && iin) ? __uint_as_float(ps_s[jr * WX + i]) : 0.0f;
                __stcs(orow + a, pn);
                dest_pixel(A, acc, pn, a, b, srow, gx0n, L);
                if (fm) {
                    float e = 0.0f, w = 0.0f, nn = 0.0f, ss = 0.0f;
                    if (jin) {
                        if ((unsigned)(i + 1) < (unsigned)WX) e = __uint_as_float(ps_s[jr * WX + i + 1]);
                        if ((unsigned)(i - 1) < (unsigned)WX) w = __uint_as_float(ps_s[jr * WX + i - 1]);
                    }
                    if (iin) {
                        if ((unsigned)(j + 1) < (unsigned)WY)
                            nn = __uint_as_float(ps_s[(jr + 1) * WX + i]);
                        if ((unsigned)(j - 1) < (unsigned)WY)
                            ss = __uint_as_float(ps_s[(jr - 1) * WX + i]);
                    }
                    const float pgx = 0.5f * (e - w), pgy = 0.5f * (nn - ss);
                    acc.Per += (double)sqrtf(pgx * pgx + pgy * pgy);
                }
            }
        }
    }
    reduce_commit<K, false>(A, n, rank, sh, acc.V, acc.Cx, acc.Cy, acc.Per, acc.blox, acc.bhix,
                            acc.bloy, acc.bhiy, acc.pmaxb);
    if (abort) (void)dev::mbar_wait_bounded(&sh.bar, 0, kWaitPolls);
}

// ---------------------------------------------------------------------------
// Global-memory path: classes 4 (224^2) and 5 (286^2 fallback). phi^n is read
// from the tile (its zero ring is the tile invariant), phi^{n+1} is written to
// the shifted destination in global memory, and after a cluster barrier each
// CTA re-reads its destination rows for the scatter and moments (reference
// src/kernels.cu:344-443 and :604-937).
// ---------------------------------------------------------------------------
template <int CLS, int K>
__device__ __noinline__ void global_cell(const pfb_step_args2d& A, int n, int rank, char* smem) {
    constexpr Window W = window_of(CLS);
    constexpr int WX = W.wx, WY = W.wy, TX0 = W.tx0, TY0 = W.ty0;
    constexpr int RB = band_rows(WY, K);
    StepShared& sh = *reinterpret_cast<StepShared*>(smem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int y0 = rank * RB;
    const int y1 = min(WY, y0 + RB);
    const int L = A.L, P = A.P;
    const float* tin = A.phi_in + (size_t)n * kTileArea + (size_t)TY0 * kTilePitch + TX0;
    float* tile_out = A.phi_out + (size_t)n * kTileArea;

    if (tid == 0) phase0<CLS>(A, n, sh, rank == 0);
    __syncthreads();
    const int gx0 = sh.gx0, gy0 = sh.gy0;
    const int split = min(WX, L - gx0);

    double aIx = 0.0, aIy = 0.0;
    const int cnt = (y1 - y0) * WX;
    for (int idx = tid; idx < cnt; idx += kThreads) {
        const int yy = idx / WX;
        const int x = idx - yy * WX;
        const int y = y0 + yy;
        const float* p = tin + (size_t)y * kTilePitch + x;
        const float c = __ldg(p);
        const float gx = 0.5f * (__ldg(p + 1) - __ldg(p - 1));
        const float gyv = 0.5f * (__ldg(p + kTilePitch) - __ldg(p - kTilePitch));
        int gy = gy0 + y;
        if (gy >= L) gy -= L;
        const int gxg = x < split ? gx0 + x : x - split;
        const float So = s_other(__ldg(A.S_rd + (size_t)gy * P + gxg), c, A.flags);
        aIx += (double)(c * gx * So);
        aIy += (double)(c * gyv * So);
    }
    reduce_force<K>(A, n, rank, sh, aIx, aIy);

    const int sx = sh.sx, sy = sh.sy;
    const int dwx = sh.dwx, dwy = sh.dwy, dtx0 = sh.dtx0, dty0 = sh.dty0;
    if (sh.zero_tile) {
        for (int t = rank + K * warp; t < kTilePitch; t += K * kWarps) {
            float* trow = tile_out + (size_t)t * kTilePitch;
            for (int c = lane; c < kTilePitch; c += 32) trow[c] = 0.0f;
        }
        dev::cluster_sync();
    }

    {
        const float gam = sh.gam, dwC = sh.dwC, volC = sh.volC;
        const float vx = sh.vx, vy = sh.vy, mrel = sh.mrel;
        const float repC = A.rep_coeff, dtf = A.dt;
        for (int idx = tid; idx < cnt; idx += kThreads) {
            const int yy = idx / WX;
            const int x = idx - yy * WX;
            const int y = y0 + yy;
            const float* p = tin + (size_t)y * kTilePitch + x;
            const float cC = __ldg(p), cW = __ldg(p - 1), cE = __ldg(p + 1);
            const float nC = __ldg(p + kTilePitch), nW = __ldg(p + kTilePitch - 1),
                        nE = __ldg(p + kTilePitch + 1);
            const float sC = __ldg(p - kTilePitch), sW = __ldg(p - kTilePitch - 1),
                        sE = __ldg(p - kTilePitch + 1);
            const float lap = lap9(nW, nC, nE, cW, cC, cE, sW, sC, sE);
            const float gx = 0.5f * (cE - cW);
            const float gyv = 0.5f * (nC - sC);
            int gy = gy0 + y;
            if (gy >= L) gy -= L;
            const int gxg = x < split ? gx0 + x : x - split;
            const float So = s_other(__ldg(A.S_rd + (size_t)gy * P + gxg), cC, A.flags);
            const float rhs =
                rhs_pixel(lap, cC, So, gx, gyv, gam, dwC, volC, repC, vx, vy, mrel);
            const float pnew = cC + dtf * rhs;
            const int a = x - sx, b = y - sy;
            if ((unsigned)a < (unsigned)dwx && (unsigned)b < (unsigned)dwy)
                tile_out[(size_t)(dty0 + b) * kTilePitch + dtx0 + a] = pnew;
        }
    }
    const int DB = (dwy + K - 1) / K;
    const int db0 = min(dwy, rank * DB), db1 = min(dwy, db0 + DB);
    for (int b = db0 + warp; b < db1; b += kWarps) {
        const int j = b + sy;
        const bool jin = (unsigned)j < (unsigned)WY;
        float* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
        for (int a = lane; a < dwx; a += 32) {
            const int i = a + sx;
            if (!(jin && (unsigned)i < (unsigned)WX)) orow[a] = 0.0f;
        }
    }
    dev::cluster_sync();

    PixelAcc acc;
    acc.blox = dwx;
    acc.bloy = dwy;
    const int gx0n = sh.gx0n, gy0n = sh.gy0n;
    const bool fm = sh.fm != 0;
    for (int b = db0 + warp; b < db1; b += kWarps) {
        int gy = gy0n + b;
        if (gy >= L) gy -= L;
        const float* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
        uint32_t* srow = A.S_sc + (size_t)gy * P;
        for (int a = lane; a < dwx; a += 32) {
            const float pn = __ldcg(orow + a);
            dest_pixel(A, acc, pn, a, b, srow, gx0n, L);
            if (fm) {
                const float e = a + 1 < dwx ? __ldcg(orow + a + 1) : 0.0f;
                const float w = a > 0 ? __ldcg(orow + a - 1) : 0.0f;
                const float nn = b + 1 < dwy ? __ldcg(orow + kTilePitch + a) : 0.0f;
                const float ss = b > 0 ? __ldcg(orow - kTilePitch + a) : 0.0f;
                const float pgx = 0.5f * (e - w), pgy = 0.5f * (nn - ss);
                acc.Per += (double)sqrtf(pgx * pgx + pgy * pgy);
            }
        }
    }
    reduce_commit<K, CLS == kClassFallback>(A, n, rank, sh, acc.V, acc.Cx, acc.Cy, acc.Per,
                                            acc.blox, acc.bhix, acc.bloy, acc.bhiy, acc.pmaxb);
}

template <int K>
__global__ void __launch_bounds__(kThreads, (K >= 8 ? 4 : 3))
    k_step2d(const __grid_constant__ pfb_step_args2d A) {
    extern __shared__ __align__(128) char smem[];
    const int tid = threadIdx.x;

    // Clear the S slot two steps ahead with streaming stores (the kernel does
    // not otherwise touch it).
    if (A.clear_ahead_words) {
        uint4* dst = reinterpret_cast<uint4*>(A.S_cl);
        const size_t nvec = (size_t)(A.clear_ahead_words >> 2);
        const size_t stride = (size_t)gridDim.x * kThreads;
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (size_t i = (size_t)blockIdx.x * kThreads + tid; i < nvec; i += stride)
            __stcs(dst + i, z);
    }
    if (blockIdx.x == 0 && tid == 0) {
        if (A.cursor_clear) *A.cursor_clear = 0ull;
        *A.step_wr = *A.step_rd + 1ull;
    }

    const int rank = (int)dev::cluster_rank();
    const int slot = (int)(blockIdx.x / K);
    const int n = A.perm ? (int)A.perm[slot] : slot;
    const int cls = (int)A.cell_cls[n];
    switch (cls) {
        case 0: staged_cell<0, K>(A, n, rank, smem); break;
        case 1: staged_cell<1, K>(A, n, rank, smem); break;
        case 2: staged_cell<2, K>(A, n, rank, smem); break;
        case 3: staged_cell<3, K>(A, n, rank, smem); break;
        case 4: global_cell<4, K>(A, n, rank, smem); break;
        case 5: global_cell<5, K>(A, n, rank, smem); break;
        default:
            if (rank == 0 && tid == 0) atomicAdd(A.flags + PFB_FLAG_CLASS_UNSUPPORTED, 1u);
            break;
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
template <int K>
static cudaError_t configure_one() {
    cudaError_t e = cudaFuncSetAttribute(k_step2d<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         step_smem_bytes(K));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_step2d<K>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

int step2d_configure_device() {
    static int configured_mask[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(PFB_E_CUDA, "cudaGetDevice failed");
    if (dev >= 0 && dev < 64 && configured_mask[dev]) return PFB_OK;
    cudaError_t e;
    if ((e = configure_one<2>()) != cudaSuccess || (e = configure_one<4>()) != cudaSuccess ||
        (e = configure_one<8>()) != cudaSuccess)
        return set_error(PFB_E_CUDA, "step kernel attribute: %s", cudaGetErrorString(e));
    if (dev >= 0 && dev < 64) configured_mask[dev] = 1;
    return PFB_OK;
}

int step2d_smem_bytes(int k) { return step_smem_bytes(k); }

template <int K>
static cudaError_t launch_k(const pfb_step_args2d& A, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(A.N * K), 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = (size_t)step_smem_bytes(K);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_step2d<K>, A);
}

int step2d_launch(const pfb_step_args2d* a, int cluster, cudaStream_t stream) {
    if (!a) return set_error(PFB_E_ARG, "null step arguments");
    const pfb_step_args2d& A = *a;
    if (!A.phi_in || !A.phi_out || !A.S_rd || !A.S_sc || !A.cell || !A.cell_cls || !A.step_rd ||
        !A.step_wr || !A.flags)
        return set_error(PFB_E_ARG, "null buffer in step arguments");
    if (A.clear_ahead_words && !A.S_cl) return set_error(PFB_E_ARG, "clear-ahead needs S_cl");
    if (((uintptr_t)A.phi_in & 15u) || ((uintptr_t)A.phi_out & 15u) ||
        ((uintptr_t)A.S_cl & 15u))
        return set_error(PFB_E_ARG, "phi pools and S_cl must be 16-byte aligned");
    if (A.moments) return set_error(PFB_E_ARG, "velocity observation is not supported");
    if (A.N < 0) return set_error(PFB_E_ARG, "negative cell count");
    if (A.L <= 286 || A.P < A.L) return set_error(PFB_E_ARG, "domain side must exceed 286 and P >= L");
    if (A.parity_out != 0 && A.parity_out != 1) return set_error(PFB_E_ARG, "parity_out must be 0 or 1");
    if (cluster == 0) cluster = 4;
    if (cluster != 2 && cluster != 4 && cluster != 8)
        return set_error(PFB_E_CONFIG, "cluster must be 2, 4 or 8");
    if (A.N == 0) return PFB_OK;
    int rc = step2d_configure_device();
    if (rc) return rc;
    cudaError_t e = cluster == 2   ? launch_k<2>(A, stream)
                    : cluster == 4 ? launch_k<4>(A, stream)
                                   : launch_k<8>(A, stream);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "step launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int step2d_read_status(unsigned* out, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_step2d_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status read: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_step2d_status, &z, sizeof(z));
    }
    if (out) *out = v;
    return PFB_OK;
}

}  // namespace pfb
