// Persistent, pipelined 2D step on sm_100a: a fixed grid of 8-CTA clusters,
// each walking a strided list of cells.
//
// Same update as the per-cell kernel (step2d.cu) and the reference
// (src/kernels.cu:53-592), organised for the B200:
//
//  * The cluster's eight CTAs split a cell's window into eight row bands.
//    Each CTA stages its band of phi^n (two halo rows) and of the aggregate S
//    (one halo row) with bulk TMA copies into one of two shared buffers, so
//    the copy of the next cell overlaps the arithmetic on the current one.
//  * The per-cell decisions (tumble, class, shift) are made for up to 32 cells
//    at once, one lane per cell, while the first copies are in flight.
//  * Each thread owns a 4-wide column strip of H rows and keeps the 3x6
//    rolling stencil values and S_other in registers: the Euler update reads
//    no shared memory. Off full-moment steps the update, the store of
//    phi^{n+1} (128-bit stores), the Q5.27 scatter and the FP64 moments are
//    one pass; on full-moment steps phi^{n+1} goes through shared memory for
//    the perimeter, as in the per-cell kernel.
//  * Reductions: warp butterfly, ascending warps, ascending cluster ranks via
//    distributed shared memory (partials double-buffered by cell parity, one
//    cluster barrier per reduction).
#include <cuda_runtime.h>

#include <cstdint>

#include "device_util.cuh"
#include "pfb_common.cuh"
#include "pfb_internal.h"
#include "step2d_common.cuh"

namespace pfb {

namespace {

constexpr int kPK = 8;          // CTAs per cluster
constexpr int kPWarps = 7;
constexpr int kPThreads = kPWarps * 32;
constexpr int kPlanBatch = 32;
constexpr int kPHeader = 4096;

__device__ unsigned int g_persist_status = 0u;

struct __align__(16) PersistShared {
    uint64_t bar[2];
    int abort;
    CellPlan plan[kPlanBatch];
    RedScratch<kPWarps> red;
};
static_assert(sizeof(PersistShared) <= kPHeader, "persistent header too large");

// Band geometry of a staged class with eight CTAs per cell.
__host__ __device__ constexpr int prows(int cls) { return window_of(cls).wy / kPK; }
__host__ __device__ constexpr int ppitch(int cls) { return window_of(cls).wx + 8; }
__host__ __device__ constexpr int pbuf_bytes(int cls) {
    return ((prows(cls) + 4) + (prows(cls) + 2)) * ppitch(cls) * 4;
}
__host__ __device__ constexpr int pbuf_max() {
    int m = 0;
    for (int c = 0; c <= 3; ++c) m = pbuf_bytes(c) > m ? pbuf_bytes(c) : m;
    return m;
}
constexpr int kPBuf = (pbuf_max() + 127) / 128 * 128;
constexpr int kPSmem = kPHeader + 2 * kPBuf;

// Thread map of the register stencil: NQ quads per row, G groups of H rows.
template <int CLS> struct PMap {
    static constexpr int WX = window_of(CLS).wx;
    static constexpr int WY = window_of(CLS).wy;
    static constexpr int RB = WY / kPK;
    static constexpr int NQ = WX / 4;
    static constexpr int GMAX = kPThreads / NQ;
    static constexpr int H = (RB + GMAX - 1) / GMAX;
    static constexpr int G = (RB + H - 1) / H;
    static_assert(WY % kPK == 0 && WX % 4 == 0, "band layout");
    static_assert(NQ * G <= kPThreads, "thread map");
};

// Decisions for one cell, kept out of line: it runs once per cell in one lane.
__device__ __noinline__ void plan_cell_lane(const pfb_step_args2d& A, int n, int cls,
                                            unsigned long long step, CellPlan& out, bool leader) {
    plan_cell(A, n, cls, step, out, leader);
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Issue the bulk copies of cell n's band into buffer `b` (warp 0 only).
// Returns through `s_tma` whether S was staged by TMA too (L % 4 == 0).
__device__ __forceinline__ void prefetch_band(const pfb_step_args2d& A, int n, int cls, int rank,
                                              char* buf, uint64_t* bar) {
    const int lane = threadIdx.x & 31;
    const Window W = window_of(cls);
    const int RB = W.wy / kPK, PX = W.wx + 8;
    const int y0 = rank * RB, y1 = y0 + RB;
    const int L = A.L, P = A.P;
    const bool s_tma = (L & 3) == 0;
    const int gx0 = A.cell[n].gx0, gy0 = A.cell[n].gy0;
    const int soff = s_tma ? (gx0 & 3) : 0;
    const int gxa = gx0 - soff;
    const bool wrap = gx0 + W.wx > L;
    float* phi_s = reinterpret_cast<float*>(buf);
    uint32_t* s_s = reinterpret_cast<uint32_t*>(buf + (RB + 4) * PX * 4);
    const float* tile = A.phi_in + (size_t)n * kTileArea;
    const int ra = max(0, y0 - 2), rb = min(W.wy, y1 + 2);
    const int sa = max(0, y0 - 1), sb = min(W.wy, y1 + 1);
    // copy lengths in words of one S row
    int n1, n2;
    if (!wrap) {
        n1 = min((soff + W.wx + 3) & ~3, P - gxa);
        n2 = 0;
    } else {
        n1 = L - gxa;
        n2 = (gx0 + W.wx - L + 3) & ~3;
    }
    uint32_t bytes = 0;
    for (int y = ra + lane; y < rb; y += 32) bytes += (uint32_t)(W.wx * 4);
    if (s_tma)
        for (int y = sa + lane; y < sb; y += 32) bytes += (uint32_t)((n1 + n2) * 4);
    bytes = __reduce_add_sync(0xFFFFFFFFu, bytes);
    fence_proxy_async();
    if (lane == 0) dev::mbar_arrive_expect_tx(bar, bytes);
    __syncwarp();
    for (int y = ra + lane; y < rb; y += 32)
        dev::bulk_g2s(phi_s + (y - y0 + 2) * PX + 4,
                      tile + (size_t)(W.ty0 + y) * kTilePitch + W.tx0, (uint32_t)(W.wx * 4), bar);
    if (s_tma) {
        for (int y = sa + lane; y < sb; y += 32) {
            int gy = gy0 + y;
            if (gy >= L) gy -= L;
            const uint32_t* row = A.S_rd + (size_t)gy * P;
            uint32_t* dst = s_s + (y - y0 + 1) * PX;
            dev::bulk_g2s(dst, row + gxa, (uint32_t)(n1 * 4), bar);
            if (n2) dev::bulk_g2s(dst + (L - gxa), row, (uint32_t)(n2 * 4), bar);
        }
    }
}

// Euler update of four consecutive pixels of one row from the rolling
// three-row window (s = row above, c = this row, n = row below; w/e are the
// pixels left and right of the four).
__device__ __forceinline__ void stencil_row(float ws, float4 vs, float es, float wc, float4 vc,
                                            float ec, float wn, float4 vn, float en,
                                            const float (&so)[4], float gam, float dwC,
                                            float volC, float repC, float vx, float vy,
                                            float mrel, float dtf, float (&pn)[4]) {
    const float S[6] = {ws, vs.x, vs.y, vs.z, vs.w, es};
    const float Cr[6] = {wc, vc.x, vc.y, vc.z, vc.w, ec};
    const float N[6] = {wn, vn.x, vn.y, vn.z, vn.w, en};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float lap = lap9(N[j], N[j + 1], N[j + 2], Cr[j], Cr[j + 1], Cr[j + 2], S[j],
                               S[j + 1], S[j + 2]);
        const float gx = 0.5f * (Cr[j + 2] - Cr[j]);
        const float gy = 0.5f * (N[j + 1] - S[j + 1]);
        const float rhs =
            rhs_pixel(lap, Cr[j + 1], so[j], gx, gy, gam, dwC, volC, repC, vx, vy, mrel);
        pn[j] = Cr[j + 1] + dtf * rhs;
    }
}

// Per-cell work of a staged class on its band in `buf`.
template <int CLS>
__device__ __noinline__ void staged_persist(const pfb_step_args2d& A, const CellPlan& P,
                                               int rank, char* buf, uint64_t* bar,
                                               uint32_t parity, PersistShared& sh, int par,
                                               bool fm) {
    using M = PMap<CLS>;
    constexpr int WX = M::WX, WY = M::WY, RB = M::RB, NQ = M::NQ, H = M::H, G = M::G;
    constexpr int PX = WX + 8;
    constexpr int TX0 = window_of(CLS).tx0, TY0 = window_of(CLS).ty0;
    float* phi_s = reinterpret_cast<float*>(buf);
    uint32_t* s_s = reinterpret_cast<uint32_t*>(buf + (RB + 4) * PX * 4);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int y0 = rank * RB, y1 = y0 + RB;
    const int L = A.L, Pp = A.P;
    const bool s_tma = (L & 3) == 0;
    const int soff = s_tma ? (P.gx0 & 3) : 0;

    // Zero ring of in-window rows and whole out-of-window rows (never targets
    // of the copies): rank 0 has two rows above the window, the last rank two
    // below it.
    for (int k = tid; k < RB + 4; k += kPThreads) {
        const int y = y0 - 2 + k;
        if (y >= 0 && y < WY) {
            phi_s[k * PX + 3] = 0.0f;
            phi_s[k * PX + 4 + WX] = 0.0f;
        }
    }
    if (rank == 0 || rank == kPK - 1) {
        const int kb = rank == 0 ? 0 : RB + 2;
        for (int i = tid; i < 2 * PX; i += kPThreads) phi_s[kb * PX + i] = 0.0f;
    }
    if (!s_tma) {
        // Odd lattice sides: gather S rows with plain loads.
        const int split = min(WX, L - P.gx0);
        const int sa = max(0, y0 - 1), sb = min(WY, y1 + 1);
        for (int idx = tid; idx < (sb - sa) * WX; idx += kPThreads) {
            const int yy = idx / WX, x = idx - yy * WX, y = sa + yy;
            int gy = P.gy0 + y;
            if (gy >= L) gy -= L;
            const int gx = x < split ? P.gx0 + x : x - split;
            s_s[(y - y0 + 1) * PX + x] = __ldg(A.S_rd + (size_t)gy * Pp + gx);
        }
    }
    if (!dev::mbar_wait_bounded(bar, parity, kWaitPolls)) {
        sh.abort = 1;
        atomicOr(&g_persist_status, 1u);
    }
    __syncthreads();
    const bool abort = sh.abort != 0;

    const bool active = !abort && tid < NQ * G;
    const int q = tid % NQ, g = tid / NQ;
    const int r0 = g * H;
    const int nr = active ? min(H, RB - r0) : 0;
    const int x0 = 4 * q;

    // S_other of the thread's strip stays in registers between the passes;
    // phi is read from the staged band with a rolling three-row window.
    float so[H][4];
#pragma unroll
    for (int r = 0; r < H; ++r) so[r][0] = so[r][1] = so[r][2] = so[r][3] = 0.0f;
    // row t of the band (t = -2 .. RB+1) as (w, c0..c3, e) of this strip
    auto load_row = [&](int t, float& wv, float4& cv, float& ev) {
        const float* row = phi_s + (t + 2) * PX + 4 + x0;
        cv = *reinterpret_cast<const float4*>(row);
        wv = row[-1];
        ev = row[4];
    };

    // ---- pass 1: S_other and the interaction integral
    double aIx = 0.0, aIy = 0.0;
    if (active) {
        float w0, e0, w1, e1;
        float4 cs, cc, cn;
        load_row(r0 - 1, w0, cs, e0);
        load_row(r0, w1, cc, e1);
#pragma unroll
        for (int r = 0; r < H; ++r) {
            if (r < nr) {
                float w2, e2;
                load_row(r0 + r + 1, w2, cn, e2);
                const uint32_t* srow = s_s + (r0 + r + 1) * PX + soff + x0;
                const float C[4] = {cc.x, cc.y, cc.z, cc.w};
                const float Cs[4] = {cs.x, cs.y, cs.z, cs.w};
                const float Cn[4] = {cn.x, cn.y, cn.z, cn.w};
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const float cC = C[j];
                    const float cW = j == 0 ? w1 : C[j - 1];
                    const float cE = j == 3 ? e1 : C[j + 1];
                    // counted twice: the reference evaluates S_other in both passes
                    const float So = s_other_n(srow[j], cC, A.flags, 2u);
                    so[r][j] = So;
                    const float gx = 0.5f * (cE - cW);
                    const float gy = 0.5f * (Cn[j] - Cs[j]);
                    aIx += (double)(cC * gx * So);
                    aIy += (double)(cC * gy * So);
                }
                cs = cc;
                cc = cn;
                w1 = w2;
                e1 = e2;
            }
        }
        (void)w0;
        (void)e0;
    }
    reduce_force<kPK, kPWarps>(A, P, rank, sh.red, par, aIx, aIy);

    const float gam = P.gam, dwC = P.dwC, volC = P.volC, mrel = P.mrel;
    const float vx = sh.red.vx, vy = sh.red.vy;
    const float repC = A.rep_coeff, dtf = A.dt;
    float* tile_out = A.phi_out + (size_t)P.n * kTileArea;
    const int sx = P.sx, sy = P.sy;
    const int dwx = P.dwx, dwy = P.dwy, dtx0 = P.dtx0, dty0 = P.dty0;
    const bool ident = sx == 0 && sy == 0 && P.dcls == CLS;

    // Class change: clear the destination tile outside the new window (own
    // destination rows) and the tile rows outside it (interleaved by rank).
    const int jlo = (rank == 0) ? -(1 << 20) : y0;
    const int jhi = (rank == kPK - 1) ? (1 << 20) : y1;
    const int b_lo = max(0, jlo - sy), b_hi = min(dwy, jhi - sy);
    if (!abort && P.zero_tile) {
        for (int b = b_lo + warp; b < b_hi; b += kPWarps) {
            float* trow = tile_out + (size_t)(dty0 + b) * kTilePitch;
            for (int cc = lane; cc < kTilePitch; cc += 32)
                if (cc < dtx0 || cc >= dtx0 + dwx) trow[cc] = 0.0f;
        }
        for (int t = rank + kPK * warp; t < kTilePitch; t += kPK * kPWarps) {
            if (t >= dty0 && t < dty0 + dwy) continue;
            float* trow = tile_out + (size_t)t * kTilePitch;
            for (int cc = lane; cc < kTilePitch; cc += 32) trow[cc] = 0.0f;
        }
    }

    PixelAcc acc;
    acc.blox = dwx;
    acc.bloy = dwy;

    if (!fm) {
        // ---- pass 2, fused: Euler update, store, scatter, moments
        if (active) {
            float pmaxf = 0.0f;
            int pmax_slow = 0;
            unsigned colmask = 0u;
            float ws, es, wc, ec;
            float4 vs, vc;
            load_row(r0 - 1, ws, vs, es);
            load_row(r0, wc, vc, ec);
#pragma unroll
            for (int r = 0; r < H; ++r) {
                if (r < nr) {
                    const int y = y0 + r0 + r;
                    float wn, en;
                    float4 vn;
                    load_row(r0 + r + 1, wn, vn, en);
                    float pn[4];
                    stencil_row(ws, vs, es, wc, vc, ec, wn, vn, en, so[r], gam, dwC, volC, repC,
                                vx, vy, mrel, dtf, pn);
                    ws = wc;
                    vs = vc;
                    es = ec;
                    wc = wn;
                    vc = vn;
                    ec = en;
                    if (ident) {
                        float* orow = tile_out + (size_t)(TY0 + y) * kTilePitch + TX0 + x0;
                        __stcs(reinterpret_cast<float4*>(orow),
                               make_float4(pn[0], pn[1], pn[2], pn[3]));
                        int gy = P.gy0 + y;
                        if (gy >= L) gy -= L;
                        uint32_t* srow = A.S_sc + (size_t)gy * Pp;
                        double rowV = 0.0;
                        unsigned m = 0u;
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const float p = pn[j];
                            if (fabsf(p) <= 2.0f) {
                                pmaxf = fmaxf(pmaxf, fabsf(p));
                            } else {
                                if (!isfinite(p)) atomicOr(A.flags + PFB_FLAG_NONFINITE, 1u);
                                if (p * p > kPhiSqCap) atomicOr(A.flags + PFB_FLAG_Q_CLAMP, 1u);
                                pmax_slow = max(pmax_slow, (int)__float_as_uint(fabsf(p)));
                            }
                            const uint32_t qv = q_encode(p);
                            if (qv) {
                                int gx = P.gx0 + x0 + j;
                                if (gx >= L) gx -= L;
                                const uint32_t old = atomicAdd(srow + gx, qv);
                                if (old > 0xFFFFFFFFu - qv)
                                    atomicOr(A.flags + PFB_FLAG_S_OVERFLOW, 1u);
                            }
                            const double d = (double)p * (double)p;
                            rowV += d;
                            acc.Cx += d * (double)(x0 + j);
                            if (p > kSupportEps) m |= 1u << j;
                        }
                        acc.V += rowV;
                        acc.Cy += rowV * (double)y;
                        if (m) {
                            acc.bloy = min(acc.bloy, y);
                            acc.bhiy = max(acc.bhiy, y);
                            colmask |= m;
                        }
                    } else {
                        // shifted or re-classed destination: per-pixel map
                        const int b = y - sy;
                        if ((unsigned)b < (unsigned)dwy) {
                            int gy = P.gy0n + b;
                            if (gy >= L) gy -= L;
                            uint32_t* srow = A.S_sc + (size_t)gy * Pp;
                            float* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
#pragma unroll
                            for (int j = 0; j < 4; ++j) {
                                const int a = x0 + j - sx;
                                if ((unsigned)a < (unsigned)dwx) {
                                    __stcs(orow + a, pn[j]);
                                    dest_pixel(A, acc, pn[j], a, b, srow, P.gx0n, L);
                                }
                            }
                        }
                    }
                }
            }
            if (ident) {
                acc.pmaxb = max(acc.pmaxb, max((int)__float_as_uint(pmaxf), pmax_slow));
                if (colmask) {
                    acc.blox = min(acc.blox, x0 + __ffs(colmask) - 1);
                    acc.bhix = max(acc.bhix, x0 + 31 - __clz(colmask));
                }
            }
        }
        if (!abort && !ident) {
            // destination pixels whose source lies outside the window
            for (int b = b_lo + warp; b < b_hi; b += kPWarps) {
                const int j = b + sy;
                const bool jin = (unsigned)j < (unsigned)WY;
                float* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
                for (int a = lane; a < dwx; a += 32) {
                    const int i = a + sx;
                    if (!(jin && (unsigned)i < (unsigned)WX)) __stcs(orow + a, 0.0f);
                }
            }
        }
    } else {
        // ---- full-moment step: phi^{n+1} of own rows and a one-row halo into
        // the S buffer, then the destination pass with the perimeter.
        if (active) {
            float ws, es, wc, ec;
            float4 vs, vc;
            load_row(r0 - 1, ws, vs, es);
            load_row(r0, wc, vc, ec);
#pragma unroll
            for (int r = 0; r < H; ++r) {
                if (r < nr) {
                    float wn, en;
                    float4 vn;
                    load_row(r0 + r + 1, wn, vn, en);
                    float pn[4];
                    stencil_row(ws, vs, es, wc, vc, ec, wn, vn, en, so[r], gam, dwC, volC, repC,
                                vx, vy, mrel, dtf, pn);
                    uint32_t* dst = s_s + (r0 + r + 1) * PX + soff + x0;
#pragma unroll
                    for (int j = 0; j < 4; ++j) dst[j] = __float_as_uint(pn[j]);
                    ws = wc;
                    vs = vc;
                    es = ec;
                    wc = wn;
                    vc = vn;
                    ec = en;
                }
            }
        }
        // All own rows of S are consumed before any halo row is overwritten.
        __syncthreads();
        if (!abort) {
            // halo rows y0-1 and y1 (when inside the window), one warp each
            for (int hr = warp; hr < 2; hr += kPWarps) {
                const int y = hr == 0 ? y0 - 1 : y1;
                if (y < 0 || y >= WY) continue;
                const float* prow = phi_s + (y - y0 + 2) * PX + 4;
                uint32_t* dst = s_s + (y - y0 + 1) * PX + soff;
                for (int x = lane; x < WX; x += 32) {
                    const float* p = prow + x;
                    const float cC = p[0], cW = p[-1], cE = p[1];
                    const float nC = p[PX], nW = p[PX - 1], nE = p[PX + 1];
                    const float sC = p[-PX], sW = p[-PX - 1], sE = p[-PX + 1];
                    const float lap = lap9(nW, nC, nE, cW, cC, cE, sW, sC, sE);
                    const float gx = 0.5f * (cE - cW);
                    const float gy = 0.5f * (nC - sC);
                    const float So = s_other_n(dst[x], cC, A.flags, 0u);
                    const float rhs =
                        rhs_pixel(lap, cC, So, gx, gy, gam, dwC, volC, repC, vx, vy, mrel);
                    dst[x] = __float_as_uint(cC + dtf * rhs);
                }
            }
        }
        __syncthreads();
        if (!abort) {
            for (int b = b_lo + warp; b < b_hi; b += kPWarps) {
                const int j = b + sy;
                const bool jin = (unsigned)j < (unsigned)WY;
                const int jr = j - y0 + 1;
                int gy = P.gy0n + b;
                if (gy >= L) gy -= L;
                float* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
                uint32_t* srow = A.S_sc + (size_t)gy * Pp;
                for (int a = lane; a < dwx; a += 32) {
                    const int i = a + sx;
                    const bool iin = (unsigned)i < (unsigned)WX;
                    auto at = [&](int row, int col) {
                        return __uint_as_float(s_s[row * PX + soff + col]);
                    };
                    const float pn = (jin && iin) ? at(jr, i) : 0.0f;
                    __stcs(orow + a, pn);
                    dest_pixel(A, acc, pn, a, b, srow, P.gx0n, L);
                    float ee = 0.0f, ww = 0.0f, nn = 0.0f, ss = 0.0f;
                    if (jin) {
                        if ((unsigned)(i + 1) < (unsigned)WX) ee = at(jr, i + 1);
                        if ((unsigned)(i - 1) < (unsigned)WX) ww = at(jr, i - 1);
                    }
                    if (iin) {
                        if ((unsigned)(j + 1) < (unsigned)WY) nn = at(jr + 1, i);
                        if ((unsigned)(j - 1) < (unsigned)WY) ss = at(jr - 1, i);
                    }
                    const float pgx = 0.5f * (ee - ww), pgy = 0.5f * (nn - ss);
                    acc.Per += (double)sqrtf(pgx * pgx + pgy * pgy);
                }
            }
        }
    }
    reduce_moments<kPK, kPWarps>(A, P, rank, sh.red, par, fm, acc);
}

__global__ void __launch_bounds__(kPThreads, 3)
    k_step2d_persist(const __grid_constant__ pfb_step_args2d A) {
    extern __shared__ __align__(128) char smem[];
    PersistShared& sh = *reinterpret_cast<PersistShared*>(smem);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

    if (A.clear_ahead_words) {
        uint4* dst = reinterpret_cast<uint4*>(A.S_cl);
        const size_t nvec = (size_t)(A.clear_ahead_words >> 2);
        const size_t stride = (size_t)gridDim.x * kPThreads;
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (size_t i = (size_t)blockIdx.x * kPThreads + tid; i < nvec; i += stride)
            __stcs(dst + i, z);
    }
    const unsigned long long step = *A.step_rd;
    if (blockIdx.x == 0 && tid == 0) {
        if (A.cursor_clear) *A.cursor_clear = 0ull;
        *A.step_wr = step + 1ull;
    }
    const bool fm = full_moment_step(A, step);
    const int rank = (int)dev::cluster_rank();
    const int cid = (int)(blockIdx.x / kPK);
    const int ncl = (int)(gridDim.x / kPK);
    const int ncells = cid < A.N ? (A.N - 1 - cid) / ncl + 1 : 0;
    auto cell_of = [&](int k) {
        const int slot = cid + k * ncl;
        return A.perm ? (int)A.perm[slot] : slot;
    };

    if (tid == 0) {
        sh.abort = 0;
        dev::mbar_init(&sh.bar[0], 1);
        dev::mbar_init(&sh.bar[1], 1);
    }
    __syncthreads();

    uint32_t uses0 = 0u, uses1 = 0u;  // phases consumed per buffer
    int staged_next = 0;
    if (ncells > 0) {
        const int n0 = cell_of(0);
        const int c0 = (int)A.cell_cls[n0];
        staged_next = c0 <= 3;
        if (staged_next && warp == 0) prefetch_band(A, n0, c0, rank, smem + kPHeader, &sh.bar[0]);
    }
    for (int k = 0; k < ncells; ++k) {
        if (k % kPlanBatch == 0) {
            __syncthreads();
            if (warp == 0) {
                const int kk = k + lane;
                if (kk < ncells) {
                    const int n = cell_of(kk);
                    plan_cell_lane(A, n, (int)A.cell_cls[n], step, sh.plan[lane], rank == 0);
                }
            }
            __syncthreads();
        }
        const CellPlan& P = sh.plan[k % kPlanBatch];
        const int b = k & 1;
        char* buf = smem + kPHeader + b * kPBuf;
        char* nbuf = smem + kPHeader + (b ^ 1) * kPBuf;
        const bool staged = staged_next != 0;
        const uint32_t parity = (b ? uses1 : uses0) & 1u;
        if (staged) {
            if (b) ++uses1; else ++uses0;
        }
        // copy of the next cell's band overlaps this cell's arithmetic
        staged_next = 0;
        if (k + 1 < ncells) {
            const int nn = cell_of(k + 1);
            const int cn = (int)A.cell_cls[nn];
            staged_next = cn <= 3;
            if (staged_next && warp == 0) prefetch_band(A, nn, cn, rank, nbuf, &sh.bar[b ^ 1]);
        }
        switch (P.cls) {
            case 0: staged_persist<0>(A, P, rank, buf, &sh.bar[b], parity, sh, b, fm); break;
            case 1: staged_persist<1>(A, P, rank, buf, &sh.bar[b], parity, sh, b, fm); break;
            case 2: staged_persist<2>(A, P, rank, buf, &sh.bar[b], parity, sh, b, fm); break;
            case 3: staged_persist<3>(A, P, rank, buf, &sh.bar[b], parity, sh, b, fm); break;
            case 4: global_cell<4, kPK, kPWarps>(A, P, rank, sh.red, b, fm); break;
            case 5: global_cell<5, kPK, kPWarps>(A, P, rank, sh.red, b, fm); break;
            default:
                if (rank == 0 && tid == 0) atomicAdd(A.flags + PFB_FLAG_CLASS_UNSUPPORTED, 1u);
                break;
        }
        // generic accesses of this buffer are ordered before the next copy into it
        fence_proxy_async();
        __syncthreads();
    }
    // every CTA's partials stay readable until rank 0 has read them
    dev::cluster_sync();
}

int g_max_clusters[64] = {0};

}  // namespace

int persist2d_launch(const pfb_step_args2d& A, cudaStream_t stream, bool one_cell_per_cluster) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(PFB_E_CUDA, "cudaGetDevice failed");
    if (dev < 0 || dev >= 64) return set_error(PFB_E_CONFIG, "device index out of range");
    if (!g_max_clusters[dev]) {
        cudaError_t e = cudaFuncSetAttribute(k_step2d_persist,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, kPSmem);
        if (e != cudaSuccess)
            return set_error(PFB_E_CUDA, "persistent kernel attribute: %s", cudaGetErrorString(e));
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(kPK, 1, 1);
        cfg.blockDim = dim3(kPThreads, 1, 1);
        cfg.dynamicSmemBytes = kPSmem;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = kPK;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        int nc = 0;
        e = cudaOccupancyMaxActiveClusters(&nc, k_step2d_persist, &cfg);
        if (e != cudaSuccess || nc <= 0)
            return set_error(PFB_E_CUDA, "cluster occupancy query: %s", cudaGetErrorString(e));
        g_max_clusters[dev] = nc;
    }
    const int clusters =
        (one_cell_per_cluster || A.N < g_max_clusters[dev]) ? A.N : g_max_clusters[dev];
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(clusters * kPK), 1, 1);
    cfg.blockDim = dim3(kPThreads, 1, 1);
    cfg.dynamicSmemBytes = kPSmem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kPK;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_step2d_persist, A);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "persistent step launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int persist2d_smem_bytes() { return kPSmem; }

int persist2d_read_status(unsigned* out, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_persist_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status read: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_persist_status, &z, sizeof(z));
    }
    if (out) *out = v;
    return PFB_OK;
}

}  // namespace pfb
