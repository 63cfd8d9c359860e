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

#include <algorithm>
#include <cstdint>

#include "device_util.cuh"
#include "pfb_common.cuh"
#include "pfb_internal.h"
#include "step2d_common.cuh"
#include "storage2d.cuh"

namespace pfb {

// Block shape: threads per CTA and the CTAs per SM the register budget is
// sized for (overridable at build time to sweep launch shapes). By default
// the budget follows the shared-memory limit of the staged band: 2 CTAs per
// SM at clusters of 2 (96 registers), 3 at clusters of 4 and 8 (72).
#ifndef PFB_STEP2D_THREADS
#define PFB_STEP2D_THREADS 288
#endif
#ifdef PFB_STEP2D_MINB
__host__ __device__ constexpr int min_blocks(int) { return PFB_STEP2D_MINB; }
#else
__host__ __device__ constexpr int min_blocks(int k) { return k == 2 ? 2 : 3; }
#endif
// Rows per iteration of the pass-1 and pass-2 strip loops (0: by cluster
// size, 3 rows of pass 2 at clusters of 2 where the registers allow, else 1).
#ifndef PFB_STEP2D_P1_UNROLL
#define PFB_STEP2D_P1_UNROLL 1  // pass 1 stays rolled
#endif
#ifndef PFB_STEP2D_P2_UNROLL
#define PFB_STEP2D_P2_UNROLL 0
#endif
__host__ __device__ constexpr int row_unroll(int v, int k) { return v > 0 ? v : (k == 2 ? 3 : 1); }
// L2 eviction priorities (bit 0: the staged phi_in and S_rd rows are read
// evict-first).
#ifndef PFB_STEP2D_L2HINTS
#define PFB_STEP2D_L2HINTS 1
#endif
constexpr int kThreads = PFB_STEP2D_THREADS;
constexpr int kWarps = kThreads / 32;
static_assert(kThreads % 32 == 0, "whole warps: the reductions index per-warp slots");
constexpr int kHeaderBytes = 2048;
// the spatial velocity observer's kernels: room for its reduction arrays
constexpr int kHeaderBytesObs = 2560;
template <int OBS>
constexpr int kHeader = OBS == PFB_VELOCITY_SPATIAL ? kHeaderBytesObs : kHeaderBytes;

// Status word of this kernel family in device memory: bit 0 = a CTA gave up
// waiting for its staged band. Read with pfb_device_status().
__device__ unsigned int g_step2d_status = 0u;

template <int K, int OBS = PFB_VELOCITY_DISABLED>
struct __align__(16) StepShared {
    uint64_t bar;
    int abort;
    int gx0, gy0;
    CellPlan plan;
    RedScratch<kWarps, K, kObsVals<OBS>> red;
};
static_assert(sizeof(StepShared<8>) <= kHeaderBytes, "shared header too large");
static_assert(sizeof(StepShared<8, PFB_VELOCITY_SPATIAL>) <= kHeaderBytesObs,
              "observer shared header too large");

__host__ __device__ constexpr int band_rows(int wy, int k) { return (wy + k - 1) / k; }

// Rows per work item of the column-rolling passes: balances the threads
// against the (rows + 2) shared loads a column run costs.
__host__ __device__ constexpr int pick_run(int wx, int rows) {
    int best_h = 1;
    long best = -1;
    for (int h = 2; h <= 48; ++h) {
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

// Thread map of the register passes: a thread owns a strip four pixels wide
// and H rows tall of the band; NQ strips per row, G row groups.
template <int CLS, int K> struct QuadMap {
    static constexpr int WX = window_of(CLS).wx;
    static constexpr int RB = (window_of(CLS).wy + K - 1) / K;
    static constexpr int NQ = WX / 4;
    static constexpr int GMAX = kThreads / NQ;
    static constexpr int H = (RB + GMAX - 1) / GMAX;
    static constexpr int G = (RB + H - 1) / H;
    static_assert(WX % 4 == 0 && NQ * G <= kThreads, "strip map");
};

// Euler update of four consecutive pixels of one row from the rolling
// three-row window (s = row above, c = this row, n = row below; w/e are the
// pixels left and right of the four).
//
// Pixels (0, 1) and (2, 3) are updated as pairs with the sm_100 packed
// binary32 instructions (__ffma2_rn, __fadd2_rn, __fmul2_rn; each half
// rounds exactly as the scalar instruction). The operation sequence is the
// one the compiler gives rhs_pixel_m and lap9 as scalars, contractions
// included, measured on a B200 to agree bit for bit on 2^22 random inputs:
//   lap = fma(-20, c, fma(4, s1, s2)) * (1/6)  (s1, s2 summed left to right)
//   a   = fma(-(rep*phi), S_other, fma(vol, phi, fma(gam, lap, -(dw*X))))
//   rhs = fma(mrel, a, -fma(vx, gx, vy*gy)),  phi' = fma(dt, rhs, phi)
// with X = (phi*(1-phi))*fma(-2, phi, 1). Negated coefficients are exact
// sign flips of the scalar products. The shifted neighbours of the
// Laplacian sums and of gx are not register pairs, so those stay scalar.
struct PairCoeffs {
    float gam, dwC, volC, repC, vx, vy, mrel, dt;
};

__device__ __forceinline__ float2 dup(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 neg2(float2 v) { return make_float2(-v.x, -v.y); }

template <int J>
__device__ __forceinline__ float2 update_pair(const float (&S)[6], const float (&C)[6],
                                              const float (&N)[6], float2 so, const PairCoeffs& k) {
    const float2 ns = __fadd2_rn(make_float2(N[J + 1], N[J + 2]), make_float2(S[J + 1], S[J + 2]));
    const float s1a = __fadd_rn(__fadd_rn(ns.x, C[J + 2]), C[J]);
    const float s1b = __fadd_rn(__fadd_rn(ns.y, C[J + 3]), C[J + 1]);
    const float s2a = __fadd_rn(__fadd_rn(__fadd_rn(N[J + 2], N[J]), S[J + 2]), S[J]);
    const float s2b = __fadd_rn(__fadd_rn(__fadd_rn(N[J + 3], N[J + 1]), S[J + 3]), S[J + 1]);
    const float2 phi = make_float2(C[J + 1], C[J + 2]);
    float2 t = __ffma2_rn(dup(4.0f), make_float2(s1a, s1b), make_float2(s2a, s2b));
    t = __ffma2_rn(dup(-20.0f), phi, t);
    const float2 lap = __fmul2_rn(t, dup((float)(1.0 / 6.0)));
    const float2 gx = __fmul2_rn(dup(0.5f), make_float2(__fsub_rn(C[J + 2], C[J]), __fsub_rn(C[J + 3], C[J + 1])));
    const float2 gy = __fmul2_rn(dup(0.5f),
                                 __fadd2_rn(make_float2(N[J + 1], N[J + 2]), neg2(make_float2(S[J + 1], S[J + 2]))));
    const float2 om = __fadd2_rn(dup(1.0f), neg2(phi));
    const float2 tp = __ffma2_rn(dup(-2.0f), phi, dup(1.0f));
    const float2 X = __fmul2_rn(__fmul2_rn(phi, om), tp);
    float2 a = __ffma2_rn(dup(k.gam), lap, __fmul2_rn(dup(-k.dwC), X));
    a = __ffma2_rn(dup(k.volC), phi, a);
    a = __ffma2_rn(__fmul2_rn(dup(-k.repC), phi), so, a);
    const float2 adv = __ffma2_rn(dup(k.vx), gx, __fmul2_rn(dup(k.vy), gy));
    const float2 rhs = __ffma2_rn(dup(k.mrel), a, neg2(adv));
    return __ffma2_rn(dup(k.dt), rhs, phi);
}

// Packed pairs at clusters of 2 (96 registers); the scalar form at 4 and 8,
// where the packed one spills under the 72-register budget (both give the
// same bits). 0 selects the scalar form everywhere.
#ifndef PFB_STEP2D_PACKED
#define PFB_STEP2D_PACKED 1
#endif

template <bool PACKED>
__device__ __forceinline__ void stencil4(float ws, float4 vs, float es, float wc, float4 vc,
                                         float ec, float wn, float4 vn, float en,
                                         const float (&so)[4], const PairCoeffs& k,
                                         float (&pn)[4]) {
    const float S[6] = {ws, vs.x, vs.y, vs.z, vs.w, es};
    const float C[6] = {wc, vc.x, vc.y, vc.z, vc.w, ec};
    const float N[6] = {wn, vn.x, vn.y, vn.z, vn.w, en};
    if constexpr (PACKED) {
        const float2 lo = update_pair<0>(S, C, N, make_float2(so[0], so[1]), k);
        const float2 hi = update_pair<2>(S, C, N, make_float2(so[2], so[3]), k);
        pn[0] = lo.x;
        pn[1] = lo.y;
        pn[2] = hi.x;
        pn[3] = hi.y;
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float lap =
                lap9(N[j], N[j + 1], N[j + 2], C[j], C[j + 1], C[j + 2], S[j], S[j + 1], S[j + 2]);
            const float gx = 0.5f * (C[j + 2] - C[j]);
            const float gy = 0.5f * (N[j + 1] - S[j + 1]);
            const float rhs = rhs_pixel_m(lap, C[j + 1], so[j], gx, gy, k.gam, k.dwC, k.volC,
                                          k.repC, k.vx, k.vy, k.mrel);
            pn[j] = C[j + 1] + k.dt * rhs;
        }
    }
}

// Both staged arrays use the row pitch WX + 8 words.
__host__ __device__ constexpr int staged_bytes(int cls, int k, int header = kHeaderBytes) {
    return header + (2 * band_rows(window_of(cls).wy, k) + 6) * (window_of(cls).wx + 8) * 4;
}

__host__ __device__ constexpr int step_smem_bytes(int k, int header = kHeaderBytes) {
    int m = 0;
    for (int c = 0; c <= 3; ++c)
        m = staged_bytes(c, k, header) > m ? staged_bytes(c, k, header) : m;
    return m;
}

// ---- phi pool stores -------------------------------------------------------
// float pools store as is; 16-bit pools round stochastically (storage2d.cuh)
// and report the stored value back so that moments and the scatter see it.
template <typename T>
__device__ __forceinline__ void store4(T* o, float (&v)[4], uint32_t seed, uint32_t pix) {
    if constexpr (!Store<T>::kHalf) {
        __stcs(reinterpret_cast<float4*>(o), make_float4(v[0], v[1], v[2], v[3]));
    } else {
        uint16_t b[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            b[j] = Store<T>::bits(v[j], mix32(seed ^ ((pix + j) * 0x9E3779B9u)));
            v[j] = Store<T>::value(b[j]);
        }
        __stcs(reinterpret_cast<uint2*>(o),
               make_uint2((uint32_t)b[0] | ((uint32_t)b[1] << 16),
                          (uint32_t)b[2] | ((uint32_t)b[3] << 16)));
    }
}

template <typename T>
__device__ __forceinline__ float store1(T* o, float v, uint32_t seed, uint32_t pix) {
    if constexpr (!Store<T>::kHalf) {
        __stcs(o, v);
        return v;
    } else {
        const uint16_t b = Store<T>::bits(v, mix32(seed ^ (pix * 0x9E3779B9u)));
        __stcs(reinterpret_cast<unsigned short*>(o), b);
        return Store<T>::value(b);
    }
}

// value a store of v at tile pixel pix will hold
template <typename T>
__device__ __forceinline__ float rounded(float v, uint32_t seed, uint32_t pix) {
    if constexpr (!Store<T>::kHalf) {
        return v;
    } else {
        return Store<T>::value(Store<T>::bits(v, mix32(seed ^ (pix * 0x9E3779B9u))));
    }
}

template <typename T>
__device__ __forceinline__ void store_zero(T* o) {
    if constexpr (!Store<T>::kHalf)
        *o = 0.0f;
    else
        *reinterpret_cast<unsigned short*>(o) = 0;
}

// ---------------------------------------------------------------------------
// Staged path: classes 0-3.
// Shared layout after the header (row pitch PX = WX + 8 words):
//   phi_s [RB+4][PX] f32 : window rows y0-2 .. y1+1; column x at 4+x; columns
//                          -1 and WX are the synthesized zero ring
//   ps_s  [RB+2][PX] u32 : window rows y0-1 .. y1; window column x at soff+x
//                          (soff = gx0 & 3 when S is staged by bulk copies).
//                          Holds q_S; pass 1 replaces own rows by S_other
//                          (f32 bits); on full-moment steps phi^{n+1} is
//                          written over it.
// ---------------------------------------------------------------------------
template <int CLS, int K, typename T, int OBS, bool BINS = false>
__device__ __forceinline__ void staged_cell(const pfb_step_args2d& A, int n, int rank,
                                            char* smem, unsigned long long step, bool fm,
                                            const BinArgs& B) {
    constexpr Window W = window_of(CLS);
    constexpr int WX = W.wx, WY = W.wy, TX0 = W.tx0, TY0 = W.ty0;
    constexpr int RB = band_rows(WY, K);
    constexpr int PX = WX + 8;
    constexpr int PHI_ROWS = RB + 4;
    static_assert(WY % K == 0, "staged classes split into equal bands");
    static_assert((WX * 4) % 16 == 0 && (TX0 * 4) % 16 == 0, "bulk copies need 16-B rows");

    StepShared<K, OBS>& sh = *reinterpret_cast<StepShared<K, OBS>*>(smem);
    const CellPlan& P = sh.plan;
    float* phi_s = reinterpret_cast<float*>(smem + kHeader<OBS>);
    uint32_t* ps_s = reinterpret_cast<uint32_t*>(smem + kHeader<OBS> + PHI_ROWS * PX * 4);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int y0 = rank * RB;
    const int y1 = y0 + RB;
    const T* tile_in = reinterpret_cast<const T*>(A.phi_in) + (size_t)n * kTileArea;
    const int L = A.L, Pp = A.P;
    const bool s_tma = (L & 3) == 0;
    constexpr bool kHalf = Store<T>::kHalf;
    // 16-bit rows are copied into the back of their binary32 row and widened
    // in place after the copy completes
    constexpr int HOFF = WX / 2 + 8;
    static_assert(!kHalf || (HOFF % 4 == 0 && HOFF + WX / 2 <= PX), "16-bit staging offset");

    if (tid == 0) {
        sh.abort = 0;
        sh.gx0 = A.cell[n].gx0;
        sh.gy0 = A.cell[n].gy0;
        dev::mbar_init(&sh.bar, 1);
    }
    __syncthreads();
    const int gx0 = sh.gx0, gy0 = sh.gy0;
    const int soff = s_tma ? (gx0 & 3) : 0;

    const int ra = max(0, y0 - 2), rb = min(WY, y1 + 2);
    const int sa = max(0, y0 - 1), sb = min(WY, y1 + 1);
    if (warp == 0) {
        // Bulk copies: one per phi row; one or two per S row (split at the
        // periodic seam), each starting on a 16-byte boundary.
        const int gxa = gx0 - soff;
        const bool wrap = gx0 + WX > L;
        const int n1 = wrap ? L - gxa : min((soff + WX + 3) & ~3, Pp - gxa);
        const int n2 = wrap ? ((gx0 + WX - L + 3) & ~3) : 0;
        uint32_t bytes = 0;
        for (int y = ra + lane; y < rb; y += 32) bytes += (uint32_t)(WX * sizeof(T));
        if (s_tma)
            for (int y = sa + lane; y < sb; y += 32) bytes += (uint32_t)((n1 + n2) * 4);
        bytes = __reduce_add_sync(0xFFFFFFFFu, bytes);
        if (lane == 0) dev::mbar_arrive_expect_tx(&sh.bar, bytes);
        __syncwarp();
#if PFB_STEP2D_L2HINTS & 1
        const uint64_t pol = dev::l2_policy_evict_first();
#define PFB_G2S(d, s, n, b) dev::bulk_g2s_hint(d, s, n, b, pol)
#else
#define PFB_G2S(d, s, n, b) dev::bulk_g2s(d, s, n, b)
#endif
        for (int y = ra + lane; y < rb; y += 32)
            PFB_G2S(phi_s + (y - y0 + 2) * PX + (kHalf ? HOFF : 4),
                    tile_in + (size_t)(TY0 + y) * kTilePitch + TX0, (uint32_t)(WX * sizeof(T)),
                    &sh.bar);
        if (s_tma) {
            for (int y = sa + lane; y < sb; y += 32) {
                int gy = gy0 + y;
                if (gy >= L) gy -= L;
                const uint32_t* row = A.S_rd + (size_t)gy * Pp;
                uint32_t* dst = ps_s + (y - y0 + 1) * PX;
                PFB_G2S(dst, row + gxa, (uint32_t)(n1 * 4), &sh.bar);
                if (n2) PFB_G2S(dst + (L - gxa), row, (uint32_t)(n2 * 4), &sh.bar);
            }
        }
#undef PFB_G2S
        if (lane == 0)
            plan_cell<OBS == PFB_VELOCITY_SPATIAL>(A, n, CLS, step, sh.plan, rank == 0);
    } else {
        const int t = tid - 32;
        constexpr int NT = kThreads - 32;
        if (!s_tma) {
            // lattice sides that are not a multiple of 4: plain gather
            const int split = min(WX, L - gx0);
            const int cnt = (sb - sa) * WX;
            for (int idx = t; idx < cnt; idx += NT) {
                const int yy = idx / WX;
                const int x = idx - yy * WX;
                const int y = sa + yy;
                int gy = gy0 + y;
                if (gy >= L) gy -= L;
                const int gx = x < split ? gx0 + x : x - split;
                ps_s[(y - y0 + 1) * PX + x] = __ldg(A.S_rd + (size_t)gy * Pp + gx);
            }
        }
        // Zero ring columns of in-window rows (16-bit rows: after widening);
        // whole rows outside the window.
        if (!kHalf)
            for (int k = t; k < PHI_ROWS; k += NT) {
                const int y = y0 - 2 + k;
                if (y >= 0 && y < WY) {
                    phi_s[k * PX + 3] = 0.0f;
                    phi_s[k * PX + 4 + WX] = 0.0f;
                }
            }
        if (rank == 0 || rank == K - 1) {
            const int kb = rank == 0 ? 0 : RB + 2;
            for (int i = t; i < 2 * PX; i += NT) phi_s[kb * PX + i] = 0.0f;
        }
    }
    if (!dev::mbar_wait_bounded(&sh.bar, 0, kWaitPolls)) {
        sh.abort = 1;
        atomicOr(&g_step2d_status, 1u);
    }
    __syncthreads();
    const bool abort = sh.abort != 0;
    if constexpr (kHalf) {
        // widen each staged 16-bit row into its binary32 slots, one warp per
        // row: all lanes read the row before any lane writes
        if (!abort) {
            constexpr int PER = (WX + 31) / 32;
            for (int k = warp; k < PHI_ROWS; k += kWarps) {
                const int y = y0 - 2 + k;
                if (y < 0 || y >= WY) continue;
                float* row = phi_s + k * PX;
                const uint16_t* hrow = reinterpret_cast<const uint16_t*>(row + HOFF);
                float v[PER];
#pragma unroll
                for (int i = 0; i < PER; ++i) {
                    const int x = lane + 32 * i;
                    v[i] = x < WX ? Store<T>::value(hrow[x]) : 0.0f;
                }
                __syncwarp();
#pragma unroll
                for (int i = 0; i < PER; ++i) {
                    const int x = lane + 32 * i;
                    if (x < WX) row[4 + x] = v[i];
                }
                if (lane == 0) {
                    row[3] = 0.0f;
                    row[4 + WX] = 0.0f;
                }
            }
        }
        __syncthreads();
    }

    // ---- pass 1: S_other of the thread's strip (stored over q_S) and the
    // interaction integral. A thread owns a strip four pixels wide and up to
    // H rows tall; rows run in a rolled loop with a three-row register window.
    using QM = QuadMap<CLS, K>;
    constexpr int H = QM::H;
    constexpr int kRowsP1 = row_unroll(PFB_STEP2D_P1_UNROLL, K);
    constexpr int kRowsP2 = row_unroll(PFB_STEP2D_P2_UNROLL, K);
    constexpr bool kPacked = PFB_STEP2D_PACKED && K == 2;
    const bool active = !abort && tid < QM::NQ * QM::G;
    const int x0 = 4 * (tid % QM::NQ);
    const int r0 = (tid / QM::NQ) * H;
    const int nr = active ? min(H, RB - r0) : 0;
    auto load_row = [&](int t, float& w, float4& c, float& e) {
        const float* row = phi_s + (t + 2) * PX + 4 + x0;
        c = *reinterpret_cast<const float4*>(row);
        w = row[-1];
        e = row[4];
    };
    double aIx = 0.0, aIy = 0.0;
    ObsAcc<OBS> ob;
    if (active) {
        float ws, es, wc, ec;
        float4 vs, vc;
        load_row(r0 - 1, ws, vs, es);
        load_row(r0, wc, vc, ec);
        uint32_t* qrow = ps_s + (r0 + 1) * PX + soff + x0;
        uint32_t neg = 0u;
#pragma unroll kRowsP1
        for (int r = 0; r < nr; ++r) {
            float wn, en;
            float4 vn;
            load_row(r0 + r + 1, wn, vn, en);
            const float C[6] = {wc, vc.x, vc.y, vc.z, vc.w, ec};
            const float Sv[4] = {vs.x, vs.y, vs.z, vs.w};
            const float Nv[4] = {vn.x, vn.y, vn.z, vn.w};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float cC = C[j + 1];
                const float So = s_other_counted(qrow[j], cC, neg);
                qrow[j] = __float_as_uint(So);
                const float gx = 0.5f * (C[j + 2] - C[j]);
                const float gy = 0.5f * (Nv[j] - Sv[j]);
                aIx += (double)(cC * gx * So);
                aIy += (double)(cC * gy * So);
                if constexpr (OBS == PFB_VELOCITY_SPATIAL) {
                    const float S6[6] = {ws, vs.x, vs.y, vs.z, vs.w, es};
                    const float N6[6] = {wn, vn.x, vn.y, vn.z, vn.w, en};
                    ob.pixel(P, A.rep_coeff, x0 + j, y0 + r0 + r, cC, C[j + 2], C[j], Nv[j], Sv[j],
                             N6[j + 2], N6[j], S6[j + 2], S6[j], So);
                }
            }
            qrow += PX;
            ws = wc;
            vs = vc;
            es = ec;
            wc = wn;
            vc = vn;
            ec = en;
        }
        // counted twice: the reference evaluates S_other in both passes
        if (neg) atomicAdd(A.flags + PFB_FLAG_S_NEGATIVE, 2u * neg);
    }
    reduce_force<K, kWarps, OBS>(A, P, rank, sh.red, aIx, aIy, ob, &g_step2d_status);

    const float gam = P.gam, dwC = P.dwC, volC = P.volC;
    const float vx = sh.red.vx, vy = sh.red.vy, mrel = P.mrel;
    const float repC = A.rep_coeff, dtf = A.dt;
    const PairCoeffs kc{gam, dwC, volC, repC, vx, vy, mrel, dtf};
    const int sx = P.sx, sy = P.sy;
    const int dwx = P.dwx, dwy = P.dwy, dtx0 = P.dtx0, dty0 = P.dty0;
    const int gx0n = P.gx0n, gy0n = P.gy0n;
    T* tile_out = reinterpret_cast<T*>(A.phi_out) + (size_t)n * kTileArea;
    // stochastic-rounding stream of this cell and step (16-bit pools)
    const uint32_t sr_seed = kHalf ? mix32((uint32_t)step * 0x85EBCA6Bu ^
                                           (uint32_t)A.cell[n].global_id * 0xC2B2AE35u ^
                                           (uint32_t)A.seed)
                                   : 0u;
    // Destination row b reads source row j = b + sy; rows above the window
    // belong to rank 0, rows below it to rank K-1.
    const int jlo = (rank == 0) ? -(1 << 20) : y0;
    const int jhi = (rank == K - 1) ? (1 << 20) : y1;
    const int b_lo = max(0, jlo - sy), b_hi = min(dwy, jhi - sy);
    if (!abort && P.zero_tile) {
        // the destination tile last held another class: clear outside the window
        for (int b = b_lo + warp; b < b_hi; b += kWarps) {
            T* trow = tile_out + (size_t)(dty0 + b) * kTilePitch;
            for (int c = lane; c < kTilePitch; c += 32)
                if (c < dtx0 || c >= dtx0 + dwx) store_zero(trow + c);
        }
        for (int t = rank + K * warp; t < kTilePitch; t += K * kWarps) {
            if (t >= dty0 && t < dty0 + dwy) continue;
            T* trow = tile_out + (size_t)t * kTilePitch;
            for (int c = lane; c < kTilePitch; c += 32) store_zero(trow + c);
        }
    }

    PixelAcc acc;
    acc.blox = dwx;
    acc.bloy = dwy;
    if (!fm) {
        // ---- pass 2, fused: Euler update, store, scatter and moments
        const bool ident = sx == 0 && sy == 0 && P.dcls == CLS;
        if (active) {
            float ws, es, wc, ec;
            float4 vs, vc;
            load_row(r0 - 1, ws, vs, es);
            load_row(r0, wc, vc, ec);
            const uint32_t* qrow = ps_s + (r0 + 1) * PX + soff + x0;
            if (ident) {

                uint32_t pmaxb = 0u;
                unsigned colmask = 0u;
                int gy = gy0 + y0 + r0;
                if (gy >= L) gy -= L;
                int gx = gx0 + x0;
                if (gx >= L) gx -= L;
                // the strip's four columns wrap at most once
                int gxj[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) gxj[j] = gx + j < L ? gx + j : gx + j - L;
                T* o = tile_out + (size_t)(TY0 + y0 + r0) * kTilePitch + TX0 + x0;
                // overflow checks of a row's atomics run one row later, so the
                // atomic round trip overlaps the next row's arithmetic
                uint32_t old_prev[4] = {0u, 0u, 0u, 0u}, q_prev[4] = {0u, 0u, 0u, 0u};
#pragma unroll kRowsP2
                for (int r = 0; r < nr; ++r) {
                    float wn, en;
                    float4 vn;
                    load_row(r0 + r + 1, wn, vn, en);
                    const float so[4] = {__uint_as_float(qrow[0]), __uint_as_float(qrow[1]),
                                         __uint_as_float(qrow[2]), __uint_as_float(qrow[3])};
                    float pn[4];
                    stencil4<kPacked>(ws, vs, es, wc, vc, ec, wn, vn, en, so, kc, pn);
                    // pn becomes the stored value (16-bit pools round here)
                    store4<T>(o, pn, sr_seed, (uint32_t)(o - tile_out));
                    uint32_t* srow = A.S_sc + (size_t)gy * Pp;
                    if constexpr (!BINS) {
                        bool ovf = false;
#pragma unroll
                        for (int j = 0; j < 4; ++j) ovf |= old_prev[j] > 0xFFFFFFFFu - q_prev[j];
                        if (ovf) atomicOr(A.flags + PFB_FLAG_S_OVERFLOW, 1u);
                    }
                    // |phi| bit patterns order like the values; NaN and inf
                    // sort above 2.0, so one compare guards the rare checks
                    const uint32_t rowb =
                        max(max(__float_as_uint(fabsf(pn[0])), __float_as_uint(fabsf(pn[1]))),
                            max(__float_as_uint(fabsf(pn[2])), __float_as_uint(fabsf(pn[3]))));
                    pmaxb = max(pmaxb, rowb);
                    if (rowb > 0x40000000u) {  // some |phi| > 2 (or not finite)
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const float p = pn[j];
                            if (!isfinite(p)) atomicOr(A.flags + PFB_FLAG_NONFINITE, 1u);
                            if (p * p > kPhiSqCap) atomicOr(A.flags + PFB_FLAG_Q_CLAMP, 1u);
                        }
                    }
                    double rowV = 0.0, rowX = 0.0;
                    unsigned m = 0u;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float p = pn[j];
                        const uint32_t qv = q_encode(p);
                        if constexpr (BINS) {
                            // bounded per bin; checked by the launch's last CTA
                            red_add_nonzero(srow + gxj[j], qv);
                        } else {
                            q_prev[j] = qv;
                            old_prev[j] = dev::atom_add_nonzero(srow + gxj[j], qv);
                        }
                        const double d = (double)p * (double)p;
                        rowV += d;
                        rowX += d * (double)j;
                        if (p > kSupportEps) m |= 1u << j;
                    }
                    const int y = y0 + r0 + r;
                    acc.V += rowV;
                    acc.Cx += rowV * (double)x0 + rowX;
                    acc.Cy += rowV * (double)y;
                    if (m) {
                        acc.bloy = min(acc.bloy, y);
                        acc.bhiy = max(acc.bhiy, y);
                        colmask |= m;
                    }
                    if (++gy >= L) gy -= L;
                    o += kTilePitch;
                    qrow += PX;
                    ws = wc;
                    vs = vc;
                    es = ec;
                    wc = wn;
                    vc = vn;
                    ec = en;
                }
                if constexpr (BINS) {
                    int gys = gy0 + y0 + r0;
                    if (gys >= L) gys -= L;
                    bin_block_add(gy0 >> kBinShift, gx0 >> kBinShift, B.nbx, B.nby, gys, nr,
                                  gxj[0], 4, L, q_encode(__uint_as_float(pmaxb)));
                } else {
                    bool ovf = false;
#pragma unroll
                    for (int j = 0; j < 4; ++j) ovf |= old_prev[j] > 0xFFFFFFFFu - q_prev[j];
                    if (ovf) atomicOr(A.flags + PFB_FLAG_S_OVERFLOW, 1u);
                }
                acc.pmaxb = max(acc.pmaxb, (int)pmaxb);
                if (colmask) {
                    acc.blox = min(acc.blox, x0 + __ffs(colmask) - 1);
                    acc.bhix = max(acc.bhix, x0 + 31 - __clz(colmask));
                }
            } else {
                // shifted or re-classed destination: per-pixel map
#pragma unroll 1
                for (int r = 0; r < nr; ++r) {
                    float wn, en;
                    float4 vn;
                    load_row(r0 + r + 1, wn, vn, en);
                    const float so[4] = {__uint_as_float(qrow[0]), __uint_as_float(qrow[1]),
                                         __uint_as_float(qrow[2]), __uint_as_float(qrow[3])};
                    float pn[4];
                    stencil4<kPacked>(ws, vs, es, wc, vc, ec, wn, vn, en, so, kc, pn);
                    const int b = y0 + r0 + r - sy;
                    if ((unsigned)b < (unsigned)dwy) {
                        int gyn = gy0n + b;
                        if (gyn >= L) gyn -= L;
                        uint32_t* srow = A.S_sc + (size_t)gyn * Pp;
                        T* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
#pragma unroll
                        for (int j = 0; j < 4; ++j) {
                            const int a = x0 + j - sx;
                            if ((unsigned)a < (unsigned)dwx) {
                                const float v = store1<T>(orow + a, pn[j], sr_seed,
                                                          (uint32_t)(orow + a - tile_out));
                                dest_pixel(A, acc, v, a, b, srow, gx0n, L);
                            }
                        }
                    }
                    qrow += PX;
                    ws = wc;
                    vs = vc;
                    es = ec;
                    wc = wn;
                    vc = vn;
                    ec = en;
                }
                if constexpr (BINS) {
                    // the strip's destination block, clipped to the window
                    const int ba = max(0, y0 + r0 - sy), bb = min(dwy, y0 + r0 + nr - sy);
                    const int aa = max(0, x0 - sx), ab = min(dwx, x0 + 4 - sx);
                    int gys = gy0n + ba, gxs = gx0n + aa;
                    if (gys >= L) gys -= L;
                    if (gxs >= L) gxs -= L;
                    bin_block_add(gy0n >> kBinShift, gx0n >> kBinShift, B.nbx, B.nby, gys,
                                  bb - ba, gxs, ab - aa, L,
                                  q_encode(__uint_as_float((uint32_t)acc.pmaxb)));
                }
            }
        }
        if (!abort && !ident) {
            // destination pixels whose source lies outside the window
            for (int b = b_lo + warp; b < b_hi; b += kWarps) {
                const int j = b + sy;
                const bool jin = (unsigned)j < (unsigned)WY;
                T* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
                for (int a = lane; a < dwx; a += 32) {
                    const int i = a + sx;
                    if (!(jin && (unsigned)i < (unsigned)WX)) store_zero(orow + a);
                }
            }
        }
    } else {
        // ---- full-moment step: phi^{n+1} of own rows plus a one-row halo over
        // the staged S (own rows hold S_other, halo rows q_S), then the
        // destination pass with the perimeter. (reduce_force's barrier orders
        // the S_other stores of pass 1 before these reads.)
        if (!abort) {
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
                uint32_t* q = ps_s + (ya - y0 + 1) * PX + soff + x;
                float sW = p[-PX - 1], sC = p[-PX], sE = p[-PX + 1];
                float cW = p[-1], cC = p[0], cE = p[1];
                for (int y = ya; y < yb; ++y) {
                    const float nW = p[PX - 1], nC = p[PX], nE = p[PX + 1];
                    const float lap = lap9(nW, nC, nE, cW, cC, cE, sW, sC, sE);
                    const float gx = 0.5f * (cE - cW);
                    const float gy = 0.5f * (nC - sC);
                    const bool own = (y >= y0) && (y < y1);
                    const float So = own ? __uint_as_float(*q) : s_other_n(*q, cC, A.flags, 0u);
                    const float rhs =
                        rhs_pixel(lap, cC, So, gx, gy, gam, dwC, volC, repC, vx, vy, mrel);
                    // the value the destination store will hold (pixel (x-sx, y-sy))
                    const uint32_t pix = (uint32_t)((dty0 + y - sy) * kTilePitch + dtx0 + x - sx);
                    *q = __float_as_uint(rounded<T>(cC + dtf * rhs, sr_seed, pix));
                    sW = cW;
                    sC = cC;
                    sE = cE;
                    cW = nW;
                    cC = nC;
                    cE = nE;
                    p += PX;
                    q += PX;
                }
            }
        }
        __syncthreads();
        if (!abort) {
            for (int b = b_lo + warp; b < b_hi; b += kWarps) {
                const int j = b + sy;
                const bool jin = (unsigned)j < (unsigned)WY;
                const int jr = j - y0 + 1;  // ps_s row of source row j
                int gy = gy0n + b;
                if (gy >= L) gy -= L;
                T* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
                uint32_t* srow = A.S_sc + (size_t)gy * Pp;
                const uint32_t* row = ps_s + jr * PX + soff;
                for (int a = lane; a < dwx; a += 32) {
                    const int i = a + sx;
                    const bool iin = (unsigned)i < (unsigned)WX;
                    const float pn = (jin && iin) ? __uint_as_float(row[i]) : 0.0f;
                    // already rounded when computed: the store keeps it exactly
                    store1<T>(orow + a, pn, sr_seed, (uint32_t)(orow + a - tile_out));
                    dest_pixel(A, acc, pn, a, b, srow, gx0n, L);
                    float e = 0.0f, w = 0.0f, nn = 0.0f, ss = 0.0f;
                    if (jin) {
                        if ((unsigned)(i + 1) < (unsigned)WX) e = __uint_as_float(row[i + 1]);
                        if ((unsigned)(i - 1) < (unsigned)WX) w = __uint_as_float(row[i - 1]);
                    }
                    if (iin) {
                        if ((unsigned)(j + 1) < (unsigned)WY) nn = __uint_as_float(row[PX + i]);
                        if ((unsigned)(j - 1) < (unsigned)WY) ss = __uint_as_float(row[-PX + i]);
                    }
                    const float pgx = 0.5f * (e - w), pgy = 0.5f * (nn - ss);
                    acc.Per += (double)sqrtf(pgx * pgx + pgy * pgy);
                }
            }
        }
    }
    if (abort) (void)dev::mbar_wait_bounded(&sh.bar, 0, kWaitPolls);
    reduce_moments<K, kWarps>(A, P, rank, sh.red, fm, acc, &g_step2d_status);
}

template <int CLS, int K, int OBS>
__device__ __forceinline__ void global_cell_v1(const pfb_step_args2d& A, int n, int rank,
                                               char* smem, unsigned long long step, bool fm,
                                               unsigned long long* bound = nullptr, int nbx = 0,
                                               int nby = 0) {
    StepShared<K, OBS>& sh = *reinterpret_cast<StepShared<K, OBS>*>(smem);
    if (threadIdx.x == 0)
        plan_cell<OBS == PFB_VELOCITY_SPATIAL>(A, n, CLS, step, sh.plan, rank == 0);
    __syncthreads();
    global_cell<CLS, K, kWarps, OBS>(A, sh.plan, rank, sh.red, fm, &g_step2d_status, bound, nbx,
                                     nby, &sh.abort);
}

// One system's step for CTA `lb` of the `nb` CTAs that serve it. BINS: the
// identity path scatters without returns under per-bin bounds (B holds both
// sets; this launch bounds into set step & 1, and settles and clears the set
// of the previous launch, which has finished).
template <int K, typename T, int OBS = PFB_VELOCITY_DISABLED, bool BINS = false>
__device__ __forceinline__ void step_body(const pfb_step_args2d& A, int lb, int nb, char* smem,
                                          const BinArgs& B = BinArgs{}) {
    const int tid = threadIdx.x;

    // Clear the S slot two steps ahead with streaming stores (the kernel does
    // not otherwise touch it).
    if (A.clear_ahead_words) {
        uint4* dst = reinterpret_cast<uint4*>(A.S_cl);
        const size_t nvec = (size_t)(A.clear_ahead_words >> 2);
        const size_t stride = (size_t)nb * kThreads;
        const uint4 z = make_uint4(0u, 0u, 0u, 0u);
        for (size_t i = (size_t)lb * kThreads + tid; i < nvec; i += stride) __stcs(dst + i, z);
    }
    const unsigned long long step = *A.step_rd;
    if (lb == 0 && tid == 0) {
        if (A.cursor_clear) *A.cursor_clear = 0ull;
        *A.step_wr = step + 1ull;
    }
    const bool fm = full_moment_step(A, step);
    if constexpr (BINS) {
        const int nbins = B.nbx * B.nby;
        const int par = (int)(step & 1ull);
        // the previous launch's bounds: check (recounting the rare bin at
        // 2^32) and clear them for the next launch; its field is our phi_in
        for (int first = lb * kThreads; first < nbins; first += nb * kThreads)
            bin_settle_chunk<T>(B.bound + (size_t)(1 - par) * nbins, B.geo + (size_t)(1 - par) * A.N,
                                reinterpret_cast<const T*>(A.phi_in), A.N, A.L, B.nbx, first,
                                min(kThreads, nbins - first), A.flags, B.recounts, smem);
        for (int k = tid; k < kBinTab * kBinTab; k += kThreads) g_bintab[k] = 0u;
    }

    const int rank = (int)dev::cluster_rank();
    StepShared<K, OBS>& sh = *reinterpret_cast<StepShared<K, OBS>*>(smem);
    if (tid == 0) red_init(sh.red, rank);
    if (BINS && tid == 0) sh.plan.n = -1;  // set when the cell's step is planned
    dev::cluster_arrive_relaxed();  // matched by the wait in reduce_force
    const int slot = lb / K;
    const int n = A.perm ? (int)A.perm[slot] : slot;
    const int cls = (int)A.cell_cls[n];
    switch (cls) {
        case 0: staged_cell<0, K, T, OBS, BINS>(A, n, rank, smem, step, fm, B); break;
        case 1: staged_cell<1, K, T, OBS, BINS>(A, n, rank, smem, step, fm, B); break;
        case 2: staged_cell<2, K, T, OBS, BINS>(A, n, rank, smem, step, fm, B); break;
        case 3: staged_cell<3, K, T, OBS, BINS>(A, n, rank, smem, step, fm, B); break;
        case 4:
            if constexpr (Store<T>::kHalf) {
                // 16-bit pools: the global-memory classes are not provided
                if (rank == 0 && tid == 0) atomicAdd(A.flags + PFB_FLAG_CLASS_UNSUPPORTED, 1u);
                dev::cluster_wait();
            } else {
                global_cell_v1<4, K, OBS>(A, n, rank, smem, step, fm, BINS && !fm ? B.bound + (size_t)(step & 1ull) * B.nbx * B.nby : nullptr, B.nbx, B.nby);
            }
            break;
        case 5:
            if constexpr (Store<T>::kHalf) {
                if (rank == 0 && tid == 0) atomicAdd(A.flags + PFB_FLAG_CLASS_UNSUPPORTED, 1u);
                dev::cluster_wait();
            } else {
                global_cell_v1<5, K, OBS>(A, n, rank, smem, step, fm, BINS && !fm ? B.bound + (size_t)(step & 1ull) * B.nbx * B.nby : nullptr, B.nbx, B.nby);
            }
            break;
        default:
            if (rank == 0 && tid == 0) atomicAdd(A.flags + PFB_FLAG_CLASS_UNSUPPORTED, 1u);
            dev::cluster_wait();  // uniform over the cluster
            break;
    }
    if constexpr (BINS) {
        // the shared table into this launch's bounds; the committed window
        // geometry for the launch that will settle them (everything read
        // again here rather than kept live through the passes)
        __syncthreads();
        const CellPlan& P = reinterpret_cast<StepShared<K, OBS>*>(smem)->plan;
        if (P.n >= 0) {
            const unsigned long long st = *A.step_rd;
            unsigned long long* set = B.bound + (size_t)(st & 1ull) * B.nbx * B.nby;
            if (!full_moment_step(A, st))
                bin_table_flush(set, P.gy0n >> kBinShift, P.gx0n >> kBinShift, B.nbx, B.nby);
            if (dev::cluster_rank() == 0 && threadIdx.x == 0)
                B.geo[(size_t)(st & 1ull) * A.N + P.n] = make_int4(P.gx0n, P.gy0n, P.dcls, 0);
        }
    }
}

template <int K, typename T = float, int OBS = PFB_VELOCITY_DISABLED, bool BINS = false>
__global__ void __launch_bounds__(kThreads, min_blocks(K))
    k_step2d(const __grid_constant__ pfb_step_args2d A, const __grid_constant__ BinArgs B) {
    extern __shared__ __align__(128) char smem[];
    step_body<K, T, OBS, BINS>(A, (int)blockIdx.x, (int)gridDim.x, smem, B);
}

// Many independent systems in one launch: system r is served by CTAs
// [block_start[r], block_start[r+1]) (multiples of K, so clusters never
// straddle systems); its arguments are copied into shared memory. All
// systems of one launch share the pool storage type T.
template <int K, typename T = float>
__global__ void __launch_bounds__(kThreads, min_blocks(K))
    k_step2d_batch(const pfb_step_args2d* __restrict__ args, const int* __restrict__ block_start,
                   int R) {
    extern __shared__ __align__(128) char smem[];
    __shared__ __align__(16) pfb_step_args2d sA;
    const int b = (int)blockIdx.x;
    int lo = 0, hi = R - 1;  // last r with block_start[r] <= b
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(block_start + mid) <= b)
            lo = mid;
        else
            hi = mid - 1;
    }
    const int r = lo;
    static_assert(sizeof(pfb_step_args2d) % 8 == 0, "argument record copy");
    const uint64_t* srcw = reinterpret_cast<const uint64_t*>(args + r);
    uint64_t* dstw = reinterpret_cast<uint64_t*>(&sA);
    if (threadIdx.x < sizeof(pfb_step_args2d) / 8) dstw[threadIdx.x] = __ldg(srcw + threadIdx.x);
    __syncthreads();
    const int b0 = __ldg(block_start + r);
    step_body<K, T>(sA, b - b0, __ldg(block_start + r + 1) - b0, smem);
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
template <int K, typename T>
static cudaError_t configure_pool() {
    cudaError_t e = cudaFuncSetAttribute(k_step2d<K, T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         step_smem_bytes(K));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_step2d<K, T>, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_step2d<K, T, PFB_VELOCITY_DISABLED, true>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, step_smem_bytes(K));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_step2d<K, T, PFB_VELOCITY_DISABLED, true>,
                             cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_step2d_batch<K, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             step_smem_bytes(K));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_step2d_batch<K, T>,
                                cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

template <int K, int OBS>
static cudaError_t configure_observed() {
    cudaError_t e = cudaFuncSetAttribute(k_step2d<K, float, OBS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         step_smem_bytes(K, kHeader<OBS>));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(k_step2d<K, float, OBS>,
                                cudaFuncAttributePreferredSharedMemoryCarveout, 100);
}

template <int K>
static cudaError_t configure_one() {
    cudaError_t e = configure_pool<K, float>();
    if (e != cudaSuccess) return e;
    if ((e = configure_observed<K, PFB_VELOCITY_ADVECTION>()) != cudaSuccess) return e;
    if ((e = configure_observed<K, PFB_VELOCITY_SPATIAL>()) != cudaSuccess) return e;
    if constexpr (K != 8) {
        if ((e = configure_pool<K, __half>()) != cudaSuccess) return e;
        if ((e = configure_pool<K, __nv_bfloat16>()) != cudaSuccess) return e;
    }
    return cudaSuccess;
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

template <int K, typename T = float, int OBS = PFB_VELOCITY_DISABLED, bool BINS = false>
static cudaError_t launch_k(const pfb_step_args2d& A, cudaStream_t stream,
                            const BinArgs& B = BinArgs{}) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(A.N * K), 1, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = (size_t)step_smem_bytes(K, kHeader<OBS>);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_step2d<K, T, OBS, BINS>, A, B);
}

// Contract checks common to every single-system launch.
static int check_step_args(const pfb_step_args2d* a) {
    if (!a) return set_error(PFB_E_ARG, "null step arguments");
    const pfb_step_args2d& A = *a;
    if (!A.phi_in || !A.phi_out || !A.S_rd || !A.S_sc || !A.cell || !A.cell_cls || !A.step_rd ||
        !A.step_wr || !A.flags)
        return set_error(PFB_E_ARG, "null buffer in step arguments");
    if (A.clear_ahead_words && !A.S_cl) return set_error(PFB_E_ARG, "clear-ahead needs S_cl");
    if (((uintptr_t)A.phi_in & 15u) || ((uintptr_t)A.phi_out & 15u) ||
        ((uintptr_t)A.S_cl & 15u) || ((uintptr_t)A.S_rd & 15u))
        return set_error(PFB_E_ARG, "phi pools and S slots must be 16-byte aligned");
    if (A.N < 0) return set_error(PFB_E_ARG, "negative cell count");
    if (A.L < kMinSide || A.P < A.L || (A.P & 3))
        return set_error(PFB_E_ARG, "domain side must be at least %d, P >= L and P %% 4 == 0",
                         kMinSide);
    if (A.parity_out != 0 && A.parity_out != 1) return set_error(PFB_E_ARG, "parity_out must be 0 or 1");
    return PFB_OK;
}

int step2d_launch_storage(const pfb_step_args2d* a, int cluster, int variant, int storage,
                          cudaStream_t stream) {
    int rc = check_step_args(a);
    if (rc) return rc;
    const pfb_step_args2d& A = *a;
    if (A.moments) return set_error(PFB_E_ARG, "moments are read by the observed launch only");
    if (cluster == 0) cluster = kDefaultCluster;
    if (cluster != 2 && cluster != 4 && cluster != 8)
        return set_error(PFB_E_CONFIG, "cluster must be 2, 4 or 8");
    if (variant == 0) variant = 1;
    if (variant != 1) return set_error(PFB_E_CONFIG, "unknown kernel variant");
    if (A.N == 0) return PFB_OK;
    rc = step2d_configure_device();
    if (rc) return rc;
    if (storage != kStoreF32 && storage != kStoreF16 && storage != kStoreBF16)
        return set_error(PFB_E_ARG, "unknown phi storage %d", storage);
    if (storage != kStoreF32 && cluster == 8)
        return set_error(PFB_E_CONFIG, "16-bit phi pools use clusters of 2 or 4");
    cudaError_t e;
    if (storage == kStoreF16)
        e = cluster == 2 ? launch_k<2, __half>(A, stream) : launch_k<4, __half>(A, stream);
    else if (storage == kStoreBF16)
        e = cluster == 2 ? launch_k<2, __nv_bfloat16>(A, stream)
                         : launch_k<4, __nv_bfloat16>(A, stream);
    else
        e = cluster == 2   ? launch_k<2>(A, stream)
            : cluster == 4 ? launch_k<4>(A, stream)
                           : launch_k<8>(A, stream);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "step launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int step2d_launch_binned(const pfb_step_args2d* a, int cluster, int storage,
                         const BinArgs& B, cudaStream_t stream) {
    int rc = check_step_args(a);
    if (rc) return rc;
    const pfb_step_args2d& A = *a;
    if (A.moments) return set_error(PFB_E_ARG, "moments are read by the observed launch only");
    if (!B.bound || !B.geo || !B.recounts)
        return set_error(PFB_E_ARG, "binned launch without its bin buffers");
    if (B.nbx != (A.L + (1 << kBinShift) - 1) >> kBinShift || B.nby != B.nbx)
        return set_error(PFB_E_ARG, "bin grid does not match the lattice side");
    if (cluster == 0) cluster = kDefaultCluster;
    if (cluster != 2 && cluster != 4 && cluster != 8)
        return set_error(PFB_E_CONFIG, "cluster must be 2, 4 or 8");
    if (storage != kStoreF32 && storage != kStoreF16 && storage != kStoreBF16)
        return set_error(PFB_E_ARG, "unknown phi storage %d", storage);
    if (storage != kStoreF32 && cluster == 8)
        return set_error(PFB_E_CONFIG, "16-bit phi pools use clusters of 2 or 4");
    if (A.N == 0) return PFB_OK;
    if ((rc = step2d_configure_device())) return rc;
    constexpr int D = PFB_VELOCITY_DISABLED;
    cudaError_t e;
    if (storage == kStoreF16)
        e = cluster == 2 ? launch_k<2, __half, D, true>(A, stream, B)
                         : launch_k<4, __half, D, true>(A, stream, B);
    else if (storage == kStoreBF16)
        e = cluster == 2 ? launch_k<2, __nv_bfloat16, D, true>(A, stream, B)
                         : launch_k<4, __nv_bfloat16, D, true>(A, stream, B);
    else
        e = cluster == 2   ? launch_k<2, float, D, true>(A, stream, B)
            : cluster == 4 ? launch_k<4, float, D, true>(A, stream, B)
                           : launch_k<8, float, D, true>(A, stream, B);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "step launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
    k_settle_bins2d(const __grid_constant__ BinArgs B, const T* phi, int N, int L,
                    unsigned long long step, uint32_t* flags) {
    __shared__ __align__(16) char scratch[256 * sizeof(unsigned long long) + (kThreads + 1) * 4];
    const int nbins = B.nbx * B.nby;
    const int par = (int)(step & 1ull);
    for (int first = blockIdx.x * kThreads; first < nbins; first += gridDim.x * kThreads)
        bin_settle_chunk<T>(B.bound + (size_t)par * nbins, B.geo + (size_t)par * N, phi, N, L,
                            B.nbx, first, min(kThreads, nbins - first), flags, B.recounts,
                            scratch);
}

int step2d_settle_bins(const BinArgs& B, const void* phi, int storage, int N, int L,
                       unsigned long long step, uint32_t* flags, cudaStream_t stream) {
    if (!B.bound || !B.geo || !B.recounts || !phi || !flags || N <= 0)
        return set_error(PFB_E_ARG, "settle_bins: bad arguments");
    const int nbins = B.nbx * B.nby;
    const int grid = std::min(148 * 2, (nbins + kThreads - 1) / kThreads);
    if (storage == kStoreF16)
        k_settle_bins2d<__half><<<grid, kThreads, 0, stream>>>(B, static_cast<const __half*>(phi), N,
                                                              L, step, flags);
    else if (storage == kStoreBF16)
        k_settle_bins2d<__nv_bfloat16><<<grid, kThreads, 0, stream>>>(
            B, static_cast<const __nv_bfloat16*>(phi), N, L, step, flags);
    else
        k_settle_bins2d<float><<<grid, kThreads, 0, stream>>>(B, static_cast<const float*>(phi), N,
                                                             L, step, flags);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "settle_bins: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int step2d_launch_observed(const pfb_step_args2d* a, int cluster, int observation,
                           cudaStream_t stream) {
    if (observation == PFB_VELOCITY_DISABLED) {
        if (!a) return set_error(PFB_E_ARG, "null step arguments");
        pfb_step_args2d b = *a;
        b.moments = nullptr;
        return step2d_launch_storage(&b, cluster, 0, kStoreF32, stream);
    }
    int rc = check_step_args(a);
    if (rc) return rc;
    const pfb_step_args2d& A = *a;
    if (observation != PFB_VELOCITY_ADVECTION && observation != PFB_VELOCITY_SPATIAL)
        return set_error(PFB_E_ARG, "unknown velocity observation %d", observation);
    if (observation == PFB_VELOCITY_SPATIAL && !A.moments)
        return set_error(PFB_E_ARG, "the spatial observer needs moment accumulators");
    if (!(A.physical_dt > 0.0)) return set_error(PFB_E_ARG, "physical_dt must be positive");
    if (cluster == 0) cluster = kDefaultCluster;
    if (cluster != 2 && cluster != 4 && cluster != 8)
        return set_error(PFB_E_CONFIG, "cluster must be 2, 4 or 8");
    if (A.N == 0) return PFB_OK;
    if ((rc = step2d_configure_device())) return rc;
    cudaError_t e;
    if (observation == PFB_VELOCITY_ADVECTION)
        e = cluster == 2   ? launch_k<2, float, PFB_VELOCITY_ADVECTION>(A, stream)
            : cluster == 4 ? launch_k<4, float, PFB_VELOCITY_ADVECTION>(A, stream)
                           : launch_k<8, float, PFB_VELOCITY_ADVECTION>(A, stream);
    else
        e = cluster == 2   ? launch_k<2, float, PFB_VELOCITY_SPATIAL>(A, stream)
            : cluster == 4 ? launch_k<4, float, PFB_VELOCITY_SPATIAL>(A, stream)
                           : launch_k<8, float, PFB_VELOCITY_SPATIAL>(A, stream);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "step launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int step2d_launch_variant(const pfb_step_args2d* a, int cluster, int variant,
                          cudaStream_t stream) {
    return step2d_launch_storage(a, cluster, variant, kStoreF32, stream);
}

template <int K, typename T = float>
static cudaError_t launch_batch_k(const pfb_step_args2d* args, const int* block_start, int R,
                                  int total_blocks, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)total_blocks, 1, 1);
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
    return cudaLaunchKernelEx(&cfg, k_step2d_batch<K, T>, args, block_start, R);
}

int step2d_launch_batch(const pfb_step_args2d* d_args, const int* d_block_start, int R,
                        int total_blocks, int cluster, int storage, cudaStream_t stream) {
    if (!d_args || !d_block_start || R <= 0 || total_blocks < 0)
        return set_error(PFB_E_ARG, "invalid batch arguments");
    if (cluster == 0) cluster = kDefaultCluster;
    if (cluster != 2 && cluster != 4 && cluster != 8)
        return set_error(PFB_E_CONFIG, "cluster must be 2, 4 or 8");
    if (storage < 0 || storage > 2) return set_error(PFB_E_ARG, "storage must be 0, 1 or 2");
    if (storage && cluster == 8)
        return set_error(PFB_E_CONFIG, "16-bit phi pools run with clusters of 2 or 4");
    if (total_blocks % cluster) return set_error(PFB_E_ARG, "block count must be a multiple of K");
    if (total_blocks == 0) return PFB_OK;
    int rc = step2d_configure_device();
    if (rc) return rc;
    cudaError_t e;
    if (storage == kStoreF16)
        e = cluster == 2 ? launch_batch_k<2, __half>(d_args, d_block_start, R, total_blocks, stream)
                         : launch_batch_k<4, __half>(d_args, d_block_start, R, total_blocks, stream);
    else if (storage == kStoreBF16)
        e = cluster == 2
                ? launch_batch_k<2, __nv_bfloat16>(d_args, d_block_start, R, total_blocks, stream)
                : launch_batch_k<4, __nv_bfloat16>(d_args, d_block_start, R, total_blocks, stream);
    else
        e = cluster == 2   ? launch_batch_k<2>(d_args, d_block_start, R, total_blocks, stream)
            : cluster == 4 ? launch_batch_k<4>(d_args, d_block_start, R, total_blocks, stream)
                           : launch_batch_k<8>(d_args, d_block_start, R, total_blocks, stream);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "batch launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int step2d_launch(const pfb_step_args2d* a, int cluster, cudaStream_t stream) {
    return step2d_launch_variant(a, cluster, 0, stream);
}

int step2d_read_status(unsigned* out, int clear) {
    const unsigned pv = 0;
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_step2d_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status read: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_step2d_status, &z, sizeof(z));
    }
    if (out) *out = v | pv;
    return PFB_OK;
}

}  // namespace pfb
