// Device pieces shared by the two 2D step kernels (per-cell clusters in
// step2d.cu, persistent pipelined clusters in step2d_persist.cu): the
// per-cell decision record, the tumble/class/shift decision, S_other, and the
// per-pixel store/scatter/moment update.
#pragma once

#include <cstdint>

#include "device_util.cuh"
#include "pfb_common.cuh"
#include "pfb_internal.h"
#include "storage2d.cuh"

namespace pfb {

// Polls of an mbarrier before a CTA gives up (each poll suspends briefly).
constexpr uint32_t kWaitPolls = 1u << 24;

// Everything one step decides for a cell before touching its field.
struct CellPlan {
    int n;              // cell slot
    int cls;            // source class
    int sx, sy;         // recentring shift
    int gx0, gy0;       // source origin
    int gx0n, gy0n;     // destination origin
    int dcls;           // destination class
    int zero_tile;      // destination tile must be cleared (class changed)
    int pctr, tumbled, no_margin;
    int dwx, dwy, dtx0, dty0;
    float gam, dwC, volC, vA, pcos, psin, theta, mrel;
    double ginv, gcx, gcy;  // spatial observer geometry: 2/V, Cx/V, Cy/V
};

// S_other = (q_S - q(phi)) 2^-27; a negative difference is counted, not
// floored silently (reference src/kernels.cu:19-25). `count` adds to the
// S_other_negative counter (0 to not count).
__device__ __forceinline__ float s_other_n(uint32_t qS, float phi, uint32_t* flags,
                                           uint32_t count) {
    const uint32_t qc = q_encode(phi);
    if (qS >= qc) return (float)(qS - qc) * kQInv;
    if (count) atomicAdd(flags + PFB_FLAG_S_NEGATIVE, count);
    return 0.0f;
}

// Branch-free form for the hot loops: the caller counts the negative cases
// in `neg` and adds them to the flag once.
__device__ __forceinline__ float s_other_counted(uint32_t qS, float phi, uint32_t& neg) {
    const uint32_t qc = q_encode(phi);
    const bool ok = qS >= qc;
    neg += ok ? 0u : 1u;
    return ok ? (float)(qS - qc) * kQInv : 0.0f;
}

// Tumble, class choice and recentring shift of cell n whose field is in class
// `cls` (reference src/kernels.cu:93-191 and :624-711). Deterministic in its
// inputs, so every CTA that runs it for the same cell decides the same thing;
// only `leader` raises flags. GEO also records the spatial observer's
// geometry of the field about to be read.
template <bool GEO = false>
__device__ __forceinline__ void plan_cell(const pfb_step_args2d& A, int n, int cls,
                                          unsigned long long step, CellPlan& out, bool leader) {
    const Window W = window_of(cls);
    const pfb_cell2d& cs = A.cell[n];
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
    int dcls = cls;
    int no_margin = 0;
    unsigned pctr = cs.promote_ctr;
    if (ex > 0) {
        if (ex + kPromoteSlack > W.wx || ey + kPromoteSlack > W.wy) {
            const int grow = smallest_class_holding(ex, ey, kPromoteSlack, A.L);
            if (grow >= 0) {
                dcls = grow;
            } else if (cls == kClassFallback && ex <= W.wx && ey <= W.wy) {
                no_margin = 1;
            } else if (leader) {
                atomicAdd(A.flags + PFB_FLAG_CLASS_EXHAUSTED, 1u);
            }
            pctr = 0u;
        } else {
            const int small = smallest_class_holding(ex, ey, kDemoteSlack, A.L);
            if (small >= 0 && small != cls &&
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
        if (dcls == cls) {
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

    out.n = n;
    out.cls = cls;
    out.gx0 = cs.gx0;
    out.gy0 = cs.gy0;
    out.sx = sx;
    out.sy = sy;
    out.gx0n = gx0n;
    out.gy0n = gy0n;
    out.dcls = dcls;
    out.zero_tile = (dcls != (int)cs.cls_written[A.parity_out]);
    out.pctr = (int)pctr;
    out.tumbled = tumbled;
    out.no_margin = no_margin;
    out.dwx = D.wx;
    out.dwy = D.wy;
    out.dtx0 = D.tx0;
    out.dty0 = D.ty0;
    out.gam = gam;
    out.dwC = dwC;
    out.volC = volC;
    out.vA = cs.v_A;
    out.pcos = pc;
    out.psin = ps;
    out.theta = theta;
    out.mrel = mrel;
    if constexpr (GEO) {
        out.ginv = 2.0 / cs.V;
        out.gcx = cs.Cx / cs.V;
        out.gcy = cs.Cy / cs.V;
    }
}

__device__ __forceinline__ bool full_moment_step(const pfb_step_args2d& A,
                                                 unsigned long long step) {
    return A.full_moment_every > 0 &&
           ((step + 1ull) % (unsigned long long)A.full_moment_every) == 0ull;
}

// ---- exact overflow detection for non-returning scatters -------------------
// The Q5.27 aggregate only ever receives non-negative addends, so the running
// sum at a pixel crosses 2^32 - 1 (the reference's S_overflow test on each
// returning atomicAdd, src/kernels.cu:496-497) exactly when the pixel's final
// total T(p) does, whatever the order of the adds. A launch that scatters with
// non-returning red.add keeps, per 16 x 16 lattice bin, an upper bound of T(p)
// over the bin: each CTA gathers the largest addend of each strip into a
// shared table over its destination window's bins (atomicMax) and adds the
// table to the global bounds with non-returning adds at its end. The next
// launch, which starts only when this one has finished, checks these bounds
// while it clears them: a bin at or above 2^32 is recounted exactly (64-bit
// sums of q of the field this launch wrote, over the windows this launch
// committed, kept per step parity in `geo`) and S_overflow is raised iff some
// T(p) >= 2^32. The driver settles the last launch of a run the same way.
constexpr int kBinTab = 16;  // the shared table is kBinTab x kBinTab bins

__device__ __forceinline__ void red_add_nonzero(uint32_t* p, uint32_t v) {
    asm volatile(
        "{\n\t.reg .pred nz;\n\t"
        "setp.ne.u32 nz, %1, 0;\n\t"
        "@nz red.global.add.u32 [%0], %1;\n\t}" ::"l"(p),
        "r"(v)
        : "memory");
}

// Per-CTA table of the largest addend per bin over the destination window
// (kBinTab x kBinTab bins from the bin holding the window origin), filled with
// shared atomicMax and added to the launch's bounds at the CTA's end.
__shared__ unsigned int g_bintab[kBinTab * kBinTab];

// Forward cyclic run of bins touched by lattice rows (or columns) g .. g+n-1
// (0 <= g < L, 1 <= n < L): first bin and count. The last bin of a side that
// is not a multiple of 16 is partial, so a short run can cross it.
__device__ __forceinline__ int bin_run(int g, int n, int L, int nb, int* first) {
    int g1 = g + n - 1;
    if (g1 >= L) g1 -= L;
    const int a = g >> kBinShift, b = g1 >> kBinShift;
    *first = a;
    return b >= a ? b - a + 1 : b - a + nb + 1;
}

// A block of destination pixels (rows gy .. gy+nr-1, columns gx .. gx+nc-1 of
// the periodic lattice, nr, nc <= 16) of a destination window whose origin
// lies in bin (tr0, tc0), largest addend q: q raises every bin the block
// touches (at most 3 x 3) in the shared table. A window of a staged class
// (at most 176 pixels a side) spans at most 13 bins a side, so every bin has
// a table entry.
__device__ __forceinline__ void bin_block_add(int tr0, int tc0, int nbx, int nby, int gy, int nr,
                                              int gx, int nc, int L, uint32_t q) {
    if (nr <= 0 || nc <= 0 || q == 0u) return;
    int r0 = 0, c0 = 0;
    const int nrb = bin_run(gy, nr, L, nby, &r0);
    const int ncb = bin_run(gx, nc, L, nbx, &c0);
    int lr = r0 - tr0;
    if (lr < 0) lr += nby;
    int lc0 = c0 - tc0;
    if (lc0 < 0) lc0 += nbx;
    for (int i = 0; i < nrb; ++i, ++lr)
        for (int j = 0, lc = lc0; j < ncb; ++j, ++lc)
            if (lr < kBinTab && lc < kBinTab) atomicMax(g_bintab + lr * kBinTab + lc, q);
}

// The shared table added to the bounds `set` (non-returning adds). All
// threads of the CTA call it after a CTA barrier.
__device__ __forceinline__ void bin_table_flush(unsigned long long* set, int tr0, int tc0, int nbx,
                                                int nby) {
    for (int k = threadIdx.x; k < kBinTab * kBinTab; k += blockDim.x) {
        const unsigned q = g_bintab[k];
        if (!q) continue;
        int r = tr0 + k / kBinTab, c = tc0 + k % kBinTab;
        if (r >= nby) r -= nby;
        if (c >= nbx) c -= nbx;
        atomicAdd(set + r * nbx + c, (unsigned long long)q);
    }
}

// The largest addend of a whole CTA (q_of the largest |phi| over its threads,
// pmaxb) added to every bin of a box of destination rows [b0, b1) and window
// columns [0, wx) at lattice origin (gx0, gy0), straight into the global
// bounds. All threads of the CTA call it; `slot` is a shared word.
__device__ __forceinline__ void bin_box_add(unsigned long long* bound, int nbx, int nby,
                                            int pmaxb, int b0, int b1, int wx, int gx0, int gy0,
                                            int L, int* slot) {
    if (threadIdx.x == 0) *slot = 0;
    __syncthreads();
    const int m = __reduce_max_sync(0xFFFFFFFFu, pmaxb);
    if ((threadIdx.x & 31) == 0) atomicMax(slot, m);
    __syncthreads();
    const uint32_t q = q_encode(__uint_as_float((uint32_t)*slot));
    if (q == 0u || b1 <= b0) return;
    int gy = gy0 + b0;
    if (gy >= L) gy -= L;
    int r0 = 0, c0 = 0;
    const int nr = bin_run(gy, b1 - b0, L, nby, &r0);
    const int nc = bin_run(gx0, wx, L, nbx, &c0);
    for (int k = threadIdx.x; k < nr * nc; k += blockDim.x) {
        int r = r0 + k / nc, c = c0 + k % nc;
        if (r >= nby) r -= nby;
        if (c >= nbx) c -= nbx;
        atomicAdd(bound + r * nbx + c, (unsigned long long)q);
    }
}

// Exact recount of bin `bin` of a launch's bounds: 64-bit totals of q over the
// windows `geo` (that launch's commits) of the field `phi` it wrote; returns
// true when some total reaches 2^32. All threads of the CTA call it; `acc` is
// 256 shared 64-bit words.
template <typename T>
__device__ __noinline__ bool bin_recount(const T* phi, const int4* geo, int N, int L, int nbx,
                                         int bin, unsigned long long* acc) {
    for (int k = threadIdx.x; k < 256; k += blockDim.x) acc[k] = 0ull;
    __syncthreads();
    const int px0 = (bin % nbx) << kBinShift, py0 = (bin / nbx) << kBinShift;
    const int w = min(16, L - px0), h = min(16, L - py0);
    for (int c = threadIdx.x; c < N; c += blockDim.x) {
        const int4 g = geo[c];
        const Window W = window_of(g.z);
        const T* tile = phi + (size_t)c * kTileArea;
        for (int j = 0; j < h; ++j) {
            int b = py0 + j - g.y;
            if (b < 0) b += L;
            if (b >= W.wy) continue;
            for (int i = 0; i < w; ++i) {
                int a = px0 + i - g.x;
                if (a < 0) a += L;
                if (a >= W.wx) continue;
                const T raw = tile[(size_t)(W.ty0 + b) * kTilePitch + W.tx0 + a];
                float v;
                if constexpr (sizeof(T) == 2)
                    v = Store<T>::value(*reinterpret_cast<const uint16_t*>(&raw));
                else
                    v = raw;
                const uint32_t q = q_encode(v);
                if (q) atomicAdd(acc + j * 16 + i, (unsigned long long)q);
            }
        }
    }
    __syncthreads();
    bool over = false;
    for (int k = threadIdx.x; k < 256; k += blockDim.x) over |= acc[k] >= (1ull << 32);
    return __syncthreads_or(over) != 0;
}

template <typename T>
__device__ __noinline__ void bin_settle_hot(unsigned long long* bound, const int4* geo,
                                            const T* phi, int N, int L, int nbx, int i, bool hot,
                                            uint32_t* flags, unsigned int* recounts,
                                            char* scratch);

// Checks and clears bins [first, first + count) of a finished launch's bounds
// (count <= blockDim.x), recounting those at or above 2^32. All threads of the
// CTA call it; `scratch` holds 256 64-bit words and an int list of blockDim.x.
template <typename T>
__device__ void bin_settle_chunk(unsigned long long* bound, const int4* geo, const T* phi, int N,
                                 int L, int nbx, int first, int count, uint32_t* flags,
                                 unsigned int* recounts, char* scratch) {
    const int i = first + (int)threadIdx.x;
    bool hot = false;
    if ((int)threadIdx.x < count) {
        const unsigned long long v = bound[i];
        if (v) {
            hot = v >= (1ull << 32);
            bound[i] = 0ull;
        }
    }
    if (!__syncthreads_or(hot)) return;
    bin_settle_hot<T>(bound, geo, phi, N, L, nbx, i, hot, flags, recounts, scratch);
}

// The rare part of bin_settle_chunk: recount the chunk's hot bins one by one.
template <typename T>
__device__ __noinline__ void bin_settle_hot(unsigned long long* bound, const int4* geo,
                                            const T* phi, int N, int L, int nbx, int i, bool hot,
                                            uint32_t* flags, unsigned int* recounts,
                                            char* scratch) {
    unsigned long long* acc = reinterpret_cast<unsigned long long*>(scratch);
    int* list = reinterpret_cast<int*>(scratch + 256 * sizeof(unsigned long long));
    int* nlist = list + blockDim.x;
    if (threadIdx.x == 0) *nlist = 0;
    __syncthreads();
    if (hot) list[atomicAdd(nlist, 1)] = i;
    __syncthreads();
    const int n = *nlist;
    for (int k = 0; k < n; ++k) {
        const int bin = list[k];
        if (bin_recount<T>(phi, geo, N, L, nbx, bin, acc) && threadIdx.x == 0)
            atomicOr(flags + PFB_FLAG_S_OVERFLOW, 1u);
        if (threadIdx.x == 0) atomicAdd(recounts, 1u);
        __syncthreads();
    }
}

// Running per-thread moments of destination pixels.
struct PixelAcc {
    double V = 0.0, Cx = 0.0, Cy = 0.0, Per = 0.0;
    int blox, bhix = -1, bloy, bhiy = -1, pmaxb = 0;
};

// Flags, phi_max, Q5.27 scatter and moments of one destination pixel.
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

// Commit of one cell's step (reference src/kernels.cu:573-590, :914-935).
// m = {V, Cx, Cy, perimeter}, b = {lo_x, hi_x, lo_y, hi_y, phi_max bits}.
__device__ __forceinline__ void commit_cell(const pfb_step_args2d& A, const CellPlan& P,
                                            bool fm, const double* m, const int* b) {
    pfb_cell2d& cs = A.cell[P.n];
    cs.gx0 = P.gx0n;
    cs.gy0 = P.gy0n;
    cs.cls = (uint8_t)P.dcls;
    cs.cls_written[A.parity_out] = (uint8_t)P.dcls;
    cs.theta = P.theta;
    cs.V = m[0];
    cs.Cx = m[1];
    cs.Cy = m[2];
    if (fm) cs.perim = m[3];
    cs.bb_lo_x = b[0];
    cs.bb_hi_x = b[1];
    cs.bb_lo_y = b[2];
    cs.bb_hi_y = b[3];
    cs.promote_ctr = (uint32_t)P.pctr;
    cs.shift_ctr += (P.sx | P.sy) ? 1u : 0u;
    cs.tumble_ctr += (uint32_t)P.tumbled;
    cs.phi_max = __uint_as_float((uint32_t)b[4]);
    A.cell_cls[P.n] = (uint8_t)P.dcls;
    if (P.cls == kClassFallback) {
        const bool edge =
            b[1] >= 0 && (b[0] == 0 || b[1] == P.dwx - 1 || b[2] == 0 || b[3] == P.dwy - 1);
        cs.reserved[0] = 1u;
        if (P.no_margin || (P.dcls == kClassFallback && edge)) ++cs.reserved[1];
    }
}

// Reduction scratch in shared memory. Cluster reductions push each CTA's
// partial into its peers' receive slots with st.async, completing on the
// peer's mbarrier: no cluster barrier (and no release fence over the CTA's
// outstanding global stores) sits on the path. Receive slots are indexed by
// the sender's rank and summed in ascending rank order.
// The spatial velocity observer's six sums (Bx, By, Gx, Gy, Kx, Ky) travel
// with the force in their own arrays at the end of the scratch (NO = 6), so
// the layout of every other kernel is unchanged.
template <int NW, int K, int NO>
struct ObsRed {
    double d[NW][NO];
    alignas(16) double recv[K][NO];
};
template <int NW, int K>
struct ObsRed<NW, K, 0> {};

template <int NW, int K, int NO = 0>
struct RedScratch {
    uint64_t barI;  // K force partials (16 B, + 8 NO B) received, every CTA
    uint64_t barM;  // K moment partials (64 B each) received, rank 0
    double red_d[NW][4];
    int red_i[NW][5];
    alignas(16) double recvI[K][2];
    alignas(16) double recvM[K][4];
    alignas(16) int recvB[K][4];
    alignas(16) int recvP[K][4];
    float vx, vy;
    ObsRed<NW, K, NO> o;
};

// ---- velocity observers (reference include/fused_moments.cuh) -------------
// OBS 0: none; 1: advection accumulators; 2: advection plus the spatial
// rates. The spatial observer adds six sums to the force reduction: the
// same-cell neighbour overlaps Bx, By, the interfacial moments Gx, Gy and the
// overlap moments Kx, Ky.
template <int OBS> constexpr int kObsVals = OBS == PFB_VELOCITY_SPATIAL ? 6 : 0;

template <int OBS> struct ObsAcc {
    __device__ __forceinline__ void pixel(const CellPlan&, float, int, int, float, float, float,
                                          float, float, float, float, float, float, float) {}
    __device__ __forceinline__ double val(int) const { return 0.0; }
};

template <> struct ObsAcc<PFB_VELOCITY_SPATIAL> {
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // Bx, By, Gx, Gy, Kx, Ky
    // One pixel of phi^n at window (x, y) with its eight neighbours and
    // S_other, in FP64 from the binary32 inputs.
    __device__ __forceinline__ void pixel(const CellPlan& P, float repC, int x, int y, float p,
                                          float e, float w, float nn, float ss, float ne,
                                          float nw, float se, float sw, float other) {
        const double d = p;
        v[0] += d * (double)e;
        v[1] += d * (double)nn;
        const double lap =
            (4.0 * ((double)nn + ss + e + w) + (double)ne + nw + se + sw - 20.0 * d) / 6.0;
        const double weight = P.ginv * d;
        const double inter =
            weight * ((double)P.gam * lap - (double)P.dwC * d * (1.0 - d) * (1.0 - 2.0 * d));
        const double ox = (double)x - P.gcx, oy = (double)y - P.gcy;
        v[2] += ox * inter;
        v[3] += oy * inter;
        const double over = -weight * (double)repC * d * (double)other;
        v[4] += ox * over;
        v[5] += oy * over;
    }
    __device__ __forceinline__ double val(int j) const { return v[j]; }
};

__device__ __forceinline__ double linear_corr(double dt, unsigned long long steps, double first,
                                              double last) {
    return steps ? dt * 0.5 * (double)(steps - 1) * (last - first) : 0.0;
}

// Observer commit of one cell by one thread once the cluster totals
// t = {Ix, Iy, Bx, By, Gx, Gy, Kx, Ky} are known (reference
// record_advection and RelaxMoments::finish): the spatial observer first
// closes the interval held since its previous sample, then the advection
// integrals advance, then the new rates replace the held ones.
template <int OBS>
__device__ __forceinline__ void observe_commit(const pfb_step_args2d& A, const CellPlan& P,
                                               const double* t, float vxf, float vyf) {
    if constexpr (OBS != PFB_VELOCITY_DISABLED) {
        pfb_cell2d& c = A.cell[P.n];
        pfb_advection_accum& a = c.advection;
        const double dt = A.physical_dt;
        const double ax = (double)P.vA * (double)P.pcos, ay = (double)P.vA * (double)P.psin;
        const double ix = (double)A.mot_coeff * t[0], iy = (double)A.mot_coeff * t[1];
        if constexpr (OBS == PFB_VELOCITY_SPATIAL) {
            pfb_moment_accum2d& m = static_cast<pfb_moment_accum2d*>(A.moments)[P.n];
            const double tot[4] = {a.q[0] + a.q[2], a.q[1] + a.q[3], a.q[4], a.q[5]};
            const unsigned long long interval = a.count - m.last_sample;
            if (m.spatial_count) {
                for (int j = 0; j < 4; ++j) m.q[4 + j] += dt * (double)interval * m.held[j];
                for (int xy = 0; xy < 2; ++xy) {
                    const double beta = m.held[4 + xy];
                    m.q[10 + xy] += (beta - 1.0) * (tot[xy] - m.last_totals[xy]) +
                                    beta * (tot[2 + xy] - m.last_totals[2 + xy]);
                }
            }
            for (int j = 0; j < 4; ++j) m.last_totals[j] = tot[j];
            m.last_interval = interval;
            m.last_sample = a.count;
            ++m.spatial_count;
            m.held[4] = t[2] / c.V;
            m.held[5] = t[3] / c.V;
        }
        a.q[0] += dt * ax;
        a.q[1] += dt * ay;
        a.q[2] += dt * ix;
        a.q[3] += dt * iy;
        a.q[4] += dt * ((double)vxf - ax - ix);
        a.q[5] += dt * ((double)vyf - ay - iy);
        ++a.count;
        if constexpr (OBS == PFB_VELOCITY_SPATIAL) {
            pfb_moment_accum2d& m = static_cast<pfb_moment_accum2d*>(A.moments)[P.n];
            const double mrel = (double)c.M_pf / kMobilityM0;
            for (int j = 0; j < 4; ++j) {
                double rate = t[4 + j];
                if (mrel != 1.0) rate *= mrel;
                if (m.spatial_count > 1)
                    m.correction[j] += linear_corr(dt, m.last_interval, m.held[j], rate);
                m.held[j] = rate;
            }
        }
    }
}

// Receive barriers of one cluster reduction round; thread 0 of every CTA
// calls it before the kernel's first (relaxed) cluster arrive.
template <int NW, int K, int NO>
__device__ __forceinline__ void red_init(RedScratch<NW, K, NO>& R, int rank) {
    dev::mbar_init(&R.barI, 1);
    dev::mbar_init(&R.barM, 1);
    dev::mbar_arrive_expect_tx(&R.barI, (uint32_t)(K * (16 + 8 * NO)));
    if (rank == 0) dev::mbar_arrive_expect_tx(&R.barM, (uint32_t)(K * 64));
}

// Interaction integral of this CTA -> cluster total -> velocity, identical
// in every CTA. Sums run in ascending warp, then ascending rank order. Rank 0
// stores v and I in the cell record and commits the velocity observer. All
// threads call it; the caller has issued the cluster arrive that follows
// red_init.
template <int K, int NW, int OBS, int NO>
__device__ __forceinline__ void reduce_force(const pfb_step_args2d& A, const CellPlan& P,
                                             int rank, RedScratch<NW, K, NO>& R, double aIx,
                                             double aIy, const ObsAcc<OBS>& ob,
                                             unsigned int* status) {
    static_assert(NW <= 32 && K <= 32, "one lane per warp and per rank");
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if constexpr (OBS != PFB_VELOCITY_SPATIAL) {
        aIx = dev::warp_sum_down(aIx);
        aIy = dev::warp_sum_down(aIy);
        if (lane == 0) {
            R.red_d[warp][0] = aIx;
            R.red_d[warp][1] = aIy;
        }
        __syncthreads();
        dev::cluster_wait();  // every peer's receive barrier is initialised
        if (warp == 0) {
            const double px = lane < NW ? R.red_d[lane][0] : 0.0;
            const double py = lane < NW ? R.red_d[lane][1] : 0.0;
            const double s0 = dev::ordered_lane_sum(px, NW);
            const double s1 = dev::ordered_lane_sum(py, NW);
            if (lane < K)
                dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&R.recvI[rank][0]), lane), s0,
                                    s1, dev::map_to_rank(dev::smem_addr(&R.barI), lane));
            if (!dev::mbar_wait_bounded(&R.barI, 0, kWaitPolls)) atomicOr(status, 2u);
            const double2 v = lane < K ? make_double2(R.recvI[lane][0], R.recvI[lane][1])
                                       : make_double2(0.0, 0.0);
            const double sIx = dev::ordered_lane_sum(v.x, K);
            const double sIy = dev::ordered_lane_sum(v.y, K);
            if (lane == 0) {
                const double vxd = (double)P.vA * (double)P.pcos + (double)A.mot_coeff * sIx;
                const double vyd = (double)P.vA * (double)P.psin + (double)A.mot_coeff * sIy;
                R.vx = (float)vxd;
                R.vy = (float)vyd;
                if (rank == 0) {
                    pfb_cell2d& cs = A.cell[P.n];
                    cs.vx = (float)vxd;
                    cs.vy = (float)vyd;
                    cs.Ix = sIx;
                    cs.Iy = sIy;
                    if constexpr (OBS == PFB_VELOCITY_ADVECTION) {
                        const double t[2] = {sIx, sIy};
                        observe_commit<OBS>(A, P, t, (float)vxd, (float)vyd);
                    }
                }
            }
        }
        __syncthreads();
    } else {
        // the spatial observer's six sums travel with the force
        static_assert(NO == 6, "observer scratch");
        const double fx = dev::warp_sum_down(aIx);
        const double fy = dev::warp_sum_down(aIy);
        double part[NO];
#pragma unroll
        for (int j = 0; j < NO; ++j) part[j] = dev::warp_sum_down(ob.val(j));
        if (lane == 0) {
            R.red_d[warp][0] = fx;
            R.red_d[warp][1] = fy;
#pragma unroll
            for (int j = 0; j < NO; ++j) R.o.d[warp][j] = part[j];
        }
        __syncthreads();
        dev::cluster_wait();
        if (warp == 0) {
            double s[2 + NO];
            s[0] = dev::ordered_lane_sum(lane < NW ? R.red_d[lane][0] : 0.0, NW);
            s[1] = dev::ordered_lane_sum(lane < NW ? R.red_d[lane][1] : 0.0, NW);
#pragma unroll
            for (int j = 0; j < NO; ++j)
                s[2 + j] = dev::ordered_lane_sum(lane < NW ? R.o.d[lane][j] : 0.0, NW);
            if (lane < K) {
                const uint32_t bar = dev::map_to_rank(dev::smem_addr(&R.barI), lane);
                dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&R.recvI[rank][0]), lane), s[0],
                                    s[1], bar);
#pragma unroll
                for (int j = 0; j < NO; j += 2)
                    dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&R.o.recv[rank][j]), lane),
                                        s[2 + j], s[3 + j], bar);
            }
            if (!dev::mbar_wait_bounded(&R.barI, 0, kWaitPolls)) atomicOr(status, 2u);
            double t[2 + NO];
            t[0] = dev::ordered_lane_sum(lane < K ? R.recvI[lane][0] : 0.0, K);
            t[1] = dev::ordered_lane_sum(lane < K ? R.recvI[lane][1] : 0.0, K);
#pragma unroll
            for (int j = 0; j < NO; ++j)
                t[2 + j] = dev::ordered_lane_sum(lane < K ? R.o.recv[lane][j] : 0.0, K);
            if (lane == 0) {
                const double vxd = (double)P.vA * (double)P.pcos + (double)A.mot_coeff * t[0];
                const double vyd = (double)P.vA * (double)P.psin + (double)A.mot_coeff * t[1];
                R.vx = (float)vxd;
                R.vy = (float)vyd;
                if (rank == 0) {
                    pfb_cell2d& cs = A.cell[P.n];
                    cs.vx = (float)vxd;
                    cs.vy = (float)vyd;
                    cs.Ix = t[0];
                    cs.Iy = t[1];
                    observe_commit<OBS>(A, P, t, (float)vxd, (float)vyd);
                }
            }
        }
        __syncthreads();
    }
}

// Moments of this CTA -> pushed to rank 0 -> summed in rank order and
// committed by rank 0 (reference src/kernels.cu:542-590).
template <int K, int NW, int NO>
__device__ __forceinline__ void reduce_moments(const pfb_step_args2d& A, const CellPlan& P,
                                               int rank, RedScratch<NW, K, NO>& R, bool fm,
                                               PixelAcc acc, unsigned int* status) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    acc.V = dev::warp_sum_down(acc.V);
    acc.Cx = dev::warp_sum_down(acc.Cx);
    acc.Cy = dev::warp_sum_down(acc.Cy);
    acc.Per = dev::warp_sum_down(acc.Per);
    acc.blox = dev::warp_min_down(acc.blox);
    acc.bhix = dev::warp_max_down(acc.bhix);
    acc.bloy = dev::warp_min_down(acc.bloy);
    acc.bhiy = dev::warp_max_down(acc.bhiy);
    acc.pmaxb = dev::warp_max_down(acc.pmaxb);
    if (lane == 0) {
        R.red_d[warp][0] = acc.V;
        R.red_d[warp][1] = acc.Cx;
        R.red_d[warp][2] = acc.Cy;
        R.red_d[warp][3] = acc.Per;
        R.red_i[warp][0] = acc.blox;
        R.red_i[warp][1] = acc.bhix;
        R.red_i[warp][2] = acc.bloy;
        R.red_i[warp][3] = acc.bhiy;
        R.red_i[warp][4] = acc.pmaxb;
    }
    __syncthreads();
    if (warp != 0) return;  // callers that need the whole CTA afterwards re-join it
    double m[4];
    for (int k = 0; k < 4; ++k) m[k] = dev::ordered_lane_sum(lane < NW ? R.red_d[lane][k] : 0.0, NW);
    const int b0 = __reduce_min_sync(0xFFFFFFFFu, lane < NW ? R.red_i[lane][0] : P.dwx);
    const int b1 = __reduce_max_sync(0xFFFFFFFFu, lane < NW ? R.red_i[lane][1] : -1);
    const int b2 = __reduce_min_sync(0xFFFFFFFFu, lane < NW ? R.red_i[lane][2] : P.dwy);
    const int b3 = __reduce_max_sync(0xFFFFFFFFu, lane < NW ? R.red_i[lane][3] : -1);
    const int b4 = __reduce_max_sync(0xFFFFFFFFu, lane < NW ? R.red_i[lane][4] : 0);
    if (lane == 0) {
        const uint32_t bar = dev::map_to_rank(dev::smem_addr(&R.barM), 0);
        dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&R.recvM[rank][0]), 0), m[0], m[1], bar);
        dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&R.recvM[rank][2]), 0), m[2], m[3], bar);
        dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&R.recvB[rank][0]), 0), b0, b1, b2, b3,
                            bar);
        dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&R.recvP[rank][0]), 0), b4, 0, 0, 0,
                            bar);
    }
    if (rank != 0) return;
    if (!dev::mbar_wait_bounded(&R.barM, 0, kWaitPolls)) atomicOr(status, 2u);
    double t[4];
    for (int k = 0; k < 4; ++k) t[k] = dev::ordered_lane_sum(lane < K ? R.recvM[lane][k] : 0.0, K);
    int b[5];
    b[0] = __reduce_min_sync(0xFFFFFFFFu, lane < K ? R.recvB[lane][0] : P.dwx);
    b[1] = __reduce_max_sync(0xFFFFFFFFu, lane < K ? R.recvB[lane][1] : -1);
    b[2] = __reduce_min_sync(0xFFFFFFFFu, lane < K ? R.recvB[lane][2] : P.dwy);
    b[3] = __reduce_max_sync(0xFFFFFFFFu, lane < K ? R.recvB[lane][3] : -1);
    b[4] = __reduce_max_sync(0xFFFFFFFFu, lane < K ? R.recvP[lane][0] : 0);
    if (lane == 0) commit_cell(A, P, fm, t, b);
}

// Global-memory path for classes 4 (224^2) and 5 (286^2 fallback): phi^n is
// read from the tile (its zero ring is the tile invariant), phi^{n+1} is
// written to the shifted destination in global memory, and after a cluster
// barrier each CTA re-reads its destination rows for scatter and moments
// (reference src/kernels.cu:344-443 and :604-937). All NT threads of every CTA
// of the cluster call it together.
template <int CLS, int K, int NW, int OBS = PFB_VELOCITY_DISABLED>
__device__ __noinline__ void global_cell(const pfb_step_args2d& A, const CellPlan& P, int rank,
                                         RedScratch<NW, K, kObsVals<OBS>>& R, bool fm,
                                         unsigned int* status,
                                         unsigned long long* bound = nullptr, int nbx = 0,
                                         int nby = 0, int* slot = nullptr) {
    constexpr int NT = NW * 32;
    constexpr Window W = window_of(CLS);
    constexpr int WX = W.wx, WY = W.wy, TX0 = W.tx0, TY0 = W.ty0;
    constexpr int RB = (WY + K - 1) / K;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int y0 = min(WY, rank * RB);
    const int y1 = min(WY, y0 + RB);
    const int L = A.L, Pp = A.P;
    const float* tin = A.phi_in + (size_t)P.n * kTileArea + (size_t)TY0 * kTilePitch + TX0;
    float* tile_out = A.phi_out + (size_t)P.n * kTileArea;
    const int gx0 = P.gx0, gy0 = P.gy0;
    const int split = min(WX, L - gx0);

    double aIx = 0.0, aIy = 0.0;
    ObsAcc<OBS> ob;
    const int cnt = (y1 - y0) * WX;
    for (int idx = tid; idx < cnt; idx += NT) {
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
        const float So = s_other_n(__ldg(A.S_rd + (size_t)gy * Pp + gxg), c, A.flags, 1u);
        aIx += (double)(c * gx * So);
        aIy += (double)(c * gyv * So);
        if constexpr (OBS == PFB_VELOCITY_SPATIAL)
            ob.pixel(P, A.rep_coeff, x, y, c, __ldg(p + 1), __ldg(p - 1), __ldg(p + kTilePitch),
                     __ldg(p - kTilePitch), __ldg(p + kTilePitch + 1), __ldg(p + kTilePitch - 1),
                     __ldg(p - kTilePitch + 1), __ldg(p - kTilePitch - 1), So);
    }
    reduce_force<K, NW, OBS>(A, P, rank, R, aIx, aIy, ob, status);

    const int sx = P.sx, sy = P.sy;
    const int dwx = P.dwx, dwy = P.dwy, dtx0 = P.dtx0, dty0 = P.dty0;
    if (P.zero_tile) {
        for (int t = rank + K * warp; t < kTilePitch; t += K * NW) {
            float* trow = tile_out + (size_t)t * kTilePitch;
            for (int c = lane; c < kTilePitch; c += 32) trow[c] = 0.0f;
        }
        dev::cluster_sync();
    }
    {
        const float gam = P.gam, dwC = P.dwC, volC = P.volC, mrel = P.mrel;
        const float vx = R.vx, vy = R.vy;
        const float repC = A.rep_coeff, dtf = A.dt;
        for (int idx = tid; idx < cnt; idx += NT) {
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
            const float So = s_other_n(__ldg(A.S_rd + (size_t)gy * Pp + gxg), cC, A.flags, 1u);
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
    for (int b = db0 + warp; b < db1; b += NW) {
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
    for (int b = db0 + warp; b < db1; b += NW) {
        int gy = P.gy0n + b;
        if (gy >= L) gy -= L;
        const float* orow = tile_out + (size_t)(dty0 + b) * kTilePitch + dtx0;
        uint32_t* srow = A.S_sc + (size_t)gy * Pp;
        for (int a = lane; a < dwx; a += 32) {
            const float pn = __ldcg(orow + a);
            dest_pixel(A, acc, pn, a, b, srow, P.gx0n, L);
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
    // returning adds, but the launch also has non-returning ones elsewhere:
    // bound this CTA's destination band (the whole CTA calls it)
    if (bound) bin_box_add(bound, nbx, nby, acc.pmaxb, db0, db1, P.dwx, P.gx0n, P.gy0n, L, slot);
    reduce_moments<K, NW>(A, P, rank, R, fm, acc, status);
}

}  // namespace pfb
