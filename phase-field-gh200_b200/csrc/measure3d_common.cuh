// Device pieces of the 3D measurement shared by the standalone measurement
// (k_measure3d) and the fused step (k_step3d): the per-voxel sums of one
// strip item, the cluster fold of the partial sums into rank 0, the commit
// of the measured record with its recentring plan, and the cell motion.
//
// Per-voxel semantics follow measure_one_cell (reference
// src/pf3d/kernels.cu:1271-1409); the commit follows commit_measurement
// (src/pf3d/kernels.cu:418-497) and the motion k_apply_cell_motion
// (src/pf3d/kernels.cu:1739-1788).
#pragma once

#include <cuda_runtime.h>

#include "device_util.cuh"
#include "pfb3d_common.cuh"
#include "phi3d.cuh"

namespace pfb {
namespace p3 {

constexpr int kThreads3 = 256;
constexpr int kWarps3 = kThreads3 / 32;

struct Acc3 {
    double V = 0.0, Cx = 0.0, Cy = 0.0, Cz = 0.0, Sf = 0.0, Ix = 0.0, Iy = 0.0, Iz = 0.0;
    int lox, hix = -1, loy, hiy = -1, loz, hiz = -1;
    unsigned pmax = 0u;
};

// Counted flags of the measurement: non-finite samples, aggregate below the
// cell's own contribution, support on the slab's top plane.
struct MeasureCounts {
    unsigned nonfinite = 0u, negative = 0u, top = 0u;
};

// Per-cell constants of a measurement sweep.
struct MeasureCell {
    const uint32_t* S;
    pfb_layout3d L;
    int B, ox, oy;
    bool wall;     // hard-wall channel: the wall field adds to the other-cell term
    bool surface;  // accumulate the surface proxy
};

// Six values of row y of a plane: columns x0 - 1 .. x0 + 4 (zero outside).
template <typename T>
__device__ __forceinline__ void load_row6(const T* plane, int B, int y, int x0, float* v) {
    if ((unsigned)y >= (unsigned)B) {
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = 0.0f;
        return;
    }
    const T* row = plane + y * B;
    phi_ld4(row + x0, v + 1);
    v[0] = x0 > 0 ? phi_ld1(row + x0 - 1) : 0.0f;
    v[5] = x0 + 4 < B ? phi_ld1(row + x0 + 4) : 0.0f;
}

// Sums of one item: columns x0 .. x0 + 3 of rows y0 .. y0 + 3 of brick plane
// z (world plane wz); pm, pc, pp are planes z - 1, z, z + 1.
template <typename T = float>
__device__ __forceinline__ void measure_item(const MeasureCell& M, const T* pm,
                                             const T* pc, const T* pp, int x0, int y0,
                                             int z, int wz, float wallv, bool top_plane,
                                             Acc3& acc, MeasureCounts& cnt) {
    const int B = M.B;
    const pfb_layout3d& L = M.L;
    float rs[6], rc[6], rn[6];
    load_row6(pc, B, y0 - 1, x0, rs);
    load_row6(pc, B, y0, x0, rc);
    int wxj[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) wxj[j] = wrap_offset(M.ox, x0 + j, L.nx);
    // aggregate words of a row, fetched one row ahead
    auto load_agg = [&](int y, uint32_t* out) {
        const size_t srow = s_index(L, 0, wrap_offset(M.oy, y, L.ny), wz);
#pragma unroll
        for (int j = 0; j < 4; ++j) out[j] = __ldg(M.S + srow + wxj[j]);
    };
    uint32_t agg_next[4];
    load_agg(y0, agg_next);
#pragma unroll 1
    for (int r = 0; r < 4; ++r) {
        const int y = y0 + r;
        load_row6(pc, B, y + 1, x0, rn);
        float zmv[4], zpv[4];
        phi_ld4(pm + y * B + x0, zmv);
        phi_ld4(pp + y * B + x0, zpv);
        uint32_t agg[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) agg[j] = agg_next[j];
        if (r < 3) load_agg(y + 1, agg_next);
        double rV = 0.0, rX = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float c = rc[j + 1];
            const bool cfin = isfinite(c);
            cnt.nonfinite += cfin ? 0u : 1u;
            const float gx = 0.5f * (rc[j + 2] - rc[j]);
            const float gy = 0.5f * (rn[j + 1] - rs[j + 1]);
            const float gz = 0.5f * (zpv[j] - zmv[j]);
            const uint32_t own = q_of3(c);
            const bool nz = cfin && c != 0.0f;
            const bool neg = nz && agg[j] < own;
            cnt.negative += neg ? 1u : 0u;
            float other = (nz && !neg) ? (float)(agg[j] - own) * kQInv : 0.0f;
            if (M.wall) other += wallv;
            const double sq = cfin ? (double)c * (double)c : 0.0;
            rV += sq;
            rX += sq * (double)j;
            if (M.surface && cfin)
                acc.Sf += sqrt((double)gx * gx + (double)gy * gy + (double)gz * gz);
            acc.Ix += cfin ? (double)(c * gx * other) : 0.0;
            acc.Iy += cfin ? (double)(c * gy * other) : 0.0;
            acc.Iz += cfin ? (double)(c * gz * other) : 0.0;
            if (cfin) acc.pmax = max(acc.pmax, __float_as_uint(fabsf(c)));
            const int x = x0 + j;
            if (cfin && fabsf(c) > kSupportEps3) {
                if (top_plane) ++cnt.top;
                acc.lox = min(acc.lox, x);
                acc.hix = max(acc.hix, x);
                acc.loy = min(acc.loy, y);
                acc.hiy = max(acc.hiy, y);
                acc.loz = min(acc.loz, z);
                acc.hiz = max(acc.hiz, z);
            }
        }
        acc.V += rV;
        acc.Cx += rV * (double)x0 + rX;
        acc.Cy += rV * (double)y;
        acc.Cz += rV * (double)z;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            rs[c] = rc[c];
            rc[c] = rn[c];
        }
    }
}

// ---- cluster fold -----------------------------------------------------------
// Bytes one rank pushes into rank 0: 8 sums, 8 integers, 4 counts.
constexpr uint32_t kFoldBytes = 8 * 8 + 8 * 4 + 4 * 4;

template <int K>
struct MeasureFold {
    uint64_t bar;  // rank 0: completes when all K records have landed
    int pad[2];
    double wd[kWarps3][8];
    int wi[kWarps3][8];
    unsigned wc[kWarps3][4];
    alignas(16) double rd[K][8];
    alignas(16) int ri[K][8];  // support box (6), phi_max bits, 0
    alignas(16) unsigned rc[K][4];
};

// Result of the fold (in every lane of rank 0's warp 0).
struct MeasureTotals {
    double t[8];  // V, Cx, Cy, Cz, surface, Ix, Iy, Iz
    int lo_x, hi_x, lo_y, hi_y, lo_z, hi_z;
    unsigned pmax_bits;
    unsigned nonfinite, negative, top;
};

// Thread 0; the caller publishes the initialisation to the cluster.
template <int K>
__device__ __forceinline__ void fold_init(MeasureFold<K>& F, int rank) {
    dev::mbar_init(&F.bar, 1);
    if (rank == 0) dev::mbar_arrive_expect_tx(&F.bar, (uint32_t)K * kFoldBytes);
}

// Every thread: warp sums of its partial record into F.w*. The caller
// synchronises the CTA afterwards.
template <int K>
__device__ __forceinline__ void fold_warps(MeasureFold<K>& F, Acc3& acc, MeasureCounts c) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    c.nonfinite = __reduce_add_sync(0xFFFFFFFFu, c.nonfinite);
    c.negative = __reduce_add_sync(0xFFFFFFFFu, c.negative);
    c.top = __reduce_add_sync(0xFFFFFFFFu, c.top);
    acc.V = dev::warp_sum_down(acc.V);
    acc.Cx = dev::warp_sum_down(acc.Cx);
    acc.Cy = dev::warp_sum_down(acc.Cy);
    acc.Cz = dev::warp_sum_down(acc.Cz);
    acc.Sf = dev::warp_sum_down(acc.Sf);
    acc.Ix = dev::warp_sum_down(acc.Ix);
    acc.Iy = dev::warp_sum_down(acc.Iy);
    acc.Iz = dev::warp_sum_down(acc.Iz);
    const int b0 = __reduce_min_sync(0xFFFFFFFFu, acc.lox), b1 = __reduce_max_sync(0xFFFFFFFFu, acc.hix);
    const int b2 = __reduce_min_sync(0xFFFFFFFFu, acc.loy), b3 = __reduce_max_sync(0xFFFFFFFFu, acc.hiy);
    const int b4 = __reduce_min_sync(0xFFFFFFFFu, acc.loz), b5 = __reduce_max_sync(0xFFFFFFFFu, acc.hiz);
    const unsigned pm = __reduce_max_sync(0xFFFFFFFFu, acc.pmax);
    if (lane == 0) {
        double* d = F.wd[warp];
        d[0] = acc.V; d[1] = acc.Cx; d[2] = acc.Cy; d[3] = acc.Cz;
        d[4] = acc.Sf; d[5] = acc.Ix; d[6] = acc.Iy; d[7] = acc.Iz;
        int* q = F.wi[warp];
        q[0] = b0; q[1] = b1; q[2] = b2; q[3] = b3; q[4] = b4; q[5] = b5; q[6] = (int)pm; q[7] = 0;
        F.wc[warp][0] = c.nonfinite;
        F.wc[warp][1] = c.negative;
        F.wc[warp][2] = c.top;
        F.wc[warp][3] = 0u;
    }
}

// Warp 0 of every rank, after the CTA barrier and after rank 0's barrier is
// known to be initialised: the CTA's record (warps in ascending order) is
// pushed into rank 0's slot `rank`.
template <int K>
__device__ __forceinline__ void fold_send(MeasureFold<K>& F, int rank, int B) {
    const int lane = threadIdx.x & 31;
    double s[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        s[k] = dev::ordered_lane_sum(lane < kWarps3 ? F.wd[lane][k] : 0.0, kWarps3);
    int v[8];
    v[0] = __reduce_min_sync(0xFFFFFFFFu, lane < kWarps3 ? F.wi[lane][0] : B);
    v[1] = __reduce_max_sync(0xFFFFFFFFu, lane < kWarps3 ? F.wi[lane][1] : -1);
    v[2] = __reduce_min_sync(0xFFFFFFFFu, lane < kWarps3 ? F.wi[lane][2] : B);
    v[3] = __reduce_max_sync(0xFFFFFFFFu, lane < kWarps3 ? F.wi[lane][3] : -1);
    v[4] = __reduce_min_sync(0xFFFFFFFFu, lane < kWarps3 ? F.wi[lane][4] : B);
    v[5] = __reduce_max_sync(0xFFFFFFFFu, lane < kWarps3 ? F.wi[lane][5] : -1);
    v[6] = (int)__reduce_max_sync(0xFFFFFFFFu, lane < kWarps3 ? (unsigned)F.wi[lane][6] : 0u);
    v[7] = 0;
    unsigned cn[3];
#pragma unroll
    for (int f = 0; f < 3; ++f)
        cn[f] = __reduce_add_sync(0xFFFFFFFFu, lane < kWarps3 ? F.wc[lane][f] : 0u);
    if (lane == 0) {
        const uint32_t bar = dev::map_to_rank(dev::smem_addr(&F.bar), 0);
#pragma unroll
        for (int k = 0; k < 8; k += 2)
            dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&F.rd[rank][k]), 0), s[k],
                                s[k + 1], bar);
        dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&F.ri[rank][0]), 0), v[0], v[1],
                            v[2], v[3], bar);
        dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&F.ri[rank][4]), 0), v[4], v[5],
                            v[6], v[7], bar);
        dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&F.rc[rank][0]), 0), (int)cn[0],
                            (int)cn[1], (int)cn[2], 0, bar);
    }
}

// Warp 0 of rank 0: wait for the K records and fold them in rank order.
// false when the wait gave up (the totals are then meaningless).
template <int K>
__device__ __forceinline__ bool fold_receive(MeasureFold<K>& F, int B, uint32_t polls,
                                             MeasureTotals& r) {
    const int lane = threadIdx.x & 31;
    const bool ok = dev::mbar_wait_bounded(&F.bar, 0, polls);
#pragma unroll
    for (int k = 0; k < 8; ++k) r.t[k] = dev::ordered_lane_sum(lane < K ? F.rd[lane][k] : 0.0, K);
    r.lo_x = __reduce_min_sync(0xFFFFFFFFu, lane < K ? F.ri[lane][0] : B);
    r.hi_x = __reduce_max_sync(0xFFFFFFFFu, lane < K ? F.ri[lane][1] : -1);
    r.lo_y = __reduce_min_sync(0xFFFFFFFFu, lane < K ? F.ri[lane][2] : B);
    r.hi_y = __reduce_max_sync(0xFFFFFFFFu, lane < K ? F.ri[lane][3] : -1);
    r.lo_z = __reduce_min_sync(0xFFFFFFFFu, lane < K ? F.ri[lane][4] : B);
    r.hi_z = __reduce_max_sync(0xFFFFFFFFu, lane < K ? F.ri[lane][5] : -1);
    r.pmax_bits = __reduce_max_sync(0xFFFFFFFFu, lane < K ? (unsigned)F.ri[lane][6] : 0u);
    r.nonfinite = __reduce_add_sync(0xFFFFFFFFu, lane < K ? F.rc[lane][0] : 0u);
    r.negative = __reduce_add_sync(0xFFFFFFFFu, lane < K ? F.rc[lane][1] : 0u);
    r.top = __reduce_add_sync(0xFFFFFFFFu, lane < K ? F.rc[lane][2] : 0u);
    return ok;
}

// Sticky cell flag plus `count` on the global counter; returns the bit.
__device__ __forceinline__ uint32_t raise_counted(pfb_cell3d* cell, uint32_t* gflags, int flag,
                                                  unsigned count) {
    if (!count) return 0u;
    atomicOr(&cell->flags, 1u << flag);
    if (gflags) atomicAdd(&gflags[flag], count);
    return 1u << flag;
}

// Commit of the measured record (one thread): moments, support box,
// phi_max, the recentring plan and the support-margin check of a brick of
// edge B. Returns the flag bits raised for the cell; *sx, *sy, *sz receive
// the planned shift.
__device__ __forceinline__ uint32_t commit_measure(const pfb_measure_args3d& A, int B,
                                                   pfb_cell3d* cell, const MeasureTotals& r,
                                                   int* psx, int* psy, int* psz) {
    uint32_t raised = 0u;
    raised |= raise_counted(cell, A.global_flags, PFB3D_FLAG_NONFINITE, r.nonfinite);
    raised |= raise_counted(cell, A.global_flags, PFB3D_FLAG_S_NEGATIVE, r.negative);
    raised |= raise_counted(cell, A.global_flags, PFB3D_FLAG_SLAB_TOP_CONTACT, r.top);
    cell->V = r.t[0];
    cell->Cx = r.t[1];
    cell->Cy = r.t[2];
    cell->Cz = r.t[3];
    if (A.compute_surface) cell->surface = r.t[4];
    cell->Ix = r.t[5];
    cell->Iy = r.t[6];
    cell->Iz = r.t[7];
    cell->bb_lo_x = r.lo_x; cell->bb_hi_x = r.hi_x;
    cell->bb_lo_y = r.lo_y; cell->bb_hi_y = r.hi_y;
    cell->bb_lo_z = r.lo_z; cell->bb_hi_z = r.hi_z;
    cell->phi_max = __uint_as_float(r.pmax_bits);
    int sx = 0, sy = 0, sz = 0;
    const double V = r.t[0];
    if (V > 0.0 && isfinite(V)) {
        const double mid = 0.5 * (double)(B - 1);
        sx = clamp_shift(__double2int_rn(r.t[1] / V - mid), A.max_shift, r.lo_x, r.hi_x, B);
        sy = clamp_shift(__double2int_rn(r.t[2] / V - mid), A.max_shift, r.lo_y, r.hi_y, B);
        sz = clamp_shift(__double2int_rn(r.t[3] / V - mid), A.max_shift, r.lo_z, r.hi_z, B);
    } else {
        raised |= raise_counted(cell, A.global_flags, PFB3D_FLAG_V_NONPOSITIVE, 1u);
    }
    cell->pending_shift_x = sx;
    cell->pending_shift_y = sy;
    cell->pending_shift_z = sz;
    if (r.hi_x >= r.lo_x) {
        const int ex = r.hi_x - r.lo_x + 1, ey = r.hi_y - r.lo_y + 1, ez = r.hi_z - r.lo_z + 1;
        const int m = A.support_margin, ml = m / 2, mu = m - ml;
        if (ex + m > B || ey + m > B || ez + m > B || r.lo_x - sx < ml || r.hi_x - sx >= B - mu ||
            r.lo_y - sy < ml || r.hi_y - sy >= B - mu || r.lo_z - sz < ml || r.hi_z - sz >= B - mu)
            raised |= raise_counted(cell, A.global_flags, PFB3D_FLAG_SUPPORT_EXHAUSTED, 1u);
    }
    *psx = sx;
    *psy = sy;
    *psz = sz;
    return raised;
}

// Any fatal counter on the device (loads that bypass the L1: the counters
// are raised by atomics of other CTAs during the launch).
__device__ __forceinline__ bool fatal_counters(const uint32_t* g) {
    if (!g) return false;
    for (int f = 0; f < PFB3D_FLAG_COUNT; ++f)
        if (((PFB3D_FATAL_MASK >> f) & 1u) && __ldcg(g + f)) return true;
    return false;
}

// Tumble and velocity of one cell (one thread). `fatal`: the cell or the
// step already holds a fatal flag, nothing moves. Returns false when the
// new velocity is not finite (flag raised, record unchanged).
__device__ __forceinline__ bool motion_cell(const pfb_measure_args3d& A, pfb_cell3d* c, bool fatal,
                                            double Ix, double Iy, double Iz, float* vout) {
    if (fatal) {
        vout[0] = c->velocity_x;
        vout[1] = c->velocity_y;
        vout[2] = c->velocity_z;
        return true;
    }
    const unsigned long long step = A.step ? *A.step : 0ull;
    const bool active = step >= A.aging_steps;
    const bool slab = substrate_slab(A.layout.boundary_flags);
    double px = c->polarity_x, py = c->polarity_y, pz = c->polarity_z;
    bool tumbled = false;
    if (A.apply_tumble && active) {
        Dir3 d;
        if (tumble3(step - A.aging_steps, c->global_id, A.polarity_stream, A.p_tumble, slab, &d)) {
            px = d.x;
            py = d.y;
            pz = d.z;
            tumbled = true;
        }
    }
    const float fx = (float)px, fy = (float)py, fz = slab ? 0.0f : (float)pz;
    const float speed = active ? c->v_A : 0.0f;
    const float vx = speed * fx + A.motility_coeff * (float)Ix;
    const float vy = speed * fy + A.motility_coeff * (float)Iy;
    const float vz = slab ? 0.0f : speed * fz + A.motility_coeff * (float)Iz;
    if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz) || !isfinite(vx) || !isfinite(vy) ||
        !isfinite(vz)) {
        atomicOr(&c->flags, 1u << PFB3D_FLAG_NONFINITE);
        if (A.global_flags) atomicAdd(&A.global_flags[PFB3D_FLAG_NONFINITE], 1u);
        vout[0] = c->velocity_x;
        vout[1] = c->velocity_y;
        vout[2] = c->velocity_z;
        return false;
    }
    c->polarity_x = fx;
    c->polarity_y = fy;
    c->polarity_z = fz;
    c->velocity_x = vx;
    c->velocity_y = vy;
    c->velocity_z = vz;
    if (tumbled) ++c->tumble_ctr;
    vout[0] = vx;
    vout[1] = vy;
    vout[2] = vz;
    return true;
}

}  // namespace p3
}  // namespace pfb
