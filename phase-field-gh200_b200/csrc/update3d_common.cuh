// Device pieces of the 3D update shared by the standalone update
// (k_update3d) and the fused step (k_step3d): the 27-point stencil in the
// reference's z, y, x order, the phase-field right-hand side, the update of
// one strip item with its Q5.27 scatter, the keep path of a fatal step and
// the destination-clip check of a shifted cell.
//
// phi and S follow k_update_periodic_slab_walk_fast
// (reference src/pf3d/kernels_periodic_slab_walk.cu:54-318) and
// k_update_tiled_fast (src/pf3d/kernels.cu:498-793) bit for bit.
#pragma once

#include <cuda_runtime.h>

#include "device_util.cuh"
#include "pfb3d_common.cuh"
#include "phi3d.cuh"

namespace pfb {
namespace p3 {

__device__ __forceinline__ void raise3(pfb_cell3d* cell, uint32_t* gflags, int flag,
                                       unsigned count) {
    if (!count) return;
    atomicOr(&cell->flags, 1u << flag);
    if (gflags) atomicAdd(&gflags[flag], count);
}

__device__ __forceinline__ bool fatal3(const pfb_cell3d* cell, const uint32_t* gflags) {
    if (cell->flags & PFB3D_FATAL_MASK) return true;
    if (gflags)
        for (int f = 0; f < PFB3D_FLAG_COUNT; ++f)
            if (((PFB3D_FATAL_MASK >> f) & 1u) && gflags[f]) return true;
    return false;
}

// The 27-point Laplacian and centred gradients of column j (0..3) of the
// window w[plane][row][col], plane/row 0 = -1 offset: weights and the z, y, x
// summation order of the reference's stencil27_at.
__device__ __forceinline__ void stencil27w(const float (&w)[3][3][6], int j, float& lap,
                                           float& gx, float& gy, float& gz) {
    float acc = (float)kWCentre * w[1][1][j + 1];
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
                const int d = (dz != 1) + (dy != 1) + (dx != 1);
                if (d == 0) continue;
                const int wgt = d == 1 ? kWFace : d == 2 ? kWEdge : kWCorner;
                acc += (float)wgt * w[dz][dy][j + dx];
            }
    lap = acc * (float)(1.0 / 30.0);
    gx = 0.5f * (w[1][1][j + 2] - w[1][1][j]);
    gy = 0.5f * (w[1][2][j + 1] - w[1][0][j + 1]);
    gz = 0.5f * (w[2][1][j + 1] - w[0][1][j + 1]);
}

// Six source values of one row, columns xs0 - 1 .. xs0 + 4 (zero outside the
// brick or when the row is outside it); the alignment decision is taken once
// per strip.
template <typename T>
__device__ __forceinline__ void row6v(const T* plane, int B, int ys, int xs0, bool vec_ok, float* v) {
    if ((unsigned)ys >= (unsigned)B) {
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = 0.0f;
        return;
    }
    const T* row = plane + ys * B;
    if (vec_ok) {
        phi_ld4(row + xs0, v + 1);
        v[0] = xs0 > 0 ? phi_ld1(row + xs0 - 1) : 0.0f;
        v[5] = xs0 + 4 < B ? phi_ld1(row + xs0 + 4) : 0.0f;
    } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const int x = xs0 - 1 + c;
            v[c] = (unsigned)x < (unsigned)B ? phi_ld1(row + x) : 0.0f;
        }
    }
}

// stencil27w over a window whose rows rotate through slots: row offset -1,
// 0, +1 of every plane live in slots s0, s1, s2.
__device__ __forceinline__ void stencil27r(const float (&w)[3][3][6], int s0, int s1, int s2,
                                           int j, float& lap, float& gx, float& gy, float& gz) {
    const int sl[3] = {s0, s1, s2};
    float acc = (float)kWCentre * w[1][s1][j + 1];
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
                const int d = (dz != 1) + (dy != 1) + (dx != 1);
                if (d == 0) continue;
                const int wgt = d == 1 ? kWFace : d == 2 ? kWEdge : kWCorner;
                acc += (float)wgt * w[dz][sl[dy]][j + dx];
            }
    lap = acc * (float)(1.0 / 30.0);
    gx = 0.5f * (w[1][s1][j + 2] - w[1][s1][j]);
    gy = 0.5f * (w[1][s2][j + 1] - w[1][s0][j + 1]);
    gz = 0.5f * (w[2][s1][j + 1] - w[0][s1][j + 1]);
}

struct CellCoef {
    float gamma, bulk, volume, inter, vx, vy, vz, dt;
};

__device__ __forceinline__ float rhs3(const CellCoef& k, float c, float lap, float gx, float gy,
                                      float gz, float other) {
    return k.gamma * lap - k.bulk * c * (1.0f - c) * (1.0f - 2.0f * c) + k.volume * c -
           k.inter * c * other - (k.vx * gx + k.vy * gy + k.vz * gz);
}

// Per-cell constants of an update sweep.
struct UpdateCell {
    const uint32_t* S_in;
    uint32_t* S_out;  // null: no scatter
    pfb_layout3d L;
    int B, ox, oy;
    CellCoef k;
};

struct UpdateCounts {
    unsigned nf = 0u, neg = 0u, top = 0u, clamp = 0u, ovf = 0u;
};

// One item of destination plane dz: columns x0 .. x0 + 3 of rows
// y0 .. y0 + 3, read from source plane dz + sz (p1) and its neighbours p0,
// p2 at in-plane offset (sx, sy); `live` false (source plane outside the
// brick or the domain) writes zeros. orow points at (dz, y0, x0) of phi_out,
// voxel pix0 of the brick (16-bit pools: rounding stream sr).
// GEO: 0 periodic, 1 substrate slab, 2 hard-wall channel.
template <int GEO, typename T = float>
__device__ __forceinline__ void update_item(const UpdateCell& U, const T* p0, const T* p1,
                                            const T* p2, int x0, int y0, int sx, int sy,
                                            bool live, int wz, float wallv, bool top_plane,
                                            T* orow, UpdateCounts& c, uint32_t sr = 0u,
                                            uint32_t pix0 = 0u) {
    const int B = U.B;
    const pfb_layout3d& L = U.L;
    if (!live) {
        const float z[4] = {0.f, 0.f, 0.f, 0.f};
        const uint16_t zb[4] = {0, 0, 0, 0};
#pragma unroll
        for (int r = 0; r < 4; ++r) phi_st4(orow + r * B, z, zb);
        return;
    }
    const T* pl[3] = {p0, p1, p2};
    const int xs0 = x0 + sx;
    const bool vec_ok = (xs0 & 3) == 0 && xs0 >= 0 && xs0 + 4 <= B;
    float w[3][3][6];
#pragma unroll
    for (int p = 0; p < 3; ++p) {
        row6v(pl[p], B, y0 + sy - 1, xs0, vec_ok, w[p][0]);
        row6v(pl[p], B, y0 + sy, xs0, vec_ok, w[p][1]);
    }
    // world x of the four source columns (wrapped), or -1 outside
    int wxj[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int xs = xs0 + j;
        wxj[j] = (unsigned)xs < (unsigned)B ? wrap_offset(U.ox, xs, L.nx) : -1;
    }
    uint32_t agg_next[4];
    auto load_agg = [&](int ys, uint32_t* out) {
        const bool yin = (unsigned)ys < (unsigned)B;
        const size_t srow = yin ? s_index(L, 0, wrap_offset(U.oy, ys, L.ny), wz) : 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) out[j] = (yin && wxj[j] >= 0) ? __ldg(U.S_in + srow + wxj[j]) : 0u;
    };
    load_agg(y0 + sy, agg_next);
    const bool has_out = U.S_out != nullptr;
    uint32_t old_prev[4] = {0u, 0u, 0u, 0u}, q_prev[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int ys = y0 + r + sy;
#pragma unroll
        for (int p = 0; p < 3; ++p) row6v(pl[p], B, ys + 1, xs0, vec_ok, w[p][(r + 2) % 3]);
        uint32_t agg[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) agg[j] = agg_next[j];
        if (r < 3) load_agg(ys + 1, agg_next);
        const bool yin = (unsigned)ys < (unsigned)B;
        const size_t srow = yin ? s_index(L, 0, wrap_offset(U.oy, ys, L.ny), wz) : 0;
#pragma unroll
        for (int j = 0; j < 4; ++j) c.ovf += old_prev[j] > 0xFFFFFFFFu - q_prev[j] ? 1u : 0u;
        // rows r-1, r, r+1 of the window sit in slots (r+0..2) % 3
        const int s0 = r % 3, s1 = (r + 1) % 3, s2 = (r + 2) % 3;
        // the four stencils are independent chains: computed without
        // branches so the scheduler can interleave them
        float lap[4], gx[4], gy[4], gz[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) stencil27r(w, s0, s1, s2, j, lap[j], gx[j], gy[j], gz[j]);
        float out[4];
        uint16_t ob[4] = {0, 0, 0, 0};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const bool present = yin && wxj[j] >= 0;
            const float cv = w[1][s1][j + 1];
            const bool cfin = isfinite(cv);
            const uint32_t own = q_of3(cv);
            const bool neg = agg[j] < own;
            float other = neg ? 0.0f : (float)(agg[j] - own) * kQInv;
            if (GEO == 2) other += wallv;
            const float exact = cv + U.k.dt * rhs3(U.k, cv, lap[j], gx[j], gy[j], gz[j], other);
            const bool nfin = isfinite(exact);
            // the stored value (binary32: exact)
            const float next = phi_round<T>(exact, sr, pix0 + (uint32_t)(r * B + j), &ob[j]);
            const bool top = GEO == 1 && top_plane && fabsf(next) > kSupportEps3;
            c.nf += (present && (!cfin || !nfin)) ? 1u : 0u;
            c.neg += (present && cfin && neg) ? 1u : 0u;
            c.top += (present && cfin && nfin && top) ? 1u : 0u;
            const bool keep = present && cfin && nfin && !top;
            out[j] = keep ? next : 0.0f;
            if (!keep) ob[j] = 0;
            q_prev[j] = 0u;
            old_prev[j] = 0u;
            if (has_out) {
                c.clamp += (keep && next * next > kQClamp3) ? 1u : 0u;
                const uint32_t qv = keep ? q_of3(next) : 0u;
                q_prev[j] = qv;
                old_prev[j] = dev::atom_add_nonzero(U.S_out + srow + (keep ? wxj[j] : 0), qv);
            }
        }
        phi_st4(orow + r * B, out, ob);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) c.ovf += old_prev[j] > 0xFFFFFFFFu - q_prev[j] ? 1u : 0u;
}

// Fatal step: destination planes [d0, d1) keep the accepted field, which is
// scattered again (reference kernels.cu:505-559). Every thread of the CTA.
template <typename T = float>
__device__ __forceinline__ void keep_planes(const UpdateCell& U, const T* src, T* dst, int d0, int d1,
                                            int64_t oz, pfb_cell3d* cell, uint32_t* gflags,
                                            int nthreads) {
    const int B = U.B;
    const pfb_layout3d& L = U.L;
    for (size_t q = (size_t)d0 * B * B + threadIdx.x; q < (size_t)d1 * B * B; q += nthreads) {
        dst[q] = src[q];
        const float v = phi_ld1(src + q);
        if (U.S_out && isfinite(v)) {
            const int x = (int)(q % B), y = (int)((q / B) % B), z = (int)(q / ((size_t)B * B));
            int wz;
            if (!aggregate_z(L, oz, z, &wz)) continue;
            const size_t si = s_index(L, wrap_offset(U.ox, x, L.nx), wrap_offset(U.oy, y, L.ny), wz);
            if (v * v > kQClamp3) raise3(cell, gflags, PFB3D_FLAG_Q_CLAMP, 1u);
            const uint32_t qv = q_of3(v);
            if (qv) {
                const uint32_t old = atomicAdd(U.S_out + si, qv);
                if (old > 0xFFFFFFFFu - qv) raise3(cell, gflags, PFB3D_FLAG_S_OVERFLOW, 1u);
            }
        }
    }
}

// Source voxels of planes [d0, d1) whose destination falls outside the brick
// after the shift: nothing is written, but a supported new value is a
// DESTINATION_CLIP (read from global memory; shifts are rare). Adds to the
// non-finite, negative and top counts as the update would.
template <int GEO, typename T = float>
__device__ __forceinline__ unsigned clip_check(const UpdateCell& U, const T* src, const float* wall,
                                               int d0, int d1, int sx, int sy, int sz, int64_t oz,
                                               UpdateCounts& c, int nthreads) {
    const int B = U.B;
    const pfb_layout3d& L = U.L;
    unsigned clip = 0u;
    auto f = [&](int x, int y, int z) -> float {
        if ((unsigned)x >= (unsigned)B || (unsigned)y >= (unsigned)B) return 0.0f;
        int s;
        if (!fetch_plane(L, oz, z, B, &s)) return 0.0f;
        return phi_ld1(src + ((size_t)s * B + y) * B + x);
    };
    const size_t plane = (size_t)B * B;
    for (size_t q = (size_t)d0 * plane + threadIdx.x; q < (size_t)d1 * plane; q += nthreads) {
        const int x = (int)(q % B), y = (int)((q / B) % B), z = (int)(q / plane);
        if ((unsigned)(x - sx) < (unsigned)B && (unsigned)(y - sy) < (unsigned)B &&
            (unsigned)(z - sz) < (unsigned)B)
            continue;
        int wz;
        if (!aggregate_z(L, oz, z, &wz)) continue;
        const float cv = phi_ld1(src + q);
        if (!isfinite(cv)) {
            ++c.nf;
            continue;
        }
        float wv[3][3][6];
#pragma unroll
        for (int p = 0; p < 3; ++p)
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int cc = 0; cc < 3; ++cc) wv[p][r][cc] = f(x + cc - 1, y + r - 1, z + p - 1);
        float lap, gx, gy, gz;
        stencil27w(wv, 0, lap, gx, gy, gz);
        if (cv == 0.0f && lap == 0.0f && gx == 0.0f && gy == 0.0f && gz == 0.0f) continue;
        const size_t si = s_index(L, wrap_offset(U.ox, x, L.nx), wrap_offset(U.oy, y, L.ny), wz);
        const uint32_t agg = U.S_in[si];
        const uint32_t own = q_of3(cv);
        float other;
        if (agg >= own) {
            other = (float)(agg - own) * kQInv;
        } else {
            other = 0.0f;
            ++c.neg;
        }
        if (GEO == 2) other += wall[wz];
        const float next = cv + U.k.dt * rhs3(U.k, cv, lap, gx, gy, gz, other);
        if (!isfinite(next)) {
            ++c.nf;
            continue;
        }
        if (GEO == 1 && wz == L.nz - 1 && fabsf(next) > kSupportEps3) {
            ++c.top;
            continue;
        }
        if (fabsf(next) > kSupportEps3) ++clip;
    }
    return clip;
}

// flag slots of the per-CTA counters
enum { kCntNonfinite = 0, kCntNegative, kCntTop, kCntClamp, kCntOverflow, kCntClip };

// Per-CTA flag counts: warp sums, then thread 0 raises one count per flag.
template <int NT>
__device__ __forceinline__ void raise_update_counts(unsigned (&cnt)[NT / 32][6], const UpdateCounts& c,
                                                    unsigned clip, pfb_cell3d* cell, uint32_t* gflags) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    unsigned cs[6] = {c.nf, c.neg, c.top, c.clamp, c.ovf, clip};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const unsigned v = __reduce_add_sync(0xFFFFFFFFu, cs[f]);
        if (lane == 0) cnt[warp][f] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t[6] = {0, 0, 0, 0, 0, 0};
        for (int w = 0; w < NT / 32; ++w)
            for (int f = 0; f < 6; ++f) t[f] += cnt[w][f];
        raise3(cell, gflags, PFB3D_FLAG_NONFINITE, t[kCntNonfinite]);
        raise3(cell, gflags, PFB3D_FLAG_S_NEGATIVE, t[kCntNegative]);
        raise3(cell, gflags, PFB3D_FLAG_SLAB_TOP_CONTACT, t[kCntTop]);
        raise3(cell, gflags, PFB3D_FLAG_Q_CLAMP, t[kCntClamp]);
        raise3(cell, gflags, PFB3D_FLAG_S_OVERFLOW, t[kCntOverflow]);
        raise3(cell, gflags, PFB3D_FLAG_DESTINATION_CLIP, t[kCntClip]);
    }
}

}  // namespace p3
}  // namespace pfb
