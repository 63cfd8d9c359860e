// 3D moment-free update (sm_100a): explicit Euler step of every selected
// cell with its planned recentring shift and the Q5.27 scatter of the new
// field. One entry point for periodic, substrate-slab and hard-wall channel
// geometry; phi and S are bit-identical to the reference's
// k_update_periodic_slab_walk_fast (src/pf3d/kernels_periodic_slab_walk.cu:
// 54-318) and k_update_tiled_fast (src/pf3d/kernels.cu:498-793) on the same
// inputs, and every sticky flag is raised as often as there.
//
// Layout of the work: K CTAs per cell, CTA r owns destination planes
// [r B/K, (r+1) B/K). Destination plane dz reads source plane dz + sz and
// its two neighbours from a ring of whole brick planes staged by bulk
// copies (one 16 KB copy per plane at B = 64). A thread owns a strip of 4
// voxels x 4 rows and walks the rows with a three-row register window per
// source plane; the aggregate S_in is read from L2 one row ahead; phi_out is
// written with 16-byte streaming stores (every destination voxel once, so the
// output needs no clearing pass) and S_out receives one predicated atomic per
// non-zero voxel.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "pfb3d_common.cuh"
#include "pfb_internal.h"
#include "ring3d.cuh"

namespace pfb {
namespace p3 {

constexpr int kUThreads = 256;
constexpr int kURing = 5;
constexpr int kUCtasPerCell = 4;

__device__ unsigned int g_update3d_status = 0u;

struct UpdateHeader {
    uint64_t bars[kURing];
    int abort;
    int pad[3];
    unsigned cnt[kUThreads / 32][6];
};
constexpr int kUHeader = (int)((sizeof(UpdateHeader) + 127) / 128 * 128);

// flag slots of the per-CTA counters
enum { kCntNonfinite = 0, kCntNegative, kCntTop, kCntClamp, kCntOverflow, kCntClip };

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

// Six source values of one row: columns xs0 - 1 .. xs0 + 4 (zero outside
// the brick or when the row is outside it).
__device__ __forceinline__ void row6(const float* plane, int B, int ys, int xs0, float* v) {
    if ((unsigned)ys >= (unsigned)B) {
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = 0.0f;
        return;
    }
    const float* row = plane + ys * B;
    if ((xs0 & 3) == 0 && xs0 >= 0 && xs0 + 4 <= B) {
        const float4 m = *reinterpret_cast<const float4*>(row + xs0);
        v[0] = xs0 > 0 ? row[xs0 - 1] : 0.0f;
        v[1] = m.x;
        v[2] = m.y;
        v[3] = m.z;
        v[4] = m.w;
        v[5] = xs0 + 4 < B ? row[xs0 + 4] : 0.0f;
    } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const int x = xs0 - 1 + c;
            v[c] = (unsigned)x < (unsigned)B ? row[x] : 0.0f;
        }
    }
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

// row6 with the alignment decision taken once per strip
__device__ __forceinline__ void row6v(const float* plane, int B, int ys, int xs0, bool vec_ok,
                                      float* v) {
    if ((unsigned)ys >= (unsigned)B) {
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = 0.0f;
        return;
    }
    const float* row = plane + ys * B;
    if (vec_ok) {
        const float4 m = *reinterpret_cast<const float4*>(row + xs0);
        v[0] = xs0 > 0 ? row[xs0 - 1] : 0.0f;
        v[1] = m.x;
        v[2] = m.y;
        v[3] = m.z;
        v[4] = m.w;
        v[5] = xs0 + 4 < B ? row[xs0 + 4] : 0.0f;
    } else {
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            const int x = xs0 - 1 + c;
            v[c] = (unsigned)x < (unsigned)B ? row[x] : 0.0f;
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

// GEO: 0 periodic, 1 substrate slab, 2 hard-wall channel
template <int GEO>
__global__ void __launch_bounds__(kUThreads, 2) k_update3d(const __grid_constant__ pfb_update_args3d A) {
    extern __shared__ __align__(128) char smem[];
    UpdateHeader& H = *reinterpret_cast<UpdateHeader*>(smem);
    const int B = A.B;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int slot_cell = (int)(blockIdx.x / kUCtasPerCell);
    const int part = (int)(blockIdx.x % kUCtasPerCell);
    const int n = A.selection.ids ? A.selection.ids[slot_cell] : slot_cell;
    pfb_cell3d* cell = &A.cells[n];
    if (cell->storage_edge != 0u) return;
    const pfb_layout3d L = A.layout;
    const size_t words = (size_t)B * B * B;
    const float* src = A.phi_in + (size_t)n * words;
    float* dst = A.phi_out + (size_t)n * words;
    const int PB = B / kUCtasPerCell;
    const int d0 = part * PB, d1 = d0 + PB;
    const int ox = wrap_origin(cell->origin_x, L.nx);
    const int oy = wrap_origin(cell->origin_y, L.ny);
    const int64_t oz = cell->origin_z;

    if (tid == 0) H.abort = fatal3(cell, A.global_flags) ? 1 : 0;
    if (tid < (kUThreads / 32) * 6) (&H.cnt[0][0])[tid] = 0u;
    __syncthreads();
    if (H.abort) {
        // keep the last accepted field (reference kernels.cu:505-559)
        for (size_t q = (size_t)d0 * B * B + tid; q < (size_t)d1 * B * B; q += kUThreads) {
            const float v = src[q];
            dst[q] = v;
            if (A.S_out && isfinite(v)) {
                const int x = (int)(q % B), y = (int)((q / B) % B), z = (int)(q / ((size_t)B * B));
                int wz;
                if (!aggregate_z(L, oz, z, &wz)) continue;
                const size_t si = s_index(L, wrap_offset(ox, x, L.nx), wrap_offset(oy, y, L.ny), wz);
                if (v * v > kQClamp3) raise3(cell, A.global_flags, PFB3D_FLAG_Q_CLAMP, 1u);
                const uint32_t qv = q_of3(v);
                if (qv) {
                    const uint32_t old = atomicAdd(A.S_out + si, qv);
                    if (old > 0xFFFFFFFFu - qv) raise3(cell, A.global_flags, PFB3D_FLAG_S_OVERFLOW, 1u);
                }
            }
        }
        __syncthreads();
        if (tid == 0 && part == 0) {
            cell->pending_shift_x = 0;
            cell->pending_shift_y = 0;
            cell->pending_shift_z = 0;
        }
        return;
    }

    const int sx = cell->pending_shift_x, sy = cell->pending_shift_y, sz = cell->pending_shift_z;
    CellCoef k;
    k.gamma = cell->gamma;
    k.vx = cell->velocity_x;
    k.vy = cell->velocity_y;
    k.vz = cell->velocity_z;
    k.bulk = A.bulk_scale * k.gamma;
    k.volume = (float)(A.volume_scale * (A.V0 - cell->V));
    k.inter = A.interaction_coeff;
    k.dt = A.dt;

    PlaneRing<kURing> ring{reinterpret_cast<float*>(smem + kUHeader), H.bars, B * B};
    ring.init();
    __syncthreads();
    // request k <-> requested source plane d0 + sz - 1 + k, k = 0 .. PB + 1
    auto issue = [&](int kq) {
        int s;
        if (!fetch_plane(L, oz, d0 + sz - 1 + kq, B, &s)) s = -1;
        ring.issue(kq, src, s);
    };
    const int nreq = PB + 2;
    int issued = 0;
    for (int kq = 0; kq < kURing && kq < nreq; ++kq, ++issued) issue(kq);
    __syncthreads();
    // the first two planes are read from iteration 0 on; later ones are
    // waited for one iteration before their first read
    if (!ring.wait(0) || !ring.wait(1)) {
        H.abort = 1;
        atomicOr(&g_update3d_status, 1u);
    }

    unsigned cnt_nf = 0, cnt_neg = 0, cnt_top = 0, cnt_clamp = 0, cnt_ovf = 0;
    const int strips = B / 4;
    const int items = strips * (B / 4);
    const bool has_out = A.S_out != nullptr;
    const float* wall = GEO == 2 ? A.wall.values : nullptr;

    for (int i = 0; i < PB; ++i) {
        const int dz = d0 + i;
        const int zs = dz + sz;  // source plane
        if (!ring.wait(i + 2)) {
            H.abort = 1;
            atomicOr(&g_update3d_status, 1u);
        }
        int wz = 0;
        const bool zin = (unsigned)zs < (unsigned)B;
        const bool live = zin && aggregate_z(L, oz, zs, &wz);
        const float* pl[3] = {ring.slot(i), ring.slot(i + 1), ring.slot(i + 2)};
        const float wallv = GEO == 2 && live ? wall[wz] : 0.0f;
        const bool top_plane = GEO == 1 && live && wz == L.nz - 1;
        for (int it = tid; it < items; it += kUThreads) {
            const int x0 = 4 * (it % strips);
            const int y0 = 4 * (it / strips);
            float* orow = dst + ((size_t)dz * B + y0) * B + x0;
            if (!live || H.abort) {
                const float4 z4 = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
                for (int r = 0; r < 4; ++r) __stcs(reinterpret_cast<float4*>(orow + r * B), z4);
                continue;
            }
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
                wxj[j] = (unsigned)xs < (unsigned)B ? wrap_offset(ox, xs, L.nx) : -1;
            }
            uint32_t agg_next[4];
            auto load_agg = [&](int ys, uint32_t* out) {
                const bool yin = (unsigned)ys < (unsigned)B;
                const size_t srow = yin ? s_index(L, 0, wrap_offset(oy, ys, L.ny), wz) : 0;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    out[j] = (yin && wxj[j] >= 0) ? __ldg(A.S_in + srow + wxj[j]) : 0u;
            };
            load_agg(y0 + sy, agg_next);
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
                const size_t srow = yin ? s_index(L, 0, wrap_offset(oy, ys, L.ny), wz) : 0;
#pragma unroll
                for (int j = 0; j < 4; ++j) cnt_ovf += old_prev[j] > 0xFFFFFFFFu - q_prev[j] ? 1u : 0u;
                // rows r-1, r, r+1 of the window sit in slots (r+0..2) % 3
                const int s0 = r % 3, s1 = (r + 1) % 3, s2 = (r + 2) % 3;
                // the four stencils are independent chains: computed without
                // branches so the scheduler can interleave them
                float lap[4], gx[4], gy[4], gz[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) stencil27r(w, s0, s1, s2, j, lap[j], gx[j], gy[j], gz[j]);
                float out[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const bool present = yin && wxj[j] >= 0;
                    const float c = w[1][s1][j + 1];
                    const bool cfin = isfinite(c);
                    const uint32_t own = q_of3(c);
                    const bool neg = agg[j] < own;
                    float other = neg ? 0.0f : (float)(agg[j] - own) * kQInv;
                    if (GEO == 2) other += wallv;
                    const float next = c + k.dt * rhs3(k, c, lap[j], gx[j], gy[j], gz[j], other);
                    const bool nfin = isfinite(next);
                    const bool top = GEO == 1 && top_plane && fabsf(next) > kSupportEps3;
                    cnt_nf += (present && (!cfin || !nfin)) ? 1u : 0u;
                    cnt_neg += (present && cfin && neg) ? 1u : 0u;
                    cnt_top += (present && cfin && nfin && top) ? 1u : 0u;
                    const bool keep = present && cfin && nfin && !top;
                    out[j] = keep ? next : 0.0f;
                    q_prev[j] = 0u;
                    old_prev[j] = 0u;
                    if (has_out) {
                        cnt_clamp += (keep && next * next > kQClamp3) ? 1u : 0u;
                        const uint32_t qv = keep ? q_of3(next) : 0u;
                        q_prev[j] = qv;
                        old_prev[j] = dev::atom_add_nonzero(A.S_out + srow + (keep ? wxj[j] : 0), qv);
                    }
                }
                __stcs(reinterpret_cast<float4*>(orow + r * B),
                       make_float4(out[0], out[1], out[2], out[3]));
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) cnt_ovf += old_prev[j] > 0xFFFFFFFFu - q_prev[j] ? 1u : 0u;
        }
        __syncthreads();
        // after a timed-out wait nothing more is issued into the ring
        if (!H.abort && i + kURing < nreq) {
            issue(i + kURing);
            ++issued;
        }
    }

    // no bulk copy may still target this CTA's shared memory at exit
    if (H.abort)
        for (int kq = issued > kURing ? issued - kURing : 0; kq < issued; ++kq) ring.wait(kq);

    // ---- source voxels whose destination falls outside the brick: no write,
    // but a supported value is a DESTINATION_CLIP. Every CTA of the cell
    // checks the source planes of its own z range (from global memory;
    // shifts are rare).
    unsigned cnt_clip = 0;
    if ((sx | sy | sz) != 0 && !H.abort) {
        auto f = [&](int x, int y, int z) -> float {
            if ((unsigned)x >= (unsigned)B || (unsigned)y >= (unsigned)B) return 0.0f;
            int s;
            if (!fetch_plane(L, oz, z, B, &s)) return 0.0f;
            return src[((size_t)s * B + y) * B + x];
        };
        const size_t plane = (size_t)B * B;
        for (size_t q = (size_t)d0 * plane + tid; q < (size_t)d1 * plane; q += kUThreads) {
            const int x = (int)(q % B), y = (int)((q / B) % B), z = (int)(q / plane);
            if ((unsigned)(x - sx) < (unsigned)B && (unsigned)(y - sy) < (unsigned)B &&
                (unsigned)(z - sz) < (unsigned)B)
                continue;
            int wz;
            if (!aggregate_z(L, oz, z, &wz)) continue;
            const float c = src[q];
            if (!isfinite(c)) {
                ++cnt_nf;
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
            if (c == 0.0f && lap == 0.0f && gx == 0.0f && gy == 0.0f && gz == 0.0f) continue;
            const size_t si = s_index(L, wrap_offset(ox, x, L.nx), wrap_offset(oy, y, L.ny), wz);
            const uint32_t agg = A.S_in[si];
            const uint32_t own = q_of3(c);
            float other;
            if (agg >= own) {
                other = (float)(agg - own) * kQInv;
            } else {
                other = 0.0f;
                ++cnt_neg;
            }
            if (GEO == 2) other += wall[wz];
            const float next = c + k.dt * rhs3(k, c, lap, gx, gy, gz, other);
            if (!isfinite(next)) {
                ++cnt_nf;
                continue;
            }
            if (GEO == 1 && wz == L.nz - 1 && fabsf(next) > kSupportEps3) {
                ++cnt_top;
                continue;
            }
            if (fabsf(next) > kSupportEps3) ++cnt_clip;
        }
    }

    unsigned cs[6] = {cnt_nf, cnt_neg, cnt_top, cnt_clamp, cnt_ovf, cnt_clip};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        const unsigned v = __reduce_add_sync(0xFFFFFFFFu, cs[f]);
        if (lane == 0) H.cnt[warp][f] = v;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned t[6] = {0, 0, 0, 0, 0, 0};
        for (int w = 0; w < kUThreads / 32; ++w)
            for (int f = 0; f < 6; ++f) t[f] += H.cnt[w][f];
        raise3(cell, A.global_flags, PFB3D_FLAG_NONFINITE, t[kCntNonfinite]);
        raise3(cell, A.global_flags, PFB3D_FLAG_S_NEGATIVE, t[kCntNegative]);
        raise3(cell, A.global_flags, PFB3D_FLAG_SLAB_TOP_CONTACT, t[kCntTop]);
        raise3(cell, A.global_flags, PFB3D_FLAG_Q_CLAMP, t[kCntClamp]);
        raise3(cell, A.global_flags, PFB3D_FLAG_S_OVERFLOW, t[kCntOverflow]);
        raise3(cell, A.global_flags, PFB3D_FLAG_DESTINATION_CLIP, t[kCntClip]);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
int geometry_ok3(int B, const pfb_layout3d& L);

size_t update3d_smem(int B) { return (size_t)kUHeader + (size_t)kURing * (size_t)B * B * 4; }

int update3d_launch(const pfb_update_args3d* a, cudaStream_t stream) {
    if (!a) return set_error(PFB_E_ARG, "null update arguments");
    const pfb_update_args3d& A = *a;
    if (A.tile_pass != PFB3D_TILE_PASS_ALL)
        return set_error(PFB_E_CONFIG, "only the whole-brick tile pass is supported");
    if (A.storage.z_cap != 0) return set_error(PFB_E_CONFIG, "compact cell storage is not supported");
    if (A.compute_surface) return set_error(PFB_E_CONFIG, "the fast update measures no surface");
    if (!geometry_ok3(A.B, A.layout) || A.N <= 0)
        return set_error(PFB_E_ARG, "invalid brick edge or aggregate layout");
    if (A.selection.ids && (A.selection.count < 0 || A.selection.count > A.N))
        return set_error(PFB_E_ARG, "invalid cell selection");
    const uint32_t bf = A.layout.boundary_flags;
    const bool channel = hard_wall_channel(bf);
    if (channel ? (A.wall.values == nullptr || A.wall.planes != A.layout.nz)
                : (A.wall.values != nullptr || A.wall.planes != 0))
        return set_error(PFB_E_ARG, "wall field does not match the geometry");
    if (!A.phi_in || !A.phi_out || A.phi_in == A.phi_out || !A.S_in || !A.cells ||
        (A.S_out && A.S_out == A.S_in))
        return set_error(PFB_E_ARG, "invalid buffers in update arguments");
    if (((uintptr_t)A.phi_in & 15u) || ((uintptr_t)A.phi_out & 15u))
        return set_error(PFB_E_ARG, "phi pools must be 16-byte aligned");
    const int count = A.selection.ids ? A.selection.count : A.N;
    if (count == 0) return PFB_OK;
    const size_t smem = update3d_smem(A.B);
    if (smem > 227 * 1024) return set_error(PFB_E_CONFIG, "brick edge too large for the plane ring");
    const dim3 grid((unsigned)(count * kUCtasPerCell));
    cudaError_t e;
    if (periodic_xyz(bf)) {
        e = cudaFuncSetAttribute(k_update3d<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) k_update3d<0><<<grid, kUThreads, smem, stream>>>(A);
    } else if (substrate_slab(bf)) {
        e = cudaFuncSetAttribute(k_update3d<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) k_update3d<1><<<grid, kUThreads, smem, stream>>>(A);
    } else {
        e = cudaFuncSetAttribute(k_update3d<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) k_update3d<2><<<grid, kUThreads, smem, stream>>>(A);
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "update launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int update3d_read_status(unsigned* out, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_update3d_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status read: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_update3d_status, &z, sizeof(z));
    }
    if (out) *out = v;
    return PFB_OK;
}

}  // namespace p3
}  // namespace pfb

extern "C" int pfb3d_update(const pfb_update_args3d* args, void* stream) {
    return pfb::p3::update3d_launch(args, static_cast<cudaStream_t>(stream));
}
