// 3D measurement and motion (sm_100a).
//
// k_measure3d<K>: one thread-block cluster of K CTAs per cell; CTA r walks
// brick planes [r B/K, (r+1) B/K) through a ring of bulk-copied planes and
// accumulates V, the centroid sums, the interaction integral, the surface
// proxy, the support box and phi_max of its planes. The K partial results
// are pushed into rank 0's shared memory with st.async and summed there in
// rank order; rank 0 then plans the recentring shift and checks the support
// margin exactly as the reference's commit_measurement
// (src/pf3d/kernels.cu:418-497). Per-voxel semantics follow
// measure_one_cell (src/pf3d/kernels.cu:1271-1409).
//
// k_motion3d: tumble and velocity per cell (src/pf3d/kernels.cu:1739-1788).
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "pfb3d_common.cuh"
#include "pfb_internal.h"
#include "ring3d.cuh"

namespace pfb {
namespace p3 {

constexpr int kThreads3 = 256;
constexpr int kWarps3 = kThreads3 / 32;
constexpr int kMeasureRing = 4;
constexpr int kMeasureCluster = 4;

__device__ unsigned int g_measure3d_status = 0u;

struct Acc3 {
    double V = 0.0, Cx = 0.0, Cy = 0.0, Cz = 0.0, Sf = 0.0, Ix = 0.0, Iy = 0.0, Iz = 0.0;
    int lox, hix = -1, loy, hiy = -1, loz, hiz = -1;
    unsigned pmax = 0u;
};

template <int K>
struct MeasureHeader {
    uint64_t bars[kMeasureRing];
    uint64_t barR;
    int abort;
    int pad;
    double wd[kWarps3][8];
    int wi[kWarps3][8];
    double rd[K][8];
    int ri[K][8];
    unsigned cnt[kWarps3][4];
};

__device__ __forceinline__ void raise_counted(pfb_cell3d* cell, uint32_t* gflags, int flag,
                                              unsigned count) {
    if (!count) return;
    atomicOr(&cell->flags, 1u << flag);
    if (gflags) atomicAdd(&gflags[flag], count);
}

// Plane items: strips 4 voxels wide and 4 rows tall.
__device__ __forceinline__ void load_row6(const float* plane, int B, int y, int x0, float* v) {
    if ((unsigned)y >= (unsigned)B) {
#pragma unroll
        for (int c = 0; c < 6; ++c) v[c] = 0.0f;
        return;
    }
    const float* row = plane + y * B;
    const float4 m = *reinterpret_cast<const float4*>(row + x0);
    v[0] = x0 > 0 ? row[x0 - 1] : 0.0f;
    v[1] = m.x;
    v[2] = m.y;
    v[3] = m.z;
    v[4] = m.w;
    v[5] = x0 + 4 < B ? row[x0 + 4] : 0.0f;
}

template <int K>
__global__ void __launch_bounds__(kThreads3, 2) k_measure3d(const __grid_constant__ pfb_measure_args3d A) {
    extern __shared__ __align__(128) char smem[];
    MeasureHeader<K>& H = *reinterpret_cast<MeasureHeader<K>*>(smem);
    constexpr int kHeader = (int)((sizeof(MeasureHeader<K>) + 127) / 128 * 128);
    const int B = A.B;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rank = (int)dev::cluster_rank();
    const int slot = (int)(blockIdx.x / K);
    const int n = A.selection.ids ? A.selection.ids[slot] : slot;
    pfb_cell3d* cell = &A.cells[n];
    // Promoted cells are uniform over the cluster: every CTA returns.
    if (cell->storage_edge != 0u) return;

    PlaneRing<kMeasureRing> ring{reinterpret_cast<float*>(smem + kHeader), H.bars, B * B};
    ring.init();
    if (tid == 0) {
        dev::mbar_init(&H.barR, 1);
        if (rank == 0) dev::mbar_arrive_expect_tx(&H.barR, (uint32_t)(K * (8 * 8 + 8 * 4)));
        H.abort = 0;
    }
    __syncthreads();
    dev::cluster_arrive_relaxed();

    const pfb_layout3d L = A.layout;
    const uint32_t bf = L.boundary_flags;
    const int64_t oz = cell->origin_z;
    const int ox = wrap_origin(cell->origin_x, L.nx);
    const int oy = wrap_origin(cell->origin_y, L.ny);
    const float* field = A.phi + (size_t)n * (size_t)B * B * B;
    const int PB = B / K;
    const int z0 = rank * PB;
    const bool wall = hard_wall_channel(bf) && A.wall.values;

    // request k <-> plane z0 - 1 + k (k = 0 .. PB + 1)
    auto issue = [&](int k) {
        int src;
        if (!fetch_plane(L, oz, z0 - 1 + k, B, &src)) src = -1;
        ring.issue(k, field, src);
    };
    const int nreq = PB + 2;
    int issued = 0;
    for (int k = 0; k < kMeasureRing && k < nreq; ++k, ++issued) issue(k);
    __syncthreads();
    // the first two planes are read from iteration 0 on; later ones are
    // waited for one iteration before their first read
    if (!ring.wait(0) || !ring.wait(1)) {
        H.abort = 1;
        atomicOr(&g_measure3d_status, 1u);
    }

    Acc3 acc;
    acc.lox = acc.loy = acc.loz = B;
    unsigned c_nonfinite = 0u, c_negative = 0u, c_top = 0u;
    const int strips = B / 4;
    const int items = strips * (B / 4);

    for (int i = 0; i < PB; ++i) {
        const int z = z0 + i;
        if (!ring.wait(i + 2)) {
            H.abort = 1;
            atomicOr(&g_measure3d_status, 1u);
        }
        int wz = 0;
        const bool live = aggregate_z(L, oz, z, &wz);
        if (live && !H.abort) {
            const float* pm = ring.slot(i);
            const float* pc = ring.slot(i + 1);
            const float* pp = ring.slot(i + 2);
            const float wallv = wall ? A.wall.values[wz] : 0.0f;
            const bool top_plane = substrate_slab(bf) && wz == L.nz - 1;
            for (int it = tid; it < items; it += kThreads3) {
                const int x0 = 4 * (it % strips);
                const int y0 = 4 * (it / strips);
                float rs[6], rc[6], rn[6];
                load_row6(pc, B, y0 - 1, x0, rs);
                load_row6(pc, B, y0, x0, rc);
                int wxj[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) wxj[j] = wrap_offset(ox, x0 + j, L.nx);
                // aggregate words of a row, fetched one row ahead
                auto load_agg = [&](int y, uint32_t* out) {
                    const size_t srow = s_index(L, 0, wrap_offset(oy, y, L.ny), wz);
#pragma unroll
                    for (int j = 0; j < 4; ++j) out[j] = __ldg(A.S + srow + wxj[j]);
                };
                uint32_t agg_next[4];
                load_agg(y0, agg_next);
#pragma unroll 1
                for (int r = 0; r < 4; ++r) {
                    const int y = y0 + r;
                    load_row6(pc, B, y + 1, x0, rn);
                    const float4 zm = *reinterpret_cast<const float4*>(pm + y * B + x0);
                    const float4 zp = *reinterpret_cast<const float4*>(pp + y * B + x0);
                    const float zmv[4] = {zm.x, zm.y, zm.z, zm.w};
                    const float zpv[4] = {zp.x, zp.y, zp.z, zp.w};
                    uint32_t agg[4];
#pragma unroll
                    for (int j = 0; j < 4; ++j) agg[j] = agg_next[j];
                    if (r < 3) load_agg(y + 1, agg_next);
                    double rV = 0.0, rX = 0.0;
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float c = rc[j + 1];
                        const bool cfin = isfinite(c);
                        c_nonfinite += cfin ? 0u : 1u;
                        const float gx = 0.5f * (rc[j + 2] - rc[j]);
                        const float gy = 0.5f * (rn[j + 1] - rs[j + 1]);
                        const float gz = 0.5f * (zpv[j] - zmv[j]);
                        const uint32_t own = q_of3(c);
                        const bool nz = cfin && c != 0.0f;
                        const bool neg = nz && agg[j] < own;
                        c_negative += neg ? 1u : 0u;
                        float other = (nz && !neg) ? (float)(agg[j] - own) * kQInv : 0.0f;
                        if (wall) other += wallv;
                        const double sq = cfin ? (double)c * (double)c : 0.0;
                        rV += sq;
                        rX += sq * (double)j;
                        if (A.compute_surface && cfin)
                            acc.Sf += sqrt((double)gx * gx + (double)gy * gy + (double)gz * gz);
                        acc.Ix += cfin ? (double)(c * gx * other) : 0.0;
                        acc.Iy += cfin ? (double)(c * gy * other) : 0.0;
                        acc.Iz += cfin ? (double)(c * gz * other) : 0.0;
                        if (cfin) acc.pmax = max(acc.pmax, __float_as_uint(fabsf(c)));
                        const int x = x0 + j;
                        if (cfin && fabsf(c) > kSupportEps3) {
                            if (top_plane) ++c_top;
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
        }
        __syncthreads();
        // after a timed-out wait nothing more is issued into the ring
        if (!H.abort && i + kMeasureRing < nreq) {
            issue(i + kMeasureRing);
            ++issued;
        }
    }

    // no bulk copy may still target this CTA's shared memory at exit
    if (H.abort)
        for (int k = issued > kMeasureRing ? issued - kMeasureRing : 0; k < issued; ++k)
            ring.wait(k);

    // ---- flags: one counted raise per CTA and flag
    c_nonfinite = __reduce_add_sync(0xFFFFFFFFu, c_nonfinite);
    c_negative = __reduce_add_sync(0xFFFFFFFFu, c_negative);
    c_top = __reduce_add_sync(0xFFFFFFFFu, c_top);
    if (lane == 0) {
        H.cnt[warp][0] = c_nonfinite;
        H.cnt[warp][1] = c_negative;
        H.cnt[warp][2] = c_top;
    }

    // ---- CTA reduction: warp butterfly, then warps in order
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
        double* d = H.wd[warp];
        d[0] = acc.V; d[1] = acc.Cx; d[2] = acc.Cy; d[3] = acc.Cz;
        d[4] = acc.Sf; d[5] = acc.Ix; d[6] = acc.Iy; d[7] = acc.Iz;
        int* q = H.wi[warp];
        q[0] = b0; q[1] = b1; q[2] = b2; q[3] = b3; q[4] = b4; q[5] = b5; q[6] = (int)pm; q[7] = 0;
    }
    __syncthreads();
    dev::cluster_wait();  // rank 0's receive barrier is initialised
    if (warp == 0) {
        double s[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) s[k] = dev::ordered_lane_sum(lane < kWarps3 ? H.wd[lane][k] : 0.0, kWarps3);
        int v[8];
        v[0] = __reduce_min_sync(0xFFFFFFFFu, lane < kWarps3 ? H.wi[lane][0] : B);
        v[1] = __reduce_max_sync(0xFFFFFFFFu, lane < kWarps3 ? H.wi[lane][1] : -1);
        v[2] = __reduce_min_sync(0xFFFFFFFFu, lane < kWarps3 ? H.wi[lane][2] : B);
        v[3] = __reduce_max_sync(0xFFFFFFFFu, lane < kWarps3 ? H.wi[lane][3] : -1);
        v[4] = __reduce_min_sync(0xFFFFFFFFu, lane < kWarps3 ? H.wi[lane][4] : B);
        v[5] = __reduce_max_sync(0xFFFFFFFFu, lane < kWarps3 ? H.wi[lane][5] : -1);
        v[6] = (int)__reduce_max_sync(0xFFFFFFFFu, lane < kWarps3 ? (unsigned)H.wi[lane][6] : 0u);
        v[7] = 0;
        unsigned cn[3];
#pragma unroll
        for (int f = 0; f < 3; ++f)
            cn[f] = __reduce_add_sync(0xFFFFFFFFu, lane < kWarps3 ? H.cnt[lane][f] : 0u);
        if (lane == 0) {
            raise_counted(cell, A.global_flags, PFB3D_FLAG_NONFINITE, cn[0]);
            raise_counted(cell, A.global_flags, PFB3D_FLAG_S_NEGATIVE, cn[1]);
            raise_counted(cell, A.global_flags, PFB3D_FLAG_SLAB_TOP_CONTACT, cn[2]);
            const uint32_t bar = dev::map_to_rank(dev::smem_addr(&H.barR), 0);
#pragma unroll
            for (int k = 0; k < 8; k += 2)
                dev::st_async_v2f64(dev::map_to_rank(dev::smem_addr(&H.rd[rank][k]), 0), s[k],
                                    s[k + 1], bar);
            dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&H.ri[rank][0]), 0), v[0], v[1],
                                v[2], v[3], bar);
            dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&H.ri[rank][4]), 0), v[4], v[5],
                                v[6], v[7], bar);
        }
        if (rank == 0) {
            if (!dev::mbar_wait_bounded(&H.barR, 0, kPlaneWaitPolls))
                atomicOr(&g_measure3d_status, 2u);
            double t[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) t[k] = dev::ordered_lane_sum(lane < K ? H.rd[lane][k] : 0.0, K);
            const int lo_x = __reduce_min_sync(0xFFFFFFFFu, lane < K ? H.ri[lane][0] : B);
            const int hi_x = __reduce_max_sync(0xFFFFFFFFu, lane < K ? H.ri[lane][1] : -1);
            const int lo_y = __reduce_min_sync(0xFFFFFFFFu, lane < K ? H.ri[lane][2] : B);
            const int hi_y = __reduce_max_sync(0xFFFFFFFFu, lane < K ? H.ri[lane][3] : -1);
            const int lo_z = __reduce_min_sync(0xFFFFFFFFu, lane < K ? H.ri[lane][4] : B);
            const int hi_z = __reduce_max_sync(0xFFFFFFFFu, lane < K ? H.ri[lane][5] : -1);
            const unsigned pmb =
                __reduce_max_sync(0xFFFFFFFFu, lane < K ? (unsigned)H.ri[lane][6] : 0u);
            if (lane == 0) {
                // commit (reference src/pf3d/kernels.cu:418-497)
                cell->V = t[0];
                cell->Cx = t[1];
                cell->Cy = t[2];
                cell->Cz = t[3];
                if (A.compute_surface) cell->surface = t[4];
                cell->Ix = t[5];
                cell->Iy = t[6];
                cell->Iz = t[7];
                cell->bb_lo_x = lo_x; cell->bb_hi_x = hi_x;
                cell->bb_lo_y = lo_y; cell->bb_hi_y = hi_y;
                cell->bb_lo_z = lo_z; cell->bb_hi_z = hi_z;
                cell->phi_max = __uint_as_float(pmb);
                int sx = 0, sy = 0, sz = 0;
                if (t[0] > 0.0 && isfinite(t[0])) {
                    const double mid = 0.5 * (double)(B - 1);
                    sx = clamp_shift(__double2int_rn(t[1] / t[0] - mid), A.max_shift, lo_x, hi_x, B);
                    sy = clamp_shift(__double2int_rn(t[2] / t[0] - mid), A.max_shift, lo_y, hi_y, B);
                    sz = clamp_shift(__double2int_rn(t[3] / t[0] - mid), A.max_shift, lo_z, hi_z, B);
                } else {
                    raise_counted(cell, A.global_flags, PFB3D_FLAG_V_NONPOSITIVE, 1u);
                }
                cell->pending_shift_x = sx;
                cell->pending_shift_y = sy;
                cell->pending_shift_z = sz;
                if (hi_x >= lo_x) {
                    const int ex = hi_x - lo_x + 1, ey = hi_y - lo_y + 1, ez = hi_z - lo_z + 1;
                    const int m = A.support_margin, ml = m / 2, mu = m - ml;
                    if (ex + m > B || ey + m > B || ez + m > B || lo_x - sx < ml ||
                        hi_x - sx >= B - mu || lo_y - sy < ml || hi_y - sy >= B - mu ||
                        lo_z - sz < ml || hi_z - sz >= B - mu)
                        raise_counted(cell, A.global_flags, PFB3D_FLAG_SUPPORT_EXHAUSTED, 1u);
                }
            }
        }
    }
}

__global__ void k_motion3d(const __grid_constant__ pfb_measure_args3d A) {
    const int slot = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    const int count = A.selection.ids ? A.selection.count : A.N;
    if (slot >= count) return;
    const int n = A.selection.ids ? A.selection.ids[slot] : slot;
    pfb_cell3d* c = &A.cells[n];
    // any fatal bit of the cell or any fatal global counter stops motion
    bool fatal = (c->flags & PFB3D_FATAL_MASK) != 0u;
    if (A.global_flags)
        for (int f = 0; f < PFB3D_FLAG_COUNT; ++f)
            if (((PFB3D_FATAL_MASK >> f) & 1u) && A.global_flags[f]) fatal = true;
    if (fatal) return;
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
    const float vx = speed * fx + A.motility_coeff * (float)c->Ix;
    const float vy = speed * fy + A.motility_coeff * (float)c->Iy;
    const float vz = slab ? 0.0f : speed * fz + A.motility_coeff * (float)c->Iz;
    if (!isfinite(fx) || !isfinite(fy) || !isfinite(fz) || !isfinite(vx) || !isfinite(vy) ||
        !isfinite(vz)) {
        atomicOr(&c->flags, 1u << PFB3D_FLAG_NONFINITE);
        if (A.global_flags) atomicAdd(&A.global_flags[PFB3D_FLAG_NONFINITE], 1u);
        return;
    }
    c->polarity_x = fx;
    c->polarity_y = fy;
    c->polarity_z = fz;
    c->velocity_x = vx;
    c->velocity_y = vy;
    c->velocity_z = vz;
    if (tumbled) ++c->tumble_ctr;
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static size_t measure_smem(int B) {
    const size_t header = (sizeof(MeasureHeader<kMeasureCluster>) + 127) / 128 * 128;
    return header + (size_t)kMeasureRing * (size_t)B * B * 4;
}

int geometry_ok3(int B, const pfb_layout3d& L) {
    const uint32_t b = L.boundary_flags;
    if (!(periodic_xyz(b) || substrate_slab(b) || hard_wall_channel(b))) return 0;
    return B > 0 && B % kBrickAlign == 0 && L.nx > B && L.ny > B &&
           (hard_wall_channel(b) ? L.nz > 0 : L.nz > B) && L.pitch_x >= L.nx &&
           L.pitch_x % 4 == 0;
}

static int check_measure(const pfb_measure_args3d* a) {
    if (!a) return set_error(PFB_E_ARG, "null measure arguments");
    const pfb_measure_args3d& A = *a;
    if (A.storage.z_cap != 0) return set_error(PFB_E_CONFIG, "compact cell storage is not supported");
    if (!geometry_ok3(A.B, A.layout) || A.N <= 0)
        return set_error(PFB_E_ARG, "invalid brick edge or aggregate layout");
    if (A.selection.ids && (A.selection.count < 0 || A.selection.count > A.N))
        return set_error(PFB_E_ARG, "invalid cell selection");
    const bool channel = hard_wall_channel(A.layout.boundary_flags);
    if (channel ? (A.wall.values == nullptr || A.wall.planes != A.layout.nz)
                : (A.wall.values != nullptr || A.wall.planes != 0))
        return set_error(PFB_E_ARG, "wall field does not match the geometry");
    if (!A.phi || !A.S || !A.cells) return set_error(PFB_E_ARG, "null buffer in measure arguments");
    if ((A.apply_tumble || A.aging_steps != 0u) && !A.step)
        return set_error(PFB_E_ARG, "tumble or aging needs the device step counter");
    if (((uintptr_t)A.phi & 15u)) return set_error(PFB_E_ARG, "phi must be 16-byte aligned");
    return PFB_OK;
}

int measure3d_launch(const pfb_measure_args3d* a, cudaStream_t stream) {
    int rc = check_measure(a);
    if (rc) return rc;
    const pfb_measure_args3d& A = *a;
    const int count = A.selection.ids ? A.selection.count : A.N;
    if (count == 0) return PFB_OK;
    constexpr int K = kMeasureCluster;
    const size_t smem = measure_smem(A.B);
    if (smem > 227 * 1024) return set_error(PFB_E_CONFIG, "brick edge too large for the plane ring");
    cudaError_t e = cudaFuncSetAttribute(k_measure3d<K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "measure attribute: %s", cudaGetErrorString(e));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(count * K), 1, 1);
    cfg.blockDim = dim3(kThreads3, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_measure3d<K>, A);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "measure launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int motion3d_launch(const pfb_measure_args3d* a, cudaStream_t stream) {
    if (!a) return set_error(PFB_E_ARG, "null measure arguments");
    const pfb_measure_args3d& A = *a;
    if (A.N <= 0 || !A.cells || !A.global_flags)
        return set_error(PFB_E_ARG, "motion needs cells and global flags");
    if (A.selection.ids && (A.selection.count < 0 || A.selection.count > A.N))
        return set_error(PFB_E_ARG, "invalid cell selection");
    if ((A.apply_tumble || A.aging_steps != 0u) && !A.step)
        return set_error(PFB_E_ARG, "tumble or aging needs the device step counter");
    const int count = A.selection.ids ? A.selection.count : A.N;
    if (count == 0) return PFB_OK;
    k_motion3d<<<(count + 127) / 128, 128, 0, stream>>>(*a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "motion launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int measure3d_read_status(unsigned* out, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_measure3d_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status read: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_measure3d_status, &z, sizeof(z));
    }
    if (out) *out = v;
    return PFB_OK;
}

}  // namespace p3
}  // namespace pfb

extern "C" {

int pfb3d_measure_cells_only(const pfb_measure_args3d* args, void* stream) {
    return pfb::p3::measure3d_launch(args, static_cast<cudaStream_t>(stream));
}

int pfb3d_apply_cell_motion(const pfb_measure_args3d* args, void* stream) {
    return pfb::p3::motion3d_launch(args, static_cast<cudaStream_t>(stream));
}

int pfb3d_measure_cells(const pfb_measure_args3d* args, void* stream) {
    const int rc = pfb::p3::measure3d_launch(args, static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    return pfb::p3::motion3d_launch(args, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
