// Fused 3D step (sm_100a): measurement, motion and update of a cell in one
// launch.
//
// The reference runs the step as separate kernels (src/pf3d/sim.cu:1460-1651):
// measure every cell (src/pf3d/kernels.cu:1271-1409), apply the motion
// (:1739-1788), then update every cell (:498-793 and
// kernels_periodic_slab_walk.cu:54-318). Here one thread-block cluster of 4
// CTAs per cell does all three; CTA r owns brick planes [r B/4, (r+1) B/4)
// and streams them through a ring of bulk-copied planes (no multicast):
//
//   phase A  measures its planes (the same per-voxel sums and grouping as
//            k_measure3d),
//   fold     pushes its partial record into rank 0 with st.async; rank 0
//            folds the 4 records in rank order, commits the measured record
//            and the recentring plan, applies the tumble and velocity, and
//            pushes {V, velocity, shift, keep} back into every rank. While
//            the fold runs, each CTA already restages the first planes of
//            phase B for a zero z shift (the common case); the brick was read
//            microseconds earlier, so these copies hit L2,
//   phase B  updates its destination planes with the same per-voxel code as
//            k_update3d (planes restaged for the planned z shift).
//
// Given the same committed record, phase B's phi, S and flag counts equal
// k_update3d's bit for bit, and the committed record equals k_measure3d +
// k_motion3d's. The fatal decision is taken per cell: a cell whose record or
// measurement holds a fatal flag, or that sees a fatal counter raised earlier
// in the launch, keeps its field as the reference's update does. A cell
// updated before another cell's fatal flag was raised updates normally; the
// repair and restore passes that follow a fatal step rebuild the same phi, S
// and cell records as after the reference's step, only the global counters of
// that step can count more events.
#include <cuda_runtime.h>

#include "device_util.cuh"
#include "measure3d_common.cuh"
#include "pfb3d_common.cuh"
#include "pfb_internal.h"
#include "ring3d.cuh"
#include "update3d_common.cuh"

namespace pfb {
namespace p3 {

constexpr int kStepCluster = 4;
constexpr int kStepRing = 5;
constexpr uint32_t kBroadcastBytes = 48;

__device__ unsigned int g_step3d_status = 0u;

struct StepArgs3d {
    pfb_measure_args3d m;
    pfb_update_args3d u;
};

struct StepHeader {
    MeasureFold<kStepCluster> fold;
    uint64_t bars[kStepRing];
    uint64_t bar_bc;         // the broadcast of rank 0
    alignas(16) int bc[12];  // V (2 words), vx, vy, vz, sx, sy, sz, keep
    unsigned cnt[kWarps3][6];
    int fail;
};
constexpr size_t kStepHeader = (sizeof(StepHeader) + 127) / 128 * 128;

template <int GEO>
__global__ void __launch_bounds__(kThreads3, 2) k_step3d(const __grid_constant__ StepArgs3d P) {
    constexpr int K = kStepCluster;
    extern __shared__ __align__(128) char smem[];
    StepHeader& H = *reinterpret_cast<StepHeader*>(smem);
    const pfb_measure_args3d& A = P.m;
    const pfb_update_args3d& Q = P.u;
    const int B = A.B, PB = B / K;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rank = (int)dev::cluster_rank();
    const int slot_cell = (int)(blockIdx.x / K);
    const int n = A.selection.ids ? A.selection.ids[slot_cell] : slot_cell;
    pfb_cell3d* cell = &A.cells[n];
    // promoted cells are uniform over the cluster: every CTA returns
    if (cell->storage_edge > (uint32_t)B) return;
    const uint32_t flags0 = cell->flags;
    const pfb_layout3d L = A.layout;
    const int64_t oz = cell->origin_z;
    const size_t words = (size_t)B * B * B;
    const float* src = A.phi + (size_t)n * words;
    float* dst = Q.phi_out + (size_t)n * words;
    const int z0 = rank * PB;

    PlaneRing<kStepRing> ring{reinterpret_cast<float*>(smem + kStepHeader), H.bars, B * B};
    ring.init();
    if (tid == 0) {
        fold_init<K>(H.fold, rank);
        dev::mbar_init(&H.bar_bc, 1);
        dev::mbar_arrive_expect_tx(&H.bar_bc, kBroadcastBytes);
        H.fail = 0;
    }
    if (tid < kWarps3 * 6) (&H.cnt[0][0])[tid] = 0u;
    __syncthreads();
    dev::cluster_arrive_relaxed();

    // Ring requests are numbered across both phases: phase A's request k
    // stages plane z0 - 1 + k (k < nreq); phase B's request base + k stages
    // plane z0 + sz - 1 + k.
    const int nreq = PB + 2;
    int issued = 0;
    auto issue_plane = [&](int k, int plane) {
        int s;
        if (!fetch_plane(L, oz, plane, B, &s)) s = -1;
        ring.issue(k, src, s);
    };
    auto fail = [&](unsigned bit) {
        H.fail = 1;
        atomicOr(&g_step3d_status, bit);
    };

    // ---- phase A: measurement of planes z0 .. z0 + PB - 1
    MeasureCell M;
    M.S = A.S;
    M.L = L;
    M.B = B;
    M.ox = wrap_origin(cell->origin_x, L.nx);
    M.oy = wrap_origin(cell->origin_y, L.ny);
    M.wall = GEO == 2 && A.wall.values;
    M.surface = A.compute_surface != 0;
    const int strips = B / 4;
    const int items = strips * (B / 4);
    for (; issued < kStepRing && issued < nreq; ++issued) issue_plane(issued, z0 - 1 + issued);
    __syncthreads();
    if (!ring.wait(0) || !ring.wait(1)) fail(1u);
    Acc3 acc;
    acc.lox = acc.loy = acc.loz = B;
    MeasureCounts mc;
    for (int i = 0; i < PB; ++i) {
        if (!ring.wait(i + 2)) fail(1u);
        const int z = z0 + i;
        int wz = 0;
        if (!H.fail && aggregate_z(L, oz, z, &wz)) {
            const float wallv = M.wall ? A.wall.values[wz] : 0.0f;
            const bool top_plane = GEO == 1 && wz == L.nz - 1;
            for (int it = tid; it < items; it += kThreads3)
                measure_item(M, ring.slot(i), ring.slot(i + 1), ring.slot(i + 2), 4 * (it % strips),
                             4 * (it / strips), z, wz, wallv, top_plane, acc, mc);
        }
        __syncthreads();
        if (!H.fail && issued < nreq) {
            issue_plane(issued, z0 - 1 + issued);
            ++issued;
        }
    }

    // ---- phase B's first planes for a zero z shift, while the fold runs
    int base = issued;
    if (!H.fail)
        for (int k = 0; k < kStepRing && k < nreq; ++k, ++issued) issue_plane(issued, z0 - 1 + k);

    // ---- fold into rank 0, commit, motion, broadcast
    fold_warps<K>(H.fold, acc, mc);
    __syncthreads();
    dev::cluster_wait();  // every rank's barriers are initialised
    if (warp == 0) {
        fold_send<K>(H.fold, rank, B);
        if (rank == 0) {
            MeasureTotals r;
            const bool rok = fold_receive<K>(H.fold, B, kPlaneWaitPolls, r);
            int rec[12] = {0, 0, 0, 0, 0, 0, 0, 0, 1, 0, 0, 0};
            if (lane == 0) {
                if (!rok) atomicOr(&g_step3d_status, 2u);
                int sx = 0, sy = 0, sz = 0;
                const uint32_t raised = rok ? commit_measure(A, A.B, cell, r, &sx, &sy, &sz) : 0u;
                const bool fatal = !rok || ((flags0 | raised) & PFB3D_FATAL_MASK) != 0u ||
                                   fatal_counters(A.global_flags);
                float v[3] = {0.0f, 0.0f, 0.0f};
                const bool moved = rok && motion_cell(A, cell, fatal, r.t[5], r.t[6], r.t[7], v);
                const bool keep = fatal || !moved || fatal_counters(A.global_flags);
                if (keep) {
                    cell->pending_shift_x = 0;
                    cell->pending_shift_y = 0;
                    cell->pending_shift_z = 0;
                }
                const unsigned long long vb = (unsigned long long)__double_as_longlong(r.t[0]);
                rec[0] = (int)(uint32_t)vb;
                rec[1] = (int)(uint32_t)(vb >> 32);
                rec[2] = __float_as_int(v[0]);
                rec[3] = __float_as_int(v[1]);
                rec[4] = __float_as_int(v[2]);
                rec[5] = sx;
                rec[6] = sy;
                rec[7] = sz;
                rec[8] = keep ? 1 : 0;
            }
#pragma unroll
            for (int k = 0; k < 12; ++k) rec[k] = __shfl_sync(0xFFFFFFFFu, rec[k], 0);
            if (lane < K) {
                const uint32_t bar = dev::map_to_rank(dev::smem_addr(&H.bar_bc), (uint32_t)lane);
#pragma unroll
                for (int k = 0; k < 12; k += 4)
                    dev::st_async_v4b32(dev::map_to_rank(dev::smem_addr(&H.bc[k]), (uint32_t)lane),
                                        rec[k], rec[k + 1], rec[k + 2], rec[k + 3], bar);
            }
        }
    }
    if (!dev::mbar_wait_bounded(&H.bar_bc, 0, kPlaneWaitPolls)) fail(4u);

    // ---- phase B: update of destination planes z0 .. z0 + PB - 1
    UpdateCell U;
    U.S_in = Q.S_in;
    U.S_out = Q.S_out;
    U.L = L;
    U.B = B;
    U.ox = M.ox;
    U.oy = M.oy;
    const double V = __longlong_as_double((long long)(((unsigned long long)(uint32_t)H.bc[1] << 32) |
                                                      (uint32_t)H.bc[0]));
    U.k.gamma = cell->gamma;
    U.k.vx = __int_as_float(H.bc[2]);
    U.k.vy = __int_as_float(H.bc[3]);
    U.k.vz = __int_as_float(H.bc[4]);
    U.k.bulk = Q.bulk_scale * U.k.gamma;
    U.k.volume = (float)(Q.volume_scale * (Q.V0 - V));
    U.k.inter = Q.interaction_coeff;
    U.k.dt = Q.dt;
    const int sx = H.bc[5], sy = H.bc[6], sz = H.bc[7];
    const bool keep = H.fail || H.bc[8] != 0;
    UpdateCounts cnt;
    unsigned clip = 0u;
    if (keep) {
        keep_planes(U, src, dst, z0, z0 + PB, oz, cell, A.global_flags, kThreads3);
    } else {
        if (sz != 0) {
            // drop the speculative planes, stage the shifted ones
            for (int k = base; k < issued; ++k)
                if (!ring.wait(k)) fail(1u);
            __syncthreads();
            base = issued;
            if (!H.fail)
                for (int k = 0; k < kStepRing && k < nreq; ++k, ++issued)
                    issue_plane(issued, z0 + sz - 1 + k);
        }
        const float* wall = GEO == 2 ? Q.wall.values : nullptr;
        if (!ring.wait(base) || !ring.wait(base + 1)) fail(1u);
        for (int i = 0; i < PB; ++i) {
            if (!ring.wait(base + i + 2)) fail(1u);
            const int dz = z0 + i;
            const int zs = dz + sz;
            int wz = 0;
            const bool live = !H.fail && (unsigned)zs < (unsigned)B && aggregate_z(L, oz, zs, &wz);
            const float wallv = GEO == 2 && live ? wall[wz] : 0.0f;
            const bool top_plane = GEO == 1 && live && wz == L.nz - 1;
            for (int it = tid; it < items; it += kThreads3) {
                const int x0 = 4 * (it % strips);
                const int y0 = 4 * (it / strips);
                update_item<GEO>(U, ring.slot(base + i), ring.slot(base + i + 1),
                                 ring.slot(base + i + 2), x0, y0, sx, sy, live, wz, wallv, top_plane,
                                 dst + ((size_t)dz * B + y0) * B + x0, cnt);
            }
            __syncthreads();
            if (!H.fail && issued - base < nreq) {
                issue_plane(issued, z0 + sz - 1 + (issued - base));
                ++issued;
            }
        }
        if ((sx | sy | sz) != 0 && !H.fail)
            clip = clip_check<GEO>(U, src, wall, z0, z0 + PB, sx, sy, sz, oz, cnt, kThreads3);
    }
    raise_update_counts<kThreads3>(H.cnt, cnt, clip, cell, A.global_flags);

    // no bulk copy may still target this CTA's shared memory at exit
    for (int k = issued > kStepRing ? issued - kStepRing : 0; k < issued; ++k) (void)ring.wait(k);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static size_t step_smem(int B) { return kStepHeader + (size_t)kStepRing * (size_t)B * B * 4; }

// Cluster size of the fused step for brick edge B: 4 when B / 4 is a whole
// number of planes and the ring fits the shared memory of a CTA, else 0.
int step3d_cluster(int B) {
    if (B <= 0 || B % kBrickAlign != 0 || B % kStepCluster != 0) return 0;
    return step_smem(B) <= 227 * 1024 ? kStepCluster : 0;
}

size_t step3d_smem(int B) { return step3d_cluster(B) ? step_smem(B) : 0; }

template <int GEO>
static int step_launch_g(const StepArgs3d& P, int count, cudaStream_t stream) {
    const size_t smem = step_smem(P.m.B);
    cudaError_t e = cudaFuncSetAttribute(k_step3d<GEO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "step attribute: %s", cudaGetErrorString(e));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(count * kStepCluster), 1, 1);
    cfg.blockDim = dim3(kThreads3, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kStepCluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    e = cudaLaunchKernelEx(&cfg, k_step3d<GEO>, P);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "step launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

static bool same_layout(const pfb_layout3d& a, const pfb_layout3d& b) {
    return a.nx == b.nx && a.ny == b.ny && a.nz == b.nz && a.pitch_x == b.pitch_x &&
           a.boundary_flags == b.boundary_flags;
}

int step3d_launch(const pfb_measure_args3d* m, const pfb_update_args3d* u, cudaStream_t stream) {
    int rc = check_measure(m);
    if (!rc) rc = check_update(u);
    if (rc) return rc;
    const pfb_measure_args3d& A = *m;
    const pfb_update_args3d& Q = *u;
    if (A.phi != Q.phi_in || A.S != Q.S_in || A.cells != Q.cells ||
        A.global_flags != Q.global_flags || A.N != Q.N || A.B != Q.B ||
        !same_layout(A.layout, Q.layout) || A.wall.values != Q.wall.values ||
        A.wall.planes != Q.wall.planes || A.selection.ids != Q.selection.ids ||
        (A.selection.ids && A.selection.count != Q.selection.count))
        return set_error(PFB_E_ARG, "measure and update arguments describe different systems");
    if (step3d_cluster(A.B) == 0)
        return set_error(PFB_E_CONFIG, "brick edge %d does not fit the fused step", A.B);
    const int count = A.selection.ids ? A.selection.count : A.N;
    if (count == 0) return PFB_OK;
    StepArgs3d P;
    P.m = A;
    P.u = Q;
    const uint32_t bf = A.layout.boundary_flags;
    if (periodic_xyz(bf)) return step_launch_g<0>(P, count, stream);
    if (substrate_slab(bf)) return step_launch_g<1>(P, count, stream);
    return step_launch_g<2>(P, count, stream);
}

int step3d_read_status(unsigned* out, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_step3d_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status read: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_step3d_status, &z, sizeof(z));
    }
    if (out) *out = v;
    return PFB_OK;
}

}  // namespace p3
}  // namespace pfb

extern "C" {

int pfb3d_step_fused(const pfb_measure_args3d* measure, const pfb_update_args3d* update,
                     void* stream) {
    return pfb::p3::step3d_launch(measure, update, static_cast<cudaStream_t>(stream));
}

int pfb3d_step_cluster(int B) { return pfb::p3::step3d_cluster(B); }

int pfb3d_device_status(unsigned* out, int clear) {
    unsigned a = 0, b = 0, c = 0;
    int rc = pfb::p3::measure3d_read_status(&a, clear);
    if (!rc) rc = pfb::p3::update3d_read_status(&b, clear);
    if (!rc) rc = pfb::p3::step3d_read_status(&c, clear);
    if (out) *out = a | (b << 2) | (c << 4);
    return rc;
}

}  // extern "C"
