// 3D measurement and motion (sm_100a).
//
// k_measure3d<K>: one thread-block cluster of K CTAs per cell (K as in the
// fused step k_step3d for the same brick edge, so both group the FP64 sums
// alike); CTA r walks
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
#include "measure3d_common.cuh"
#include "ring3d.cuh"
#include "storage2d.cuh"

namespace pfb {
namespace p3 {

constexpr int kMeasureRing = 4;

__device__ unsigned int g_measure3d_status = 0u;

template <int K>
struct MeasureHeader {
    uint64_t bars[kMeasureRing];
    int abort;
    int pad[3];
    MeasureFold<K> fold;
};

// T: storage type of the phi pool (binary32, or binary16 / bfloat16 widened
// on load).
template <int K, typename T>
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
    if (cell->storage_edge > (uint32_t)B) return;

    PlaneRing<kMeasureRing, T> ring{reinterpret_cast<T*>(smem + kHeader), H.bars, B * B};
    ring.init();
    if (tid == 0) {
        fold_init<K>(H.fold, rank);
        H.abort = 0;
    }
    __syncthreads();
    dev::cluster_arrive_relaxed();

    const pfb_layout3d L = A.layout;
    const uint32_t bf = L.boundary_flags;
    const int64_t oz = cell->origin_z;
    MeasureCell M;
    M.S = A.S;
    M.L = L;
    M.B = B;
    M.ox = wrap_origin(cell->origin_x, L.nx);
    M.oy = wrap_origin(cell->origin_y, L.ny);
    M.wall = hard_wall_channel(bf) && A.wall.values;
    M.surface = A.compute_surface != 0;
    const T* field = reinterpret_cast<const T*>(A.phi) + (size_t)n * (size_t)B * B * B;
    const int PB = B / K;
    const int z0 = rank * PB;

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
    MeasureCounts mc;
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
            const float wallv = M.wall ? A.wall.values[wz] : 0.0f;
            const bool top_plane = substrate_slab(bf) && wz == L.nz - 1;
            for (int it = tid; it < items; it += kThreads3)
                measure_item(M, ring.slot(i), ring.slot(i + 1), ring.slot(i + 2), 4 * (it % strips),
                             4 * (it / strips), z, wz, wallv, top_plane, acc, mc);
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

    fold_warps<K>(H.fold, acc, mc);
    __syncthreads();
    dev::cluster_wait();  // rank 0's receive barrier is initialised
    if (warp == 0) {
        fold_send<K>(H.fold, rank, B);
        if (rank == 0) {
            MeasureTotals r;
            if (!fold_receive<K>(H.fold, B, kPlaneWaitPolls, r)) atomicOr(&g_measure3d_status, 2u);
            if (lane == 0) {
                int sx, sy, sz;
                (void)commit_measure(A, A.B, cell, r, &sx, &sy, &sz);
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
    float v[3];
    (void)motion_cell(A, c, fatal, c->Ix, c->Iy, c->Iz, v);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
template <int K>
static size_t measure_smem(int B, int bytes) {
    const size_t header = (sizeof(MeasureHeader<K>) + 127) / 128 * 128;
    return header + (size_t)kMeasureRing * (size_t)B * B * bytes;
}

int geometry_ok3(int B, const pfb_layout3d& L) {
    const uint32_t b = L.boundary_flags;
    if (!(periodic_xyz(b) || substrate_slab(b) || hard_wall_channel(b))) return 0;
    return B > 0 && B % kBrickAlign == 0 && L.nx > B && L.ny > B &&
           (hard_wall_channel(b) ? L.nz > 0 : L.nz > B) && L.pitch_x >= L.nx &&
           L.pitch_x % 4 == 0;
}

int check_measure(const pfb_measure_args3d* a) {
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
    if (((uintptr_t)A.phi & 15u)) return set_error(PFB_E_ARG, "phi pools must be 16-byte aligned");
    return PFB_OK;
}

template <int K, typename T>
static int measure_launch_k(const pfb_measure_args3d& A, int count, cudaStream_t stream) {
    const size_t smem = measure_smem<K>(A.B, (int)sizeof(T));
    if (smem > 227 * 1024) return set_error(PFB_E_CONFIG, "brick edge too large for the plane ring");
    cudaError_t e = cudaFuncSetAttribute(k_measure3d<K, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess && K > 8)
        e = cudaFuncSetAttribute(k_measure3d<K, T>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
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
    e = cudaLaunchKernelEx(&cfg, k_measure3d<K, T>, A);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "measure launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

// The measurement's cluster size: 4, as the fused step's, so the two paths
// sum the moments in the same grouping.
int measure3d_cluster(int) { return 4; }

int measure3d_launch(const pfb_measure_args3d* a, cudaStream_t stream) {
    return measure3d_launch_pool(a, kStoreF32, stream);
}

int measure3d_launch_pool(const pfb_measure_args3d* a, int storage, cudaStream_t stream) {
    int rc = check_measure(a);
    if (rc) return rc;
    const pfb_measure_args3d& A = *a;
    const int count = A.selection.ids ? A.selection.count : A.N;
    if (count == 0) return PFB_OK;
    const int K = measure3d_cluster(A.B);
    if (K != 4 || A.B % K != 0) return set_error(PFB_E_CONFIG, "brick edge is not a multiple of 4");
    if (storage == kStoreF16) return measure_launch_k<4, __half>(A, count, stream);
    if (storage == kStoreBF16) return measure_launch_k<4, __nv_bfloat16>(A, count, stream);
    if (storage != kStoreF32) return set_error(PFB_E_ARG, "unknown phi storage");
    return measure_launch_k<4, float>(A, count, stream);
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
