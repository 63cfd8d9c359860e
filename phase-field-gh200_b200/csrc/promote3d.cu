// Adaptive 3D bricks (sm_100a): the kernels of cells whose support outgrew
// the base brick. Such a cell lives in its own cube of edge E > B (its
// record's storage_edge = E), addressed through a per-cell pointer table and
// a list of promoted cell ids; the base-brick kernels skip it. Per-voxel
// arithmetic is the base kernels' (measure_item, update_item), so a promoted
// cell's update is bit-identical to the reference's promoted update on the
// same record, and its measurement agrees to the last bits of the FP64 sums.
//
// Reference behaviour restated here:
//   tier growth and centred crop rules   include/pf3d/brick_classes.hpp:13-75
//   promoted scatter and crop check      src/pf3d/kernels.cu:1188-1262
//   promoted measurement and update      src/pf3d/kernels.cu:1413-1427, 1888-1925
//   resize of a cell record              src/pf3d/adaptive_storage.cu:87-109
//
// Planes are read straight from the cube in global memory (a promoted cube
// at E = 128 has 64 KB planes, too large for a shared-memory ring); planes
// outside the cube or the domain read a static zero plane.
#include <cuda_runtime.h>

#include <cstdint>

#include "device_util.cuh"
#include "measure3d_common.cuh"
#include "pfb3d_common.cuh"
#include "pfb_internal.h"
#include "ring3d.cuh"
#include "update3d_common.cuh"

namespace pfb {
namespace p3 {

constexpr int kPromotedCluster = 4;  // measurement CTAs per cube (a cluster)
constexpr int kPromotedParts = 4;    // update CTAs per cube

// Never written: zero-initialised device memory standing for absent planes.
__device__ __align__(16) float g_zero_plane3d[kMaxPromotedEdge * kMaxPromotedEdge];
__device__ unsigned int g_promote3d_status = 0u;

// Edge of a promoted cell: its storage edge when above the base edge, at most
// max_edge and aligned; 0 otherwise (the cell is skipped).
__device__ __forceinline__ int promoted_edge(const pfb_cell3d& c, int B, int max_edge) {
    const uint32_t e = c.storage_edge;
    return (e > (uint32_t)B && e <= (uint32_t)max_edge && e % kBrickAlign == 0u) ? (int)e : 0;
}

// Plane z of a cube of edge E as the update and the measurement see it.
__device__ __forceinline__ const float* cube_plane(const float* cube, const pfb_layout3d& L,
                                                   int64_t oz, int z, int E) {
    int s;
    return fetch_plane(L, oz, z, E, &s) ? cube + (size_t)s * E * E : g_zero_plane3d;
}

template <int K>
__global__ void __launch_bounds__(kThreads3, 2)
    k_measure3d_promoted(const __grid_constant__ pfb_measure_args3d A, float* const* cubes,
                         const int* ids, int max_edge) {
    __shared__ MeasureFold<K> F;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int rank = (int)dev::cluster_rank();
    const int n = ids[blockIdx.x / K];
    pfb_cell3d* cell = &A.cells[n];
    const int E = promoted_edge(*cell, A.B, max_edge);
    const float* cube = cubes[n];
    // uniform over the cluster: every CTA of the cell returns
    if (E == 0 || cube == nullptr) return;
    if (tid == 0) fold_init<K>(F, rank);
    __syncthreads();
    dev::cluster_arrive_relaxed();

    const pfb_layout3d L = A.layout;
    const uint32_t bf = L.boundary_flags;
    const int64_t oz = cell->origin_z;
    MeasureCell M;
    M.S = A.S;
    M.L = L;
    M.B = E;
    M.ox = wrap_origin(cell->origin_x, L.nx);
    M.oy = wrap_origin(cell->origin_y, L.ny);
    M.wall = hard_wall_channel(bf) && A.wall.values;
    M.surface = A.compute_surface != 0;
    const int PB = E / K, z0 = rank * PB;
    const int strips = E / 4, items = strips * strips;
    Acc3 acc;
    acc.lox = acc.loy = acc.loz = E;
    MeasureCounts mc;
    for (int i = 0; i < PB; ++i) {
        const int z = z0 + i;
        int wz = 0;
        if (!aggregate_z(L, oz, z, &wz)) continue;
        const float* pm = cube_plane(cube, L, oz, z - 1, E);
        const float* pc = cube_plane(cube, L, oz, z, E);
        const float* pp = cube_plane(cube, L, oz, z + 1, E);
        const float wallv = M.wall ? A.wall.values[wz] : 0.0f;
        const bool top_plane = substrate_slab(bf) && wz == L.nz - 1;
        for (int it = tid; it < items; it += kThreads3)
            measure_item(M, pm, pc, pp, 4 * (it % strips), 4 * (it / strips), z, wz, wallv, top_plane,
                         acc, mc);
    }
    fold_warps<K>(F, acc, mc);
    __syncthreads();
    dev::cluster_wait();
    if (warp == 0) {
        fold_send<K>(F, rank, E);
        if (rank == 0) {
            MeasureTotals r;
            if (!fold_receive<K>(F, E, kPlaneWaitPolls, r)) atomicOr(&g_promote3d_status, 1u);
            if (lane == 0) {
                int sx, sy, sz;
                (void)commit_measure(A, E, cell, r, &sx, &sy, &sz);
            }
        }
    }
}

template <int GEO>
__global__ void __launch_bounds__(kThreads3, 2)
    k_update3d_promoted(const __grid_constant__ pfb_update_args3d A, float* const* in,
                        float* const* out, const int* ids, int max_edge) {
    __shared__ int keep;
    __shared__ unsigned cnt[kWarps3][6];
    const int tid = threadIdx.x;
    const int n = ids[blockIdx.x / kPromotedParts];
    const int part = (int)(blockIdx.x % kPromotedParts);
    pfb_cell3d* cell = &A.cells[n];
    const int E = promoted_edge(*cell, A.B, max_edge);
    const float* src = in[n];
    float* dst = out[n];
    if (E == 0 || src == nullptr || dst == nullptr || src == dst) return;
    const pfb_layout3d L = A.layout;
    const int64_t oz = cell->origin_z;
    const int PB = E / kPromotedParts, d0 = part * PB, d1 = d0 + PB;
    UpdateCell U;
    U.S_in = A.S_in;
    U.S_out = A.S_out;
    U.L = L;
    U.B = E;
    U.ox = wrap_origin(cell->origin_x, L.nx);
    U.oy = wrap_origin(cell->origin_y, L.ny);
    if (tid == 0) keep = fatal3(cell, A.global_flags) ? 1 : 0;
    if (tid < kWarps3 * 6) (&cnt[0][0])[tid] = 0u;
    __syncthreads();
    if (keep) {
        keep_planes(U, src, dst, d0, d1, oz, cell, A.global_flags, kThreads3);
        __syncthreads();
        if (tid == 0 && part == 0) {
            cell->pending_shift_x = 0;
            cell->pending_shift_y = 0;
            cell->pending_shift_z = 0;
        }
        return;
    }
    const int sx = cell->pending_shift_x, sy = cell->pending_shift_y, sz = cell->pending_shift_z;
    U.k.gamma = cell->gamma;
    U.k.vx = cell->velocity_x;
    U.k.vy = cell->velocity_y;
    U.k.vz = cell->velocity_z;
    U.k.bulk = A.bulk_scale * U.k.gamma;
    U.k.volume = (float)(A.volume_scale * (A.V0 - cell->V));
    U.k.inter = A.interaction_coeff;
    U.k.dt = A.dt;
    const float* wall = GEO == 2 ? A.wall.values : nullptr;
    const int strips = E / 4, items = strips * strips;
    UpdateCounts c;
    for (int i = 0; i < PB; ++i) {
        const int dz = d0 + i;
        const int zs = dz + sz;
        int wz = 0;
        const bool live = (unsigned)zs < (unsigned)E && aggregate_z(L, oz, zs, &wz);
        const float* p0 = cube_plane(src, L, oz, zs - 1, E);
        const float* p1 = cube_plane(src, L, oz, zs, E);
        const float* p2 = cube_plane(src, L, oz, zs + 1, E);
        const float wallv = GEO == 2 && live ? wall[wz] : 0.0f;
        const bool top_plane = GEO == 1 && live && wz == L.nz - 1;
        for (int it = tid; it < items; it += kThreads3) {
            const int x0 = 4 * (it % strips), y0 = 4 * (it / strips);
            update_item<GEO>(U, p0, p1, p2, x0, y0, sx, sy, live, wz, wallv, top_plane,
                             dst + ((size_t)dz * E + y0) * E + x0, c);
        }
    }
    unsigned clip = 0u;
    if ((sx | sy | sz) != 0) clip = clip_check<GEO>(U, src, wall, d0, d1, sx, sy, sz, oz, c, kThreads3);
    raise_update_counts<kThreads3>(cnt, c, clip, cell, A.global_flags);
}

__device__ __forceinline__ bool fatal_any(const uint32_t* g) {
    if (!g) return false;
    for (int f = 0; f < PFB3D_FLAG_COUNT; ++f)
        if (((PFB3D_FATAL_MASK >> f) & 1u) && g[f]) return true;
    return false;
}

// Q5.27 scatter of each promoted cube (one CTA per cube, one warp per row);
// with guard_fatal only on a step that holds a fatal counter.
__global__ void k_scatter3d_promoted(const __grid_constant__ pfb_scatter_args3d A,
                                     float* const* cubes, const int* ids, int max_edge,
                                     int guard_fatal) {
    if (guard_fatal && !fatal_any(A.global_flags)) return;
    const int n = ids[blockIdx.x];
    pfb_cell3d* cell = &A.cells[n];
    const int E = promoted_edge(*cell, A.B, max_edge);
    const float* cube = cubes[n];
    if (E == 0 || cube == nullptr) return;
    const pfb_layout3d& L = A.layout;
    const int ox = wrap_origin(cell->origin_x, L.nx), oy = wrap_origin(cell->origin_y, L.ny);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int row = warp; row < E * E; row += warps) {
        const int z = row / E, y = row - z * E;
        int wz;
        if (!aggregate_z(L, cell->origin_z, z, &wz)) continue;
        const size_t base = s_index(L, 0, wrap_offset(oy, y, L.ny), wz);
        const float* gr = cube + (size_t)row * E;
        for (int x = lane; x < E; x += 32) {
            const float v = gr[x];
            if (!isfinite(v)) {
                raise3(cell, A.global_flags, PFB3D_FLAG_NONFINITE, 1u);
                continue;
            }
            if (v * v > kQClamp3) raise3(cell, A.global_flags, PFB3D_FLAG_Q_CLAMP, 1u);
            const uint32_t q = q_of3(v);
            if (!q) continue;
            const uint32_t old = atomicAdd(&A.S[base + wrap_offset(ox, x, L.nx)], q);
            if (old > 0xFFFFFFFFu - q) raise3(cell, A.global_flags, PFB3D_FLAG_S_OVERFLOW, 1u);
        }
    }
}

// Fatal step: each promoted cube keeps its accepted field, the planned shift
// is dropped (reference launch_repair_promoted_after_fatal).
__global__ void k_repair3d_promoted(float* const* in, float* const* out, pfb_cell3d* cells,
                                    const uint32_t* g, const int* ids, int B, int max_edge) {
    if (!fatal_any(g)) return;
    const int n = ids[blockIdx.x];
    pfb_cell3d* cell = &cells[n];
    const int E = promoted_edge(*cell, B, max_edge);
    if (E == 0 || !in[n] || !out[n] || in[n] == out[n]) return;
    const float4* s4 = reinterpret_cast<const float4*>(in[n]);
    float4* d4 = reinterpret_cast<float4*>(out[n]);
    const size_t v4 = (size_t)E * E * E / 4;
    for (size_t i = threadIdx.x; i < v4; i += blockDim.x) d4[i] = s4[i];
    if (threadIdx.x == 0) {
        cell->pending_shift_x = 0;
        cell->pending_shift_y = 0;
        cell->pending_shift_z = 0;
    }
}

// dst (edge Ed) = src (edge Es) moved by `off` voxels on every axis
// (off = (Ed - Es) / 2: growth embeds the whole source, a crop keeps the
// centre); voxels without a source are zero.
__global__ void k_copy_centred3d(const float* src, int Es, float* dst, int Ed, int off) {
    const size_t total = (size_t)Ed * Ed * Ed;
    for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(q % Ed) - off;
        const int y = (int)((q / Ed) % Ed) - off;
        const int z = (int)(q / ((size_t)Ed * Ed)) - off;
        const bool in = (unsigned)x < (unsigned)Es && (unsigned)y < (unsigned)Es &&
                        (unsigned)z < (unsigned)Es;
        dst[q] = in ? src[((size_t)z * Es + y) * Es + x] : 0.0f;
    }
}

// A centred crop of cube n to candidate[n] is refused unless every voxel
// outside the retained cube's inner guard band (8 planes per face) is an exact
// (signed) zero and every voxel is finite (reference k_check_promoted_crops).
__global__ void k_check_crops3d(float* const* cubes, const pfb_cell3d* cells, const int* candidate,
                                uint32_t* rejected, int N, int B) {
    const int n = (int)blockIdx.x;
    if (n >= N) return;
    const int target = candidate[n];
    if (target == 0) return;
    constexpr int kGuard = 8;
    const uint32_t se = cells[n].storage_edge;
    const int E = (se > (uint32_t)B && se % kBrickAlign == 0u && se <= (uint32_t)kMaxPromotedEdge) ? (int)se : 0;
    const bool valid = E > 0 && target >= B && target < E && target > 2 * kGuard &&
                       target % kBrickAlign == 0 && cubes[n] != nullptr;
    if (!valid) {
        if (threadIdx.x == 0) atomicOr(rejected + n, 1u);
        return;
    }
    const int off = (E - target) / 2;
    const int lo = off + kGuard, hi = off + target - kGuard;
    const float* cube = cubes[n];
    const size_t total = (size_t)E * E * E;
    int bad = 0;
    for (size_t q = threadIdx.x; q < total && !bad; q += blockDim.x) {
        const float v = cube[q];
        const int x = (int)(q % E), y = (int)((q / E) % E), z = (int)(q / ((size_t)E * E));
        const bool outside = x < lo || x >= hi || y < lo || y >= hi || z < lo || z >= hi;
        if (!isfinite(v) || (outside && v != 0.0f)) bad = 1;
    }
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(rejected + n, 1u);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
int next_brick_edge3(int current, int maximum) {
    if (current <= 0 || current % kBrickAlign != 0 || maximum <= current) return 0;
    const int limit = maximum - maximum % kBrickAlign;
    if (limit <= current) return 0;
    const int64_t want = ((int64_t)current + kBrickGrowth + kBrickTier - 1) / kBrickTier * kBrickTier;
    return want < limit ? (int)want : limit;
}

int shrink_brick_edge3(int current, int minimum, const int* lo, const int* hi) {
    if (current <= 0 || current % kBrickAlign != 0 || minimum <= 0 || minimum % kBrickAlign != 0 ||
        minimum >= current || !lo || !hi)
        return current;
    int spare = current;
    for (int a = 0; a < 3; ++a) {
        if (lo[a] < 0 || hi[a] < lo[a] || hi[a] >= current) return current;
        spare = spare < lo[a] ? spare : lo[a];
        const int above = current - 1 - hi[a];
        spare = spare < above ? spare : above;
    }
    if (spare <= kBrickShrinkSpare) return current;
    const int64_t needed = (int64_t)current - 2 * (int64_t)(spare - kBrickShrinkSpare);
    const int64_t rounded = (needed + kBrickTier - 1) / kBrickTier * kBrickTier;
    if (rounded >= current) return current;
    const int cand = rounded < minimum ? minimum : (int)rounded;
    return cand < current ? cand : current;
}

static int check_table(const void* table, const int* ids, int count, int max_edge) {
    if (count < 0) return set_error(PFB_E_ARG, "negative promoted count");
    if (count > 0 && (!table || !ids)) return set_error(PFB_E_ARG, "null promoted table or id list");
    if (max_edge <= 0 || max_edge > kMaxPromotedEdge || max_edge % kBrickAlign != 0)
        return set_error(PFB_E_CONFIG, "promoted edge %d outside 8..%d", max_edge, kMaxPromotedEdge);
    return PFB_OK;
}

int measure3d_promoted_launch(const pfb_measure_args3d* a, float* const* cubes, const int* ids,
                              int count, int max_edge, cudaStream_t stream) {
    int rc = check_measure(a);
    if (!rc) rc = check_table(cubes, ids, count, max_edge);
    if (rc || count == 0) return rc;
    constexpr int K = kPromotedCluster;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)(count * K), 1, 1);
    cfg.blockDim = dim3(kThreads3, 1, 1);
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k_measure3d_promoted<K>, *a, cubes, ids, max_edge);
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "promoted measure: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int update3d_promoted_launch(const pfb_update_args3d* a, float* const* in, float* const* out,
                             const int* ids, int count, int max_edge, cudaStream_t stream) {
    // the base pools of the record are not touched here
    int rc = check_update(a, false);
    if (!rc) rc = check_table(in, ids, count, max_edge);
    if (!rc && count > 0 && !out) rc = set_error(PFB_E_ARG, "null promoted output table");
    if (rc || count == 0) return rc;
    const dim3 grid((unsigned)(count * kPromotedParts));
    const uint32_t bf = a->layout.boundary_flags;
    if (periodic_xyz(bf))
        k_update3d_promoted<0><<<grid, kThreads3, 0, stream>>>(*a, in, out, ids, max_edge);
    else if (substrate_slab(bf))
        k_update3d_promoted<1><<<grid, kThreads3, 0, stream>>>(*a, in, out, ids, max_edge);
    else
        k_update3d_promoted<2><<<grid, kThreads3, 0, stream>>>(*a, in, out, ids, max_edge);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "promoted update: %s", cudaGetErrorString(e));
}

int scatter3d_promoted_launch(const pfb_scatter_args3d* a, float* const* cubes, const int* ids,
                              int count, int max_edge, int guard_fatal, cudaStream_t stream) {
    if (!a || !a->cells || !a->S) return set_error(PFB_E_ARG, "invalid promoted scatter arguments");
    const int rc = check_table(cubes, ids, count, max_edge);
    if (rc || count == 0) return rc;
    k_scatter3d_promoted<<<count, 256, 0, stream>>>(*a, cubes, ids, max_edge, guard_fatal);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "promoted scatter: %s", cudaGetErrorString(e));
}

int repair3d_promoted_launch(const pfb_update_args3d* a, float* const* in, float* const* out,
                             const int* ids, int count, int max_edge, cudaStream_t stream) {
    if (!a || !a->cells || !a->global_flags) return set_error(PFB_E_ARG, "invalid promoted repair arguments");
    int rc = check_table(in, ids, count, max_edge);
    if (rc || count == 0) return rc;
    k_repair3d_promoted<<<count, 256, 0, stream>>>(in, out, a->cells, a->global_flags, ids, a->B, max_edge);
    if (a->S_out) {
        pfb_scatter_args3d s{};
        s.phi = nullptr;
        s.cells = a->cells;
        s.S = a->S_out;
        s.global_flags = a->global_flags;
        s.layout = a->layout;
        s.N = a->N;
        s.B = a->B;
        rc = scatter3d_promoted_launch(&s, in, ids, count, max_edge, 1, stream);
        if (rc) return rc;
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "promoted repair: %s", cudaGetErrorString(e));
}

int copy_centred3d_launch(const float* src, int Es, float* dst, int Ed, cudaStream_t stream) {
    if (!src || !dst || Es <= 0 || Ed <= 0 || Es % kBrickAlign || Ed % kBrickAlign)
        return set_error(PFB_E_ARG, "invalid centred copy");
    const size_t total = (size_t)Ed * Ed * Ed;
    const unsigned blocks = (unsigned)((total + 255) / 256 < 148 * 16 ? (total + 255) / 256 : 148 * 16);
    k_copy_centred3d<<<blocks, 256, 0, stream>>>(src, Es, dst, Ed, (Ed - Es) / 2);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "centred copy: %s", cudaGetErrorString(e));
}

int check_crops3d_launch(float* const* cubes, const pfb_cell3d* cells, const int* candidate,
                         uint32_t* rejected, int N, int B, cudaStream_t stream) {
    if (!cubes || !cells || !candidate || !rejected || N <= 0 || B <= 0)
        return set_error(PFB_E_ARG, "invalid crop check arguments");
    k_check_crops3d<<<N, 256, 0, stream>>>(cubes, cells, candidate, rejected, N, B);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "crop check: %s", cudaGetErrorString(e));
}

int promote3d_read_status(unsigned* out, int clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_promote3d_status, sizeof(v));
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "status read: %s", cudaGetErrorString(e));
    if (clear) {
        const unsigned z = 0;
        cudaMemcpyToSymbol(g_promote3d_status, &z, sizeof(z));
    }
    if (out) *out = v;
    return PFB_OK;
}

}  // namespace p3
}  // namespace pfb

using namespace pfb::p3;

extern "C" {

int pfb3d_next_brick_edge(int current, int maximum) { return next_brick_edge3(current, maximum); }

int pfb3d_shrink_brick_edge(int current, int minimum, const int* lo3, const int* hi3) {
    return shrink_brick_edge3(current, minimum, lo3, hi3);
}

int pfb3d_measure_promoted(const pfb_measure_args3d* args, float* const* promoted_phi,
                           const int* promoted_ids, int promoted_count, int promoted_edge,
                           void* stream) {
    return measure3d_promoted_launch(args, promoted_phi, promoted_ids, promoted_count, promoted_edge,
                                     static_cast<cudaStream_t>(stream));
}

int pfb3d_update_promoted(const pfb_update_args3d* args, float* const* promoted_phi_in,
                          float* const* promoted_phi_out, const int* promoted_ids,
                          int promoted_count, int promoted_edge, void* stream) {
    return update3d_promoted_launch(args, promoted_phi_in, promoted_phi_out, promoted_ids,
                                    promoted_count, promoted_edge, static_cast<cudaStream_t>(stream));
}

int pfb3d_scatter_promoted(const pfb_scatter_args3d* args, float* const* promoted_phi,
                           const int* promoted_ids, int promoted_count, int promoted_edge,
                           void* stream) {
    return scatter3d_promoted_launch(args, promoted_phi, promoted_ids, promoted_count, promoted_edge,
                                     0, static_cast<cudaStream_t>(stream));
}

int pfb3d_repair_promoted_after_fatal(const pfb_update_args3d* args, float* const* promoted_phi_in,
                                      float* const* promoted_phi_out, const int* promoted_ids,
                                      int promoted_count, int promoted_edge, void* stream) {
    return repair3d_promoted_launch(args, promoted_phi_in, promoted_phi_out, promoted_ids,
                                    promoted_count, promoted_edge, static_cast<cudaStream_t>(stream));
}

int pfb3d_check_promoted_crops(float* const* promoted_phi, const pfb_cell3d* cells,
                               const int* candidate_edges, uint32_t* rejected, int N, int base_edge,
                               void* stream) {
    return check_crops3d_launch(promoted_phi, cells, candidate_edges, rejected, N, base_edge,
                                static_cast<cudaStream_t>(stream));
}

}  // extern "C"
