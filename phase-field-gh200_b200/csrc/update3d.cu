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

#include <vector>

#include "device_util.cuh"
#include "pfb3d_common.cuh"
#include "pfb_internal.h"
#include "ring3d.cuh"
#include "storage2d.cuh"
#include "update3d_common.cuh"

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

// GEO: 0 periodic, 1 substrate slab, 2 hard-wall channel; T: storage type
// of the phi pools. out_by_slot: the output brick of selection slot k is
// phi_out + k B^3 (the scratch bricks of the in-place modes) instead of the
// cell's own slot. Rounding of 16-bit pools: stream of (step, cell, sr_seed).
struct PoolRounding {
    const uint64_t* step;
    uint64_t seed;
};

template <int GEO, typename T>
__global__ void __launch_bounds__(kUThreads, 2)
    k_update3d(const __grid_constant__ pfb_update_args3d A, int out_by_slot, PoolRounding R) {
    extern __shared__ __align__(128) char smem[];
    UpdateHeader& H = *reinterpret_cast<UpdateHeader*>(smem);
    const int B = A.B;
    const int tid = threadIdx.x;
    const int slot_cell = (int)(blockIdx.x / kUCtasPerCell);
    const int part = (int)(blockIdx.x % kUCtasPerCell);
    const int n = A.selection.ids ? A.selection.ids[slot_cell] : slot_cell;
    pfb_cell3d* cell = &A.cells[n];
    if (cell->storage_edge > (uint32_t)B) return;
    const pfb_layout3d L = A.layout;
    const size_t words = (size_t)B * B * B;
    const T* src = reinterpret_cast<const T*>(A.phi_in) + (size_t)n * words;
    T* dst = reinterpret_cast<T*>(A.phi_out) + (size_t)(out_by_slot ? slot_cell : n) * words;
    const int PB = B / kUCtasPerCell;
    const int d0 = part * PB, d1 = d0 + PB;
    const int64_t oz = cell->origin_z;
    const uint32_t sr = Store<T>::kHalf ? sr_stream(R.step ? *R.step : 0ull, cell->global_id, R.seed) : 0u;

    UpdateCell U;
    U.S_in = A.S_in;
    U.S_out = A.S_out;
    U.L = L;
    U.B = B;
    U.ox = wrap_origin(cell->origin_x, L.nx);
    U.oy = wrap_origin(cell->origin_y, L.ny);

    if (tid == 0) H.abort = fatal3(cell, A.global_flags) ? 1 : 0;
    if (tid < (kUThreads / 32) * 6) (&H.cnt[0][0])[tid] = 0u;
    __syncthreads();
    if (H.abort) {
        keep_planes(U, src, dst, d0, d1, oz, cell, A.global_flags, kUThreads);
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

    PlaneRing<kURing, T> ring{reinterpret_cast<T*>(smem + kUHeader), H.bars, B * B};
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

    UpdateCounts cnt;
    const int strips = B / 4;
    const int items = strips * (B / 4);
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
        const bool live = zin && aggregate_z(L, oz, zs, &wz) && !H.abort;
        const float wallv = GEO == 2 && live ? wall[wz] : 0.0f;
        const bool top_plane = GEO == 1 && live && wz == L.nz - 1;
        for (int it = tid; it < items; it += kUThreads) {
            const int x0 = 4 * (it % strips);
            const int y0 = 4 * (it / strips);
            const uint32_t pix0 = (uint32_t)(((size_t)dz * B + y0) * B + x0);
            update_item<GEO, T>(U, ring.slot(i), ring.slot(i + 1), ring.slot(i + 2), x0, y0, sx, sy,
                                live, wz, wallv, top_plane, dst + pix0, cnt, sr, pix0);
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

    unsigned clip = 0u;
    if ((sx | sy | sz) != 0 && !H.abort)
        clip = clip_check<GEO, T>(U, src, wall, d0, d1, sx, sy, sz, oz, cnt, kUThreads);
    raise_update_counts<kUThreads>(H.cnt, cnt, clip, cell, A.global_flags);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
int geometry_ok3(int B, const pfb_layout3d& L);

size_t update3d_smem(int B, int bytes = 4) {
    return (size_t)kUHeader + (size_t)kURing * (size_t)B * B * bytes;
}

int check_update(const pfb_update_args3d* a, bool pools) {
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
    if (!A.S_in || !A.cells || (A.S_out && A.S_out == A.S_in))
        return set_error(PFB_E_ARG, "invalid buffers in update arguments");
    if (!pools) return PFB_OK;
    if (!A.phi_in || !A.phi_out || A.phi_in == A.phi_out)
        return set_error(PFB_E_ARG, "invalid phi pools in update arguments");
    if (((uintptr_t)A.phi_in & 15u) || ((uintptr_t)A.phi_out & 15u))
        return set_error(PFB_E_ARG, "phi pools must be 16-byte aligned");
    return PFB_OK;
}

template <int GEO, typename T>
static cudaError_t update_launch_gt(const pfb_update_args3d& A, int out_by_slot, PoolRounding R,
                                    dim3 grid, size_t smem, cudaStream_t stream) {
    cudaError_t e = cudaFuncSetAttribute(k_update3d<GEO, T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e == cudaSuccess) k_update3d<GEO, T><<<grid, kUThreads, smem, stream>>>(A, out_by_slot, R);
    return e;
}

template <typename T>
static cudaError_t update_launch_t(const pfb_update_args3d& A, int out_by_slot, PoolRounding R, dim3 grid,
                                   size_t smem, cudaStream_t stream) {
    const uint32_t bf = A.layout.boundary_flags;
    if (periodic_xyz(bf)) return update_launch_gt<0, T>(A, out_by_slot, R, grid, smem, stream);
    if (substrate_slab(bf)) return update_launch_gt<1, T>(A, out_by_slot, R, grid, smem, stream);
    return update_launch_gt<2, T>(A, out_by_slot, R, grid, smem, stream);
}

static int update_launch(const pfb_update_args3d& A, int out_by_slot, int storage, PoolRounding R,
                         cudaStream_t stream) {
    const int count = A.selection.ids ? A.selection.count : A.N;
    if (count == 0) return PFB_OK;
    const size_t smem = update3d_smem(A.B, storage ? 2 : 4);
    if (smem > 227 * 1024) return set_error(PFB_E_CONFIG, "brick edge too large for the plane ring");
    const dim3 grid((unsigned)(count * kUCtasPerCell));
    cudaError_t e;
    if (storage == kStoreF16)
        e = update_launch_t<__half>(A, out_by_slot, R, grid, smem, stream);
    else if (storage == kStoreBF16)
        e = update_launch_t<__nv_bfloat16>(A, out_by_slot, R, grid, smem, stream);
    else
        e = update_launch_t<float>(A, out_by_slot, R, grid, smem, stream);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(PFB_E_CUDA, "update launch: %s", cudaGetErrorString(e));
    return PFB_OK;
}

int update3d_launch(const pfb_update_args3d* a, cudaStream_t stream) {
    return update3d_launch_pool(a, kStoreF32, nullptr, 0, stream);
}

int update3d_launch_pool(const pfb_update_args3d* a, int storage, const uint64_t* step, uint64_t seed,
                         cudaStream_t stream) {
    const int rc = check_update(a);
    if (rc) return rc;
    if (storage < kStoreF32 || storage > kStoreBF16) return set_error(PFB_E_ARG, "unknown phi storage");
    return update_launch(*a, 0, storage, PoolRounding{step, seed}, stream);
}

// In-place commit: the scratch brick of selection slot k becomes cell
// ids[k]'s field unless the cell or the step holds a fatal flag, in which
// case the field stays and the planned shift is dropped (reference
// k_update_inplace_impl, src/pf3d/kernels.cu:1996-2045).
__global__ void k_commit3d(void* pool, const void* scratch, pfb_cell3d* cells, const uint32_t* g,
                           const int* ids, int B, int bytes) {
    __shared__ int keep;
    const int k = (int)blockIdx.x;
    const int n = ids[k];
    pfb_cell3d* cell = &cells[n];
    if (cell->storage_edge > (uint32_t)B) return;
    if (threadIdx.x == 0) {
        keep = fatal3(cell, g) ? 1 : 0;
        if (keep) {
            cell->pending_shift_x = 0;
            cell->pending_shift_y = 0;
            cell->pending_shift_z = 0;
        }
    }
    __syncthreads();
    if (keep) return;
    const size_t brick = (size_t)B * B * B * bytes;
    const float4* s4 = reinterpret_cast<const float4*>(static_cast<const char*>(scratch) + (size_t)k * brick);
    float4* d4 = reinterpret_cast<float4*>(static_cast<char*>(pool) + (size_t)n * brick);
    for (size_t i = threadIdx.x; i < brick / 16; i += blockDim.x) d4[i] = s4[i];
}

// The in-place update of the reference's balanced and compact modes
// (launch_update_inplace[_fast]): the selected cells, `slots` at a time,
// update from the single pool A.phi_in into the scratch bricks, then commit.
// A.phi_out is ignored; A.S_out may be null (compact: the caller rebuilds S).
int update3d_inplace_launch(const pfb_update_args3d* a, float* scratch, int slots,
                            cudaStream_t stream) {
    return update3d_inplace_launch_pool(a, scratch, slots, kStoreF32, nullptr, 0, stream);
}

int update3d_inplace_launch_pool(const pfb_update_args3d* a, void* scratch, int slots, int storage,
                                 const uint64_t* step, uint64_t seed, cudaStream_t stream) {
    if (!a) return set_error(PFB_E_ARG, "null update arguments");
    if (!scratch || slots <= 0 || ((uintptr_t)scratch & 15u))
        return set_error(PFB_E_ARG, "in-place update needs aligned scratch bricks");
    pfb_update_args3d A = *a;
    A.phi_out = static_cast<float*>(scratch);
    int rc = check_update(&A, false);
    if (rc) return rc;
    if (!A.phi_in || ((uintptr_t)A.phi_in & 15u)) return set_error(PFB_E_ARG, "invalid phi pool");
    const int count = A.selection.ids ? A.selection.count : A.N;
    std::vector<int> identity;
    const int* ids = A.selection.ids;
    int* d_ids = nullptr;
    if (!ids) {
        // no selection: every cell in id order
        identity.resize((size_t)count);
        for (int i = 0; i < count; ++i) identity[(size_t)i] = i;
        if (cudaMalloc(&d_ids, identity.size() * sizeof(int)) != cudaSuccess ||
            cudaMemcpyAsync(d_ids, identity.data(), identity.size() * sizeof(int), cudaMemcpyHostToDevice,
                            stream) != cudaSuccess) {
            cudaFree(d_ids);
            return set_error(PFB_E_CUDA, "in-place id list");
        }
        ids = d_ids;
    }
    for (int b0 = 0; b0 < count && !rc; b0 += slots) {
        const int nb = count - b0 < slots ? count - b0 : slots;
        A.selection.ids = ids + b0;
        A.selection.count = nb;
        rc = update_launch(A, 1, storage, PoolRounding{step, seed}, stream);
        if (!rc) {
            k_commit3d<<<nb, 256, 0, stream>>>(a->phi_in, scratch, A.cells, A.global_flags, ids + b0, A.B,
                                               storage ? 2 : 4);
            const cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) rc = set_error(PFB_E_CUDA, "in-place commit: %s", cudaGetErrorString(e));
        }
    }
    if (d_ids) {
        cudaStreamSynchronize(stream);
        cudaFree(d_ids);
    }
    return rc;
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

extern "C" int pfb3d_update_inplace(const pfb_update_args3d* args, float* scratch, int scratch_slots,
                                    void* stream) {
    return pfb::p3::update3d_inplace_launch(args, scratch, scratch_slots,
                                            static_cast<cudaStream_t>(stream));
}
