// 3D step sequencing and initialisation kernels (sm_100a): aggregate clear,
// fatal-step repair, origin finalisation, accepted-state restore, step
// counter, sphere seeding and the full scatter. Semantics follow the
// reference (src/pf3d/kernels.cu:1071-1186 and :2128-2321); the repair is
// split into a clear launch and a per-cell launch instead of one CTA.
#include <cuda_runtime.h>

#include "pfb3d_common.cuh"
#include "pfb_internal.h"
#include "phi3d.cuh"

namespace pfb {
namespace p3 {

int geometry_ok3(int B, const pfb_layout3d& L);

__device__ __forceinline__ void raise1(pfb_cell3d* cell, uint32_t* gflags, int flag) {
    atomicOr(&cell->flags, 1u << flag);
    if (gflags) atomicAdd(&gflags[flag], 1u);
}

__device__ __forceinline__ bool fatal_global(const uint32_t* g) {
    if (!g) return false;
    for (int f = 0; f < PFB3D_FLAG_COUNT; ++f)
        if (((PFB3D_FATAL_MASK >> f) & 1u) && g[f]) return true;
    return false;
}

// Q5.27 contribution of one value with the clamp and overflow flags.
__device__ __forceinline__ void scatter_one(uint32_t* S, size_t i, float v, pfb_cell3d* cell,
                                            uint32_t* g) {
    if (v * v > kQClamp3) raise1(cell, g, PFB3D_FLAG_Q_CLAMP);
    const uint32_t q = q_of3(v);
    if (!q) return;
    const uint32_t old = atomicAdd(&S[i], q);
    if (old > 0xFFFFFFFFu - q) raise1(cell, g, PFB3D_FLAG_S_OVERFLOW);
}

__global__ void k_clear3d(uint4* S, size_t vec4, uint32_t* tail, size_t tail_words,
                          const uint32_t* guard) {
    if (guard && !fatal_global(guard)) return;
    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < vec4; i += stride)
        __stcs(S + i, z);
    if (blockIdx.x == 0)
        for (size_t i = threadIdx.x; i < tail_words; i += blockDim.x) tail[i] = 0u;
}

// Scatter every selected cell's field: one CTA per cell, one warp per brick
// row. T: storage type of the pool.
template <typename T>
__global__ void k_scatter3d(const T* phi, pfb_cell3d* cells, uint32_t* S, uint32_t* g,
                            pfb_layout3d L, int N, int B, pfb_selection3d sel, int guard_fatal) {
    if (guard_fatal && !fatal_global(g)) return;
    const int slot = (int)blockIdx.x;
    const int n = sel.ids ? sel.ids[slot] : slot;
    pfb_cell3d* cell = &cells[n];
    if (cell->storage_edge != 0u) return;
    const T* tile = phi + (size_t)n * B * B * B;
    const int ox = wrap_origin(cell->origin_x, L.nx), oy = wrap_origin(cell->origin_y, L.ny);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    for (int row = warp; row < B * B; row += warps) {
        const int z = row / B, y = row - z * B;
        int wz;
        if (!aggregate_z(L, cell->origin_z, z, &wz)) continue;
        const size_t base = s_index(L, 0, wrap_offset(oy, y, L.ny), wz);
        const T* gr = tile + (size_t)row * B;
        for (int x = lane; x < B; x += 32) {
            const float v = phi_ld1(gr + x);
            if (!isfinite(v)) {
                raise1(cell, g, PFB3D_FLAG_NONFINITE);
                continue;
            }
            scatter_one(S, base + wrap_offset(ox, x, L.nx), v, cell, g);
        }
    }
}

// Fatal-step repair of one cell: phi_out = phi_in (values of `bytes` each),
// pending shift cleared.
__global__ void k_repair_copy3d(const void* in, void* out, pfb_cell3d* cells, const uint32_t* g,
                                int B, int bytes, pfb_selection3d sel) {
    if (!fatal_global(g)) return;
    const int slot = (int)blockIdx.x;
    const int n = sel.ids ? sel.ids[slot] : slot;
    pfb_cell3d* cell = &cells[n];
    if (cell->storage_edge != 0u) return;
    const size_t brick = (size_t)B * B * B * bytes;
    const float4* s4 = reinterpret_cast<const float4*>(static_cast<const char*>(in) + (size_t)n * brick);
    float4* d4 = reinterpret_cast<float4*>(static_cast<char*>(out) + (size_t)n * brick);
    for (size_t i = threadIdx.x; i < brick / 16; i += blockDim.x) d4[i] = s4[i];
    if (threadIdx.x == 0) {
        cell->pending_shift_x = 0;
        cell->pending_shift_y = 0;
        cell->pending_shift_z = 0;
    }
}

__global__ void k_finalize3d(pfb_cell3d* cells, int N, uint32_t* g) {
    const int n = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (n >= N) return;
    pfb_cell3d* c = &cells[n];
    if (c->flags & PFB3D_FATAL_MASK) {
        c->pending_shift_x = c->pending_shift_y = c->pending_shift_z = 0;
        return;
    }
    const int sx = c->pending_shift_x, sy = c->pending_shift_y, sz = c->pending_shift_z;
    const int64_t mx = INT64_MAX, mn = INT64_MIN;
    auto bad = [&](int64_t o, int s) {
        return (s > 0 && o > mx - s) || (s < 0 && o < mn - s);
    };
    if (bad(c->origin_x, sx) || bad(c->origin_y, sy) || bad(c->origin_z, sz)) {
        raise1(c, g, PFB3D_FLAG_INVALID_GEOMETRY);
        c->pending_shift_x = c->pending_shift_y = c->pending_shift_z = 0;
        return;
    }
    c->origin_x += sx;
    c->origin_y += sy;
    c->origin_z += sz;
    if (sx || sy || sz) ++c->shift_ctr;
    c->pending_shift_x = c->pending_shift_y = c->pending_shift_z = 0;
}

__global__ void k_restore3d(pfb_cell3d* cells, const pfb_cell3d* acc, int N, const uint32_t* g,
                            uint32_t* requests) {
    if (!fatal_global(g)) return;
    const int n = (int)(blockIdx.x * blockDim.x + threadIdx.x);
    if (n >= N) return;
    if ((cells[n].flags & (1u << PFB3D_FLAG_SUPPORT_EXHAUSTED)) && requests) requests[n] = 1u;
    cells[n] = acc[n];
}

__global__ void k_advance3d(uint64_t* step, const uint32_t* g) {
    if (!fatal_global(g)) ++*step;
}

__global__ void k_init_spheres3d(const __grid_constant__ pfb_init_args3d A) {
    const int n = (int)blockIdx.x;
    const int B = A.B;
    const size_t words = (size_t)B * B * B;
    pfb_cell3d* c = &A.cells[n];
    const pfb_vec3 ctr = A.centres[n];
    __shared__ int64_t org[3];
    if (threadIdx.x == 0) {
        const double half = 0.5 * (double)(B - 1);
        c->origin_x = __double2ll_rn(ctr.x - half);
        c->origin_y = __double2ll_rn(ctr.y - half);
        c->origin_z = __double2ll_rn(ctr.z - half);
        c->shift_ctr = c->tumble_ctr = 0u;
        c->flags = 0u;
        c->pad0 = c->pad1 = c->pad2 = 0u;
        c->pending_shift_x = c->pending_shift_y = c->pending_shift_z = 0;
        c->V = c->Cx = c->Cy = c->Cz = 0.0;
        c->surface = c->Ix = c->Iy = c->Iz = 0.0;
        c->wall_overlap = c->outside_slit_volume = 0.0;
        c->phi_max = 0.0f;
        for (int i = 0; i < 10; ++i) c->reserved[i] = 0u;
        org[0] = c->origin_x;
        org[1] = c->origin_y;
        org[2] = c->origin_z;
    }
    __syncthreads();
    float* even = A.phi_even + (size_t)n * words;
    float* odd = A.phi_odd ? A.phi_odd + (size_t)n * words : nullptr;
    const float k = iface_k(A.lambda);
    for (size_t q = threadIdx.x; q < words; q += blockDim.x) {
        const int x = (int)(q % B), y = (int)((q / B) % B), z = (int)(q / ((size_t)B * B));
        int wz;
        const bool in_domain = aggregate_z(A.layout, org[2], z, &wz);
        const double dx = (double)(org[0] + x) - ctr.x;
        const double dy = (double)(org[1] + y) - ctr.y;
        const double dz = (double)(org[2] + z) - ctr.z;
        const float r = (float)sqrt(dx * dx + dy * dy + dz * dz);
        even[q] = in_domain ? 0.5f * (1.0f - tanhf(k * (r - A.seed_radius))) : 0.0f;
        if (odd) odd[q] = 0.0f;
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
static int sel_count(const pfb_selection3d& s, int N) { return s.ids ? s.count : N; }

int clear3d_launch(uint32_t* S, const pfb_layout3d* L, const uint32_t* guard,
                   cudaStream_t stream) {
    if (!S || !L) return set_error(PFB_E_ARG, "null aggregate or layout");
    const size_t words = (size_t)L->pitch_x * L->ny * L->nz;
    if (words == 0) return PFB_OK;
    const size_t vec4 = ((uintptr_t)S & 15u) ? 0 : words / 4;
    uint32_t* tail = S + vec4 * 4;
    const size_t tail_words = words - vec4 * 4;
    const int blocks = (int)std::min<size_t>(148 * 8, (vec4 + 255) / 256 + 1);
    k_clear3d<<<blocks, 256, 0, stream>>>(reinterpret_cast<uint4*>(S), vec4, tail, tail_words, guard);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "clear launch: %s", cudaGetErrorString(e));
}

template <typename T>
static void scatter_t(const void* phi, const pfb_scatter_args3d& A, uint32_t* S, int count, int guard,
                      cudaStream_t stream) {
    k_scatter3d<T><<<count, 256, 0, stream>>>(static_cast<const T*>(phi), A.cells, S, A.global_flags,
                                              A.layout, A.N, A.B, A.selection, guard);
}

static void scatter_pool(int storage, const void* phi, const pfb_scatter_args3d& A, uint32_t* S, int count,
                         int guard, cudaStream_t stream) {
    if (storage == kStoreF16)
        scatter_t<__half>(phi, A, S, count, guard, stream);
    else if (storage == kStoreBF16)
        scatter_t<__nv_bfloat16>(phi, A, S, count, guard, stream);
    else
        scatter_t<float>(phi, A, S, count, guard, stream);
}

int scatter3d_launch(const pfb_scatter_args3d* a, cudaStream_t stream) {
    return scatter3d_launch_pool(a, kStoreF32, stream);
}

int scatter3d_launch_pool(const pfb_scatter_args3d* a, int storage, cudaStream_t stream) {
    if (!a) return set_error(PFB_E_ARG, "null scatter arguments");
    const pfb_scatter_args3d& A = *a;
    if (A.storage.z_cap != 0) return set_error(PFB_E_CONFIG, "compact cell storage is not supported");
    if (!geometry_ok3(A.B, A.layout) || A.N <= 0 || !A.phi || !A.cells || !A.S ||
        (A.selection.ids && (A.selection.count < 0 || A.selection.count > A.N)))
        return set_error(PFB_E_ARG, "invalid scatter arguments");
    const int count = sel_count(A.selection, A.N);
    if (count == 0) return PFB_OK;
    scatter_pool(storage, A.phi, A, A.S, count, 0, stream);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "scatter launch: %s", cudaGetErrorString(e));
}

int repair3d_launch(const pfb_update_args3d* a, cudaStream_t stream) {
    return repair3d_launch_pool(a, kStoreF32, stream);
}

int repair3d_launch_pool(const pfb_update_args3d* a, int storage, cudaStream_t stream) {
    if (!a) return set_error(PFB_E_ARG, "null update arguments");
    const pfb_update_args3d& A = *a;
    if (A.storage.z_cap != 0) return set_error(PFB_E_CONFIG, "compact cell storage is not supported");
    if (!geometry_ok3(A.B, A.layout) || A.N <= 0 || !A.phi_in || !A.cells || !A.global_flags ||
        (A.selection.ids && (A.selection.count < 0 || A.selection.count > A.N)))
        return set_error(PFB_E_ARG, "invalid repair arguments");
    const int count = sel_count(A.selection, A.N);
    if (A.S_out) {
        const int rc = clear3d_launch(A.S_out, &A.layout, A.global_flags, stream);
        if (rc) return rc;
    }
    if (count > 0 && A.phi_out)
        k_repair_copy3d<<<count, 256, 0, stream>>>(A.phi_in, A.phi_out, A.cells, A.global_flags,
                                                   A.B, storage ? 2 : 4, A.selection);
    if (count > 0 && A.S_out) {
        pfb_scatter_args3d sa{};
        sa.cells = A.cells;
        sa.global_flags = A.global_flags;
        sa.layout = A.layout;
        sa.N = A.N;
        sa.B = A.B;
        sa.selection = A.selection;
        scatter_pool(storage, A.phi_in, sa, A.S_out, count, 1, stream);
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "repair launch: %s", cudaGetErrorString(e));
}

int init3d_launch(const pfb_init_args3d* a, cudaStream_t stream) {
    if (!a) return set_error(PFB_E_ARG, "null init arguments");
    const pfb_init_args3d& A = *a;
    if (A.storage.z_cap != 0) return set_error(PFB_E_CONFIG, "compact cell storage is not supported");
    if (A.N <= 0 || !A.phi_even || !A.cells || !A.centres || !geometry_ok3(A.B, A.layout) ||
        !(A.lambda > 0.0f) || !(A.seed_radius > 0.0f))
        return set_error(PFB_E_ARG, "invalid init arguments");
    k_init_spheres3d<<<A.N, 256, 0, stream>>>(A);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : set_error(PFB_E_CUDA, "init launch: %s", cudaGetErrorString(e));
}

}  // namespace p3
}  // namespace pfb

using namespace pfb::p3;

extern "C" {

int pfb3d_clear_S(uint32_t* S, const pfb_layout3d* layout, void* stream) {
    return clear3d_launch(S, layout, nullptr, static_cast<cudaStream_t>(stream));
}

int pfb3d_repair_after_fatal(const pfb_update_args3d* args, void* stream) {
    return repair3d_launch(args, static_cast<cudaStream_t>(stream));
}

int pfb3d_finalize_origins(pfb_cell3d* cells, int N, uint32_t* global_flags, void* stream) {
    if (!cells || N <= 0) return pfb::set_error(PFB_E_ARG, "invalid finalize arguments");
    k_finalize3d<<<(N + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(cells, N,
                                                                               global_flags);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : pfb::set_error(PFB_E_CUDA, "finalize: %s", cudaGetErrorString(e));
}

int pfb3d_restore_cells_after_fatal(pfb_cell3d* cells, const pfb_cell3d* accepted, int N,
                                    const uint32_t* global_flags, uint32_t* support_requests,
                                    void* stream) {
    if (!cells || !accepted || N <= 0 || !global_flags)
        return pfb::set_error(PFB_E_ARG, "invalid restore arguments");
    k_restore3d<<<(N + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        cells, accepted, N, global_flags, support_requests);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : pfb::set_error(PFB_E_CUDA, "restore: %s", cudaGetErrorString(e));
}

int pfb3d_advance_step(uint64_t* step, const uint32_t* global_flags, void* stream) {
    if (!step) return pfb::set_error(PFB_E_ARG, "null step counter");
    k_advance3d<<<1, 1, 0, static_cast<cudaStream_t>(stream)>>>(step, global_flags);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PFB_OK : pfb::set_error(PFB_E_CUDA, "advance: %s", cudaGetErrorString(e));
}

int pfb3d_initialize_spheres(const pfb_init_args3d* args, void* stream) {
    return init3d_launch(args, static_cast<cudaStream_t>(stream));
}

int pfb3d_scatter_current(const pfb_scatter_args3d* args, void* stream) {
    return scatter3d_launch(args, static_cast<cudaStream_t>(stream));
}

}  // extern "C"
