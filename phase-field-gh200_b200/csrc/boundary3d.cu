// PFB3D boundary recorder of the 3D system: projected half-height contours
// (reference src/pf3d/boundary_output.cu, include/pf3d/boundary_output.cuh,
// common/boundary_format_3d.h).
//
// Each cell's B^3 brick is projected to a (B+2)^2 plane with a zero ring
// around its x/y faces: the maximum over the brick's in-domain z planes
// (projection "maximum"), or the single plane on the substrate (projection
// "basal", substrate slab only). A frame holds every cell's 64-byte record
// (id, plane origin = brick origin - 1 in x/y, brick and plane edges, square
// count, gamma, active speed, target radius) followed by the cells' squares:
// the 2x2 plane squares that phi = 1/2 crosses, binary32 corners, in
// ascending plane order. Frames carry the FNV-1a 64 of their payload; a
// complete file ends with an end record.
//
// All cells are projected, counted and gathered by three launches per frame
// (one CTA per cell for the count and the gather) rather than per cell.
#include <cuda_runtime.h>

#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <unordered_set>
#include <vector>

#include "device_util.cuh"
#include "pfb200_3d.h"
#include "pfb200_ckpt.h"
#include "pfb_internal.h"

namespace pfb {
namespace {

constexpr int kB3Threads = 256;
constexpr int kProjBasal = 1, kProjMaximum = 2;

#pragma pack(push, 1)
struct B3Header {
    char magic[8];
    uint32_t version, header_bytes, cells, projection, boundary_flags, codec;
    int64_t nx, ny, nz;
    double dx, dy, dz, dt, tau, level;
    uint64_t interval;
    uint32_t square_bytes, cell_bytes;
    uint64_t reserved;
};
struct B3Frame {
    char magic[8];
    uint64_t step;
    double time;
    uint64_t raw_bytes, stored_bytes, checksum;
};
struct B3Cell {
    int64_t id, origin_x, origin_y, origin_z;
    uint32_t brick_edge, plane_edge, squares, reserved;
    float gamma, active_speed, radius, reserved_float;
};
struct B3Square {
    uint32_t xy;
    float phi[4];
};
#pragma pack(pop)
static_assert(sizeof(B3Header) == 128 && sizeof(B3Frame) == 48, "PFB3D headers");
static_assert(sizeof(B3Cell) == 64 && sizeof(B3Square) == 20, "PFB3D records");

// The brick planes a projection reads (reference projection_z_range):
// [z0, z1) in brick coordinates, empty when the brick misses the domain.
__device__ __forceinline__ void z_range(int64_t oz, int B, int nz, bool periodic, int projection,
                                        int* z0, int* z1) {
    *z0 = 0;
    *z1 = B;
    if (projection == kProjBasal) {
        if (oz > 0 || oz <= -(int64_t)B) {
            *z1 = 0;
        } else {
            *z0 = (int)(-oz);
            *z1 = *z0 + 1;
        }
        return;
    }
    if (periodic) return;
    if (oz >= nz || oz <= -(int64_t)B) {
        *z1 = 0;
        return;
    }
    if (oz < 0) *z0 = (int)(-oz);
    *z1 = (int)min((int64_t)B, (int64_t)nz - oz);
}

// grid (plane blocks, N): plane of cell n (edge pe[n] = E + 2 for its cube
// of edge E, at slot n of stride PS^2); status[n] = 1 on a non-finite
// sample. A cell's cube is cubes[n] when it has one, else its slot of the
// base pool (edge B).
__global__ void __launch_bounds__(kB3Threads)
    k_b3_project(const float* phi, float* const* cubes, const pfb_cell3d* cells, int B0,
                 const int* pe, int PS, int nz, int periodic, int projection, float* plane,
                 uint32_t* status) {
    const int n = blockIdx.y;
    const int PE = pe[n], B = PE - 2;
    const int q = blockIdx.x * kB3Threads + threadIdx.x;
    if (q >= PE * PE) return;
    const int x = q % PE, y = q / PE;
    float* out = plane + (size_t)n * PS * PS;
    out[q] = 0.0f;
    if (x == 0 || y == 0 || x == PE - 1 || y == PE - 1) return;
    int z0, z1;
    z_range(cells[n].origin_z, B, nz, periodic != 0, projection, &z0, &z1);
    if (z0 >= z1) return;
    const size_t slab = (size_t)B * B;
    const float* brick = (cubes && cubes[n]) ? cubes[n] : phi + (size_t)n * B0 * B0 * B0;
    const float* src = brick + ((size_t)z0 * B + (y - 1)) * B + (x - 1);
    float v = src[0];
    bool bad = !isfinite(v);
    for (int z = z0 + 1; z < z1; ++z) {
        src += slab;
        const float s = *src;
        bad |= !isfinite(s);
        if (s > v) v = s;
    }
    out[q] = v;
    if (bad) atomicOr(status + n, 1u);
}

__device__ __forceinline__ bool plane_square(const float* p, int PE, int q, B3Square* s) {
    const int x = q % (PE - 1), y = q / (PE - 1);
    const size_t at = (size_t)y * PE + x;
    s->xy = (uint32_t)x | ((uint32_t)y << 16);
    s->phi[0] = p[at];
    s->phi[1] = p[at + 1];
    s->phi[2] = p[at + PE + 1];
    s->phi[3] = p[at + PE];
    const bool in = s->phi[0] >= 0.5f;
    return (s->phi[1] >= 0.5f) != in || (s->phi[2] >= 0.5f) != in || (s->phi[3] >= 0.5f) != in;
}

__global__ void __launch_bounds__(kB3Threads)
    k_b3_count(const float* plane, const int* pe, int PS, uint32_t* counts) {
    const int n = blockIdx.x;
    const int PE = pe[n];
    const float* p = plane + (size_t)n * PS * PS;
    const int squares = (PE - 1) * (PE - 1);
    unsigned c = 0;
    for (int q = threadIdx.x; q < squares; q += kB3Threads) {
        B3Square s;
        c += plane_square(p, PE, q, &s) ? 1u : 0u;
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    __shared__ unsigned wc[kB3Threads / 32];
    if ((threadIdx.x & 31) == 0) wc[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned t = 0;
        for (int w = 0; w < kB3Threads / 32; ++w) t += wc[w];
        counts[n] = t;
    }
}

// Squares of cell n in ascending plane order from out[offsets[n]].
__global__ void __launch_bounds__(kB3Threads)
    k_b3_gather(const float* plane, const int* pe, int PS, const uint64_t* offsets, B3Square* out) {
    const int n = blockIdx.x, t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int PE = pe[n];
    const float* p = plane + (size_t)n * PS * PS;
    const int squares = (PE - 1) * (PE - 1);
    __shared__ unsigned wsum[kB3Threads / 32];
    B3Square* dst = out + offsets[n];
    unsigned base = 0;
    for (int q0 = 0; q0 < squares; q0 += kB3Threads) {
        const int q = q0 + t;
        B3Square s;
        const bool hit = q < squares && plane_square(p, PE, q, &s);
        const unsigned mask = __ballot_sync(0xFFFFFFFFu, hit);
        if (lane == 0) wsum[warp] = __popc(mask);
        __syncthreads();
        unsigned before = 0, total = 0;
        for (int w = 0; w < kB3Threads / 32; ++w) {
            before += w < warp ? wsum[w] : 0u;
            total += wsum[w];
        }
        if (hit) dst[base + before + __popc(mask & ((1u << lane) - 1u))] = s;
        base += total;
        __syncthreads();
    }
}

uint64_t fnv1a64(const unsigned char* p, size_t n) {
    uint64_t h = 14695981039346656037ull;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ull;
    }
    return h;
}

bool finite_positive(double v) { return std::isfinite(v) && v > 0.0; }

}  // namespace

struct Boundary3D {
    std::FILE* f = nullptr;
    int N = 0, nz = 0, projection = kProjMaximum;
    bool periodic = true, failed = false;
    uint64_t frames = 0, last_step = 0;
    double last_time = 0.0;
    float* d_plane = nullptr;
    size_t plane_cap = 0;
    uint32_t* d_status = nullptr;  // N status words, then N counts
    uint64_t* d_off = nullptr;
    int* d_pe = nullptr;  // plane edge of each cell
    B3Square* d_sq = nullptr;
    size_t sq_cap = 0;
    std::vector<pfb_cell3d> cells;
    std::vector<uint32_t> status;
    std::vector<uint64_t> off;
    std::vector<int> pe;
    std::vector<unsigned char> payload;

    ~Boundary3D() {
        if (f) std::fclose(f);  // no end record: the file stays unterminated
        cudaFree(d_plane);
        cudaFree(d_status);
        cudaFree(d_off);
        cudaFree(d_pe);
        cudaFree(d_sq);
    }

    int fail(int code, const char* what) {
        failed = true;
        return set_error(code, "boundary3d: %s", what);
    }

    int capture(const float* phi, float* const* cubes, const pfb_cell3d* d_cells, int B,
                cudaStream_t stream, long long step, double time) {
        if (failed || !f) return set_error(PFB_E_STATE, "boundary3d: no open file");
        if (B <= 0 || B > 65532 || !std::isfinite(time) || time < 0.0 ||
            (frames > 0 && ((uint64_t)step <= last_step || time < last_time)))
            return fail(PFB_E_ARG, "invalid brick edge or frame order");
        cudaError_t e = cudaMemcpyAsync(cells.data(), d_cells, (size_t)N * sizeof(pfb_cell3d),
                                        cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) return fail(PFB_E_CUDA, cudaGetErrorString(e));
        std::unordered_set<int64_t> ids;
        int PS = 0;
        for (int i = 0; i < N; ++i) {
            const pfb_cell3d& c = cells[(size_t)i];
            // a cube edge per cell (reference cell_support_edge)
            const int E = (cubes && c.storage_edge > (uint32_t)B) ? (int)c.storage_edge : B;
            pe[(size_t)i] = E + 2;
            PS = std::max(PS, E + 2);
            const int64_t hi = std::numeric_limits<int64_t>::max() - E;
            const bool ok = (c.storage_edge == 0 || c.storage_edge == (uint32_t)B ||
                             (cubes && c.storage_edge > (uint32_t)B && c.storage_edge <= 65532u)) &&
                            c.global_id >= 0 &&
                            c.origin_x > std::numeric_limits<int64_t>::min() &&
                            c.origin_y > std::numeric_limits<int64_t>::min() && c.origin_x <= hi &&
                            c.origin_y <= hi && c.origin_z <= hi && finite_positive(c.gamma) &&
                            finite_positive(c.R_tgt) && std::isfinite(c.v_A) && c.v_A >= 0.0f &&
                            ids.insert(c.global_id).second;
            if (!ok) return fail(PFB_E_STATE, "invalid or duplicate cell metadata");
        }
        const size_t plane = (size_t)N * PS * PS;
        if (plane > plane_cap) {
            cudaFree(d_plane);
            d_plane = nullptr;
            if (cudaMalloc(&d_plane, plane * sizeof(float)) != cudaSuccess)
                return fail(PFB_E_CUDA, "plane allocation failed");
            plane_cap = plane;
        }
        if ((e = cudaMemsetAsync(d_status, 0, (size_t)N * sizeof(uint32_t), stream)) != cudaSuccess ||
            (e = cudaMemcpyAsync(d_pe, pe.data(), (size_t)N * sizeof(int), cudaMemcpyHostToDevice,
                                 stream)) != cudaSuccess)
            return fail(PFB_E_CUDA, cudaGetErrorString(e));
        const dim3 grid((unsigned)((PS * PS + kB3Threads - 1) / kB3Threads), (unsigned)N);
        k_b3_project<<<grid, kB3Threads, 0, stream>>>(phi, cubes, d_cells, B, d_pe, PS, nz,
                                                        periodic ? 1 : 0, projection, d_plane, d_status);
        k_b3_count<<<N, kB3Threads, 0, stream>>>(d_plane, d_pe, PS, d_status + N);
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpyAsync(status.data(), d_status, 2 * (size_t)N * sizeof(uint32_t),
                                 cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
            (e = cudaStreamSynchronize(stream)) != cudaSuccess)
            return fail(PFB_E_CUDA, cudaGetErrorString(e));
        uint64_t total = 0;
        for (int i = 0; i < N; ++i) {
            if (status[(size_t)i]) return fail(PFB_E_STATE, "non-finite projected sample");
            off[(size_t)i] = total;
            total += status[(size_t)N + i];
        }
        const size_t prefix = (size_t)N * sizeof(B3Cell);
        payload.resize(prefix + (size_t)total * sizeof(B3Square));
        for (int i = 0; i < N; ++i) {
            const pfb_cell3d& c = cells[(size_t)i];
            B3Cell r{};
            r.id = c.global_id;
            r.origin_x = c.origin_x - 1;
            r.origin_y = c.origin_y - 1;
            r.origin_z = c.origin_z;
            r.brick_edge = (uint32_t)(pe[(size_t)i] - 2);
            r.plane_edge = (uint32_t)pe[(size_t)i];
            r.squares = status[(size_t)N + i];
            r.gamma = c.gamma;
            r.active_speed = c.v_A;
            r.radius = c.R_tgt;
            std::memcpy(payload.data() + (size_t)i * sizeof(B3Cell), &r, sizeof(r));
        }
        if (total > 0) {
            if (total > sq_cap) {
                cudaFree(d_sq);
                d_sq = nullptr;
                sq_cap = (size_t)(total + total / 8 + 256);
                if (cudaMalloc(&d_sq, sq_cap * sizeof(B3Square)) != cudaSuccess)
                    return fail(PFB_E_CUDA, "square allocation failed");
            }
            if ((e = cudaMemcpyAsync(d_off, off.data(), (size_t)N * sizeof(uint64_t),
                                     cudaMemcpyHostToDevice, stream)) != cudaSuccess)
                return fail(PFB_E_CUDA, cudaGetErrorString(e));
            k_b3_gather<<<N, kB3Threads, 0, stream>>>(d_plane, d_pe, PS, d_off, d_sq);
            if ((e = cudaGetLastError()) != cudaSuccess ||
                (e = cudaMemcpyAsync(payload.data() + prefix, d_sq, (size_t)total * sizeof(B3Square),
                                     cudaMemcpyDeviceToHost, stream)) != cudaSuccess ||
                (e = cudaStreamSynchronize(stream)) != cudaSuccess)
                return fail(PFB_E_CUDA, cudaGetErrorString(e));
        }
        B3Frame h{};
        std::memcpy(h.magic, "P3BFRM1", 8);
        h.step = (uint64_t)step;
        h.time = time;
        h.raw_bytes = h.stored_bytes = payload.size();
        h.checksum = fnv1a64(payload.data(), payload.size());
        if (std::fwrite(&h, sizeof(h), 1, f) != 1 ||
            std::fwrite(payload.data(), 1, payload.size(), f) != payload.size() || std::fflush(f) != 0)
            return fail(PFB_E_IO, "write failed");
        ++frames;
        last_step = (uint64_t)step;
        last_time = time;
        return PFB_OK;
    }
};

Boundary3D* boundary3d_open(const char* path, const pfb_params3d& p, int projection,
                            long long interval, int compress) {
    const bool slab = p.boundary_flags == PFB3D_BOUNDARY_SUBSTRATE_SLAB;
    const bool known = p.boundary_flags == PFB3D_BOUNDARY_PERIODIC_XYZ || slab ||
                       p.boundary_flags == PFB3D_BOUNDARY_HARD_WALL_CHANNEL;
    if (!path || !path[0] || p.num_cells <= 0 || p.Nx <= 0 || p.Ny <= 0 || p.Nz <= 0 || !known ||
        !(projection == kProjMaximum || (projection == kProjBasal && slab)) || interval <= 0 ||
        !finite_positive(p.dt) || !finite_positive(p.tau)) {
        set_error(PFB_E_ARG, "boundary3d: invalid output geometry, projection, or cadence");
        return nullptr;
    }
    if (compress) {
        set_error(PFB_E_CONFIG, "boundary3d: zstd unavailable; select --boundary-compression none");
        return nullptr;
    }
    Boundary3D* b = new Boundary3D();
    b->N = p.num_cells;
    b->nz = p.Nz;
    b->projection = projection;
    b->periodic = p.boundary_flags == PFB3D_BOUNDARY_PERIODIC_XYZ;
    b->cells.resize((size_t)b->N);
    b->status.resize(2 * (size_t)b->N);
    b->off.resize((size_t)b->N);
    b->pe.resize((size_t)b->N);
    if (cudaMalloc(&b->d_status, 2 * (size_t)b->N * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&b->d_off, (size_t)b->N * sizeof(uint64_t)) != cudaSuccess ||
        cudaMalloc(&b->d_pe, (size_t)b->N * sizeof(int)) != cudaSuccess) {
        delete b;
        set_error(PFB_E_CUDA, "boundary3d: allocation failed");
        return nullptr;
    }
    b->f = std::fopen(path, "wbx");  // a new file only
    if (!b->f) {
        set_error(PFB_E_IO, "boundary3d: cannot create new output file %s: %s", path, std::strerror(errno));
        delete b;
        return nullptr;
    }
    B3Header h{};
    std::memcpy(h.magic, "PFB3D1", 7);
    h.version = 1;
    h.header_bytes = sizeof(h);
    h.cells = (uint32_t)p.num_cells;
    h.projection = (uint32_t)projection;
    h.boundary_flags = p.boundary_flags;
    h.codec = 0;
    h.nx = p.Nx;
    h.ny = p.Ny;
    h.nz = p.Nz;
    h.dx = h.dy = h.dz = 1.0;
    h.dt = p.dt;
    h.tau = p.tau;
    h.level = 0.5;
    h.interval = (uint64_t)interval;
    h.square_bytes = sizeof(B3Square);
    h.cell_bytes = sizeof(B3Cell);
    if (std::fwrite(&h, sizeof(h), 1, b->f) != 1 || std::fflush(b->f) != 0) {
        set_error(PFB_E_IO, "boundary3d: header write failed");
        delete b;
        return nullptr;
    }
    return b;
}

int boundary3d_capture(Boundary3D* b, const float* phi, float* const* cubes, const pfb_cell3d* cells,
                       int B, cudaStream_t stream, long long step, double time) {
    return b->capture(phi, cubes, cells, B, stream, step, time);
}

int boundary3d_close(Boundary3D* b, int complete) {
    int rc = PFB_OK;
    if (b->f) {
        if (complete && !b->failed) {
            B3Frame end{};
            std::memcpy(end.magic, "P3BEND1", 8);
            end.step = b->last_step;
            end.time = b->last_time;
            if (std::fwrite(&end, sizeof(end), 1, b->f) != 1) rc = set_error(PFB_E_IO, "boundary3d: end record");
        }
        if (std::fclose(b->f) != 0) rc = set_error(PFB_E_IO, "boundary3d: close failed");
        b->f = nullptr;
    }
    if (b->failed && rc == PFB_OK) rc = set_error(PFB_E_IO, "boundary3d: the file is incomplete");
    delete b;
    return rc;
}

}  // namespace pfb
